"""The C ABI library: loads, exports every symbol of include/hislam2_b200.h, and the
host-side validation of the ops (no GPU needed: nothing here launches work)."""

import ctypes
import os
import re

import pytest
import torch

import droid_backends
from hislam2_b200 import _lib, backends

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "hislam2_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"(?:int|void|long long|const char\s*\*)\s+(hs2_\w+)\s*\(([^)]*)\)\s*;", text):
        params = [p for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        out[m.group(1)] = len(params)
    return out


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    decl = declared()
    assert len(decl) >= 11
    for name, nparams in decl.items():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name
        assert len(_lib.SIGNATURES[name]) == nparams, name
    assert lib.hs2_version() == (1 << 16)


def elf_needed(path):
    """DT_NEEDED entries of a 64-bit little-endian ELF shared object."""
    import struct
    data = open(path, "rb").read()
    assert data[:4] == b"\x7fELF" and data[4] == 2 and data[5] == 1
    shoff, = struct.unpack_from("<Q", data, 0x28)
    shentsize, shnum = struct.unpack_from("<HH", data, 0x3A)
    sections = [struct.unpack_from("<IIQQQQIIQQ", data, shoff + k * shentsize) for k in range(shnum)]
    dyn = next(s for s in sections if s[1] == 6)          # SHT_DYNAMIC
    strtab = sections[dyn[6]]                              # sh_link -> its string table
    out = []
    for off in range(dyn[4], dyn[4] + dyn[5], 16):
        tag, val = struct.unpack_from("<qQ", data, off)
        if tag == 0:
            break
        if tag == 1:                                       # DT_NEEDED
            start = strtab[4] + val
            out.append(data[start:data.index(b"\0", start)].decode())
    return out


def test_library_needs_no_shared_cuda_runtime():
    # cudart is linked statically (nvcc's default), so the library does not depend on, or clash
    # with, the CUDA runtime that PyTorch ships; the driver API is reached at run time instead
    needed = elf_needed(_lib.LIB_PATH)
    assert "libc.so.6" in needed
    assert not any(n.startswith(("libcudart", "libtorch", "libc10")) for n in needed), needed
    _lib.load()
    assert _lib.LIB_PATH in open("/proc/self/maps").read()


def test_workspace_size_validation():
    lib = _lib.load()
    n = ctypes.c_size_t(0)
    assert lib.hs2_ba_workspace_size(300, 300, 43, 77, 6000, 10, 300, 0, ctypes.byref(n)) == _lib.HS2_OK
    assert n.value > 6 * 6290 * 3311 * 4  # holds the E rows
    rc = lib.hs2_ba_workspace_size(300, 300, 43, 77, 6000, 10, 301, 0, ctypes.byref(n))
    assert rc == _lib.HS2_ERR_INVALID
    assert b"t1" in lib.hs2_last_error()
    assert lib.hs2_ba_workspace_size(8, 8, 0, 64, 10, 0, 8, 0, ctypes.byref(n)) == _lib.HS2_ERR_INVALID
    assert backends.ba_workspace_bytes(8, 8, 48, 64, 24, 2, 8, True) < backends.ba_workspace_bytes(
        8, 8, 48, 64, 24, 2, 8, False)


def test_pgba_workspace_size_validation():
    lib = _lib.load()
    n = ctypes.c_size_t(0)
    assert lib.hs2_pgba_workspace_size(300, 300, 43, 77, 6000, 10, 300, ctypes.byref(n)) == _lib.HS2_OK
    # holds the 7-plane E rows and the FP64 system of order 7 * 290 (even, no pad)
    assert n.value > 7 * 6290 * 3328 * 4 + 8 * 2030 * 2030
    m = ctypes.c_size_t(0)
    assert lib.hs2_pgba_workspace_size(300, 300, 43, 77, 6000, 11, 300, ctypes.byref(m)) == _lib.HS2_OK
    assert m.value >= 8 * 2024 * 2024   # order 7 * 289 = 2023 padded to 2024
    assert lib.hs2_pgba_workspace_size(300, 300, 43, 77, 6000, 10, 301, ctypes.byref(n)) == _lib.HS2_ERR_INVALID
    assert b"t1" in lib.hs2_last_error()


def test_corr_validation_before_any_launch():
    lib = _lib.load()
    rc = lib.hs2_corr_index_forward(None, _lib.HS2_F32, 1, 4, 4, 4, 4, None, -1, None, None)
    assert rc == _lib.HS2_ERR_INVALID
    rc = lib.hs2_altcorr_forward(None, None, _lib.HS2_F32, 1, 1, 1, 0, 4, 4, 4, 4, None, None, None, 1, 3,
                                 None, None, None)
    assert rc == _lib.HS2_ERR_INVALID
    with pytest.raises(RuntimeError, match="status 1"):
        _lib.check(rc, "altcorr_forward")


def test_ops_check_contiguity_then_device():
    v = torch.zeros(1, 4, 4, 4, 4)
    c = torch.zeros(1, 2, 4, 4)
    with pytest.raises(RuntimeError, match="volume must be contiguous"):
        droid_backends.corr_index_forward(v.transpose(1, 2), c, 3)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        droid_backends.corr_index_forward(v, c, 3)
    p = torch.zeros(8, 7)
    d = torch.ones(8, 4, 4)
    i = torch.zeros(2, dtype=torch.long)
    with pytest.raises(RuntimeError, match="poses must be contiguous"):
        droid_backends.ba(p.t().contiguous().t(), d, torch.zeros(4), torch.zeros(2, 2, 4, 4),
                          torch.zeros(2, 2, 4, 4), torch.zeros(8, 4, 4), i, i, 0, 8, 1, 1e-4, 0.1, False)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        droid_backends.ba(p, d, torch.zeros(4), torch.zeros(2, 2, 4, 4), torch.zeros(2, 2, 4, 4),
                          torch.zeros(8, 4, 4), i, i, 0, 8, 1, 1e-4, 0.1, False)
    with pytest.raises(RuntimeError, match="disps_sens"):
        droid_backends.ba(p, d, torch.zeros(4), torch.ones(8, 4, 4), torch.zeros(2, 2, 4, 4),
                          torch.zeros(2, 2, 4, 4), torch.zeros(8, 4, 4), i, i, 0, 8, 1, 1e-4, 0.1, False)
    with pytest.raises(TypeError):
        droid_backends.ba(p, d, torch.zeros(4), 1, 2, 3)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        droid_backends.frame_distance(p, d, torch.zeros(4), i, i, 0.3)


def test_pgba_checks_inputs_on_cpu():
    p, d, i = torch.zeros(4, 8), torch.ones(4, 3, 3), torch.zeros(2, dtype=torch.long)
    args = (torch.zeros(4), torch.zeros(2, 2, 3, 3), torch.zeros(2, 2, 3, 3), torch.ones(4, 3, 3),
            torch.zeros(4, 1, 1, 7, 7), torch.zeros(2, 1, 1, 7), i, i, i[:1], i[:1], 1, 4, 1e-4, 0.1)
    with pytest.raises(RuntimeError, match="poses must be contiguous"):
        droid_backends.pgba(torch.zeros(8, 4).t(), d, *args)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        droid_backends.pgba(p, d, *args)
    assert backends.pgba is droid_backends.pgba


def test_geometry_ops_check_inputs_on_cpu():
    p, d = torch.zeros(4, 7), torch.ones(4, 3, 3)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        droid_backends.iproj(p, d, torch.zeros(4))
    with pytest.raises(RuntimeError, match="contiguous"):
        droid_backends.covis_distance(p, d.transpose(1, 2), torch.zeros(4), torch.ones(1, dtype=torch.long))


def test_corr_volume_host_validation():
    lib = _lib.load()
    n = ctypes.c_size_t(0)
    ok = lib.hs2_corr_volume_workspace_size(25, 25, 128, 43, 77, _lib.HS2_F16, _lib.HS2_CV_NATIVE, ctypes.byref(n))
    assert ok == _lib.HS2_OK and n.value >= 50 * 3311 * 128 * 2
    fp8 = ctypes.c_size_t(0)
    assert lib.hs2_corr_volume_workspace_size(25, 25, 128, 43, 77, _lib.HS2_BF16, _lib.HS2_CV_E4M3,
                                              ctypes.byref(fp8)) == _lib.HS2_OK
    assert fp8.value < n.value                       # one byte per operand value plus the scales
    assert lib.hs2_corr_volume_workspace_size(2, 2, 64, 43, 77, _lib.HS2_F16, 0, ctypes.byref(n)) == \
        _lib.HS2_ERR_INVALID
    assert b"128" in lib.hs2_last_error()
    assert lib.hs2_corr_volume_workspace_size(2, 2, 128, 8, 100, _lib.HS2_F16, 0, ctypes.byref(n)) == \
        _lib.HS2_ERR_INVALID
    assert lib.hs2_corr_volume_workspace_size(2, 2, 128, 8, 64, _lib.HS2_F32, 0, ctypes.byref(n)) == \
        _lib.HS2_ERR_DTYPE
    assert lib.hs2_corr_volume_workspace_size(2, 2, 128, 8, 64, _lib.HS2_F16, 7, ctypes.byref(n)) == \
        _lib.HS2_ERR_INVALID


def test_ba_adjoint_and_batch_host_validation():
    lib = _lib.load()
    n = ctypes.c_size_t(0)
    assert lib.hs2_ba_adjoint_workspace_size(7, 7, 48, 64, 42, 2, 7, ctypes.byref(n)) == _lib.HS2_OK
    base = ctypes.c_size_t(0)
    lib.hs2_ba_workspace_size(7, 7, 48, 64, 42, 2, 7, 0, ctypes.byref(base))
    assert n.value > base.value                      # the adjoint's per-pixel scratch on top
    assert lib.hs2_ba_adjoint_workspace_size(7, 7, 48, 64, 42, 2, 8, ctypes.byref(n)) == _lib.HS2_ERR_INVALID
    W = _lib.BaWindow
    good = W(1, 10, 1, 10, 30, 40, 1, 1, 1, 1, 10, 1, 1, 40, 1, 10, 1, 1, 10, 1)
    bad_t1 = W(1, 10, 1, 10, 30, 40, 1, 1, 1, 1, 10, 1, 1, 40, 1, 11, 1, 1, 10, 1)
    too_many = W(1, 300, 1, 300, 30, 40, 1, 1, 1, 1, 300, 1, 1, 40, 0, 300, 1, 1, 300, 1)
    null_dx = W(1, 10, 1, 10, 30, 40, 1, 1, 1, 1, 10, 1, 1, 40, 1, 10, 0, 1, 10, 1)
    arr = (W * 2)(good, good)
    assert lib.hs2_ba_batch_workspace_size(arr, 2, ctypes.byref(n)) == _lib.HS2_OK
    one = ctypes.c_size_t(0)
    assert lib.hs2_ba_batch_workspace_size((W * 1)(good), 1, ctypes.byref(one)) == _lib.HS2_OK
    assert one.value < n.value
    for bad, msg in ((bad_t1, b"t1"), (too_many, b"at most 256"), (null_dx, b"null")):
        assert lib.hs2_ba_batch_workspace_size((W * 2)(good, bad), 2, ctypes.byref(n)) == _lib.HS2_ERR_INVALID
        err = lib.hs2_last_error()
        assert b"window 1" in err and msg in err, err
    assert lib.hs2_ba_batch_workspace_size(arr, 0, ctypes.byref(n)) == _lib.HS2_ERR_INVALID


def test_corr_reproject_lookup_host_validation():
    lib = _lib.load()
    ptrs = (ctypes.c_void_p * 4)(1, 1, 1, 1)
    args = [1, 10, 1, 10, 1, ptrs, 4, _lib.HS2_F16, 10, 128, 43, 77, 1, 1, 20, 4, 1, None, 1, None]
    bad_levels = list(args)
    bad_levels[6] = 5
    assert lib.hs2_corr_reproject_lookup(*bad_levels) == _lib.HS2_ERR_INVALID
    tiny = list(args)
    tiny[10], tiny[11] = 4, 4                        # 4 >> 3 == 0: no level-3 grid
    assert lib.hs2_corr_reproject_lookup(*tiny) == _lib.HS2_ERR_INVALID
    missing = list(args)
    missing[5] = (ctypes.c_void_p * 4)(1, 1, 0, 1)
    assert lib.hs2_corr_reproject_lookup(*missing) == _lib.HS2_ERR_INVALID
    assert b"level 2" in lib.hs2_last_error()
    empty = list(args)
    empty[14] = 0
    assert lib.hs2_corr_reproject_lookup(*empty) == _lib.HS2_OK


def test_gram_precision_setter_validation():
    lib = _lib.load()
    assert lib.hs2_ba_set_gram_precision(2) == _lib.HS2_ERR_INVALID
    assert b"3xTF32" in lib.hs2_last_error()
    assert lib.hs2_ba_set_gram_precision(1) == _lib.HS2_OK


def test_packed_altcorr_host_validation():
    """The channel-last correlation entry points refuse bad arguments before any launch."""
    lib = _lib.load()
    n = ctypes.c_size_t(0)
    assert lib.hs2_altcorr_pack_workspace_size(_lib.HS2_F32, 1, 4, 128, 8, 9, ctypes.byref(n)) == _lib.HS2_ERR_DTYPE
    assert lib.hs2_altcorr_pack_workspace_size(_lib.HS2_F16, 1, 4, 300, 8, 9, ctypes.byref(n)) == _lib.HS2_ERR_INVALID
    assert lib.hs2_altcorr_pack_workspace_size(_lib.HS2_F16, 1, 4, 128, 8, 9, ctypes.byref(n)) == _lib.HS2_OK
    assert n.value >= 4 * 8 * 9 * 128 * 2 + 4                   # packed rows + one flag byte per frame
    assert lib.hs2_altcorr_pack(None, _lib.HS2_F16, 1, 4, 128, 8, 9, None, 0, None, 0, None) == \
        _lib.HS2_ERR_WORKSPACE
    assert lib.hs2_altcorr_pack(None, _lib.HS2_F16, 1, 4, 128, 8, 9, None, 3, 1, n.value, None) == \
        _lib.HS2_ERR_INVALID                                     # a frame count without a frame list
    assert lib.hs2_altcorr_pack(None, _lib.HS2_BF16, 0, 4, 128, 8, 9, None, 0, 1, n.value, None) == _lib.HS2_OK
    fwd = [1, 1, _lib.HS2_F16, 1, 4, 4, 128, 8, 9, 4, 5, 1, 1, 1, 3, 3, 1, 1, None]
    f32 = list(fwd)
    f32[2] = _lib.HS2_F32
    assert lib.hs2_altcorr_forward_packed(*f32) == _lib.HS2_ERR_DTYPE
    neg = list(fwd)
    neg[6] = 0
    assert lib.hs2_altcorr_forward_packed(*neg) == _lib.HS2_ERR_INVALID
    empty = list(fwd)
    empty[14] = 0
    assert lib.hs2_altcorr_forward_packed(*empty) == _lib.HS2_OK


def test_fused_packed_lookup_host_validation():
    lib = _lib.load()
    ptrs = (ctypes.c_void_p * 4)(1, 1, 1, 1)
    args = [1, 10, 1, 10, 1, ptrs, 4, _lib.HS2_F16, 10, 128, 43, 77, 1, 1, 20, 3, 1, None, 1, None]
    for idx, val, rc in ((9, 64, _lib.HS2_ERR_INVALID),       # 128 channels only
                         (15, 9, _lib.HS2_ERR_INVALID),       # radius <= 8
                         (7, _lib.HS2_F32, _lib.HS2_ERR_DTYPE),
                         (6, 0, _lib.HS2_ERR_INVALID)):
        bad = list(args)
        bad[idx] = val
        assert lib.hs2_corr_reproject_lookup_packed(*bad) == rc, (idx, val)
    missing = list(args)
    missing[5] = (ctypes.c_void_p * 4)(1, 0, 1, 1)
    assert lib.hs2_corr_reproject_lookup_packed(*missing) == _lib.HS2_ERR_INVALID
    assert b"level 1" in lib.hs2_last_error()
    empty = list(args)
    empty[14] = 0
    assert lib.hs2_corr_reproject_lookup_packed(*empty) == _lib.HS2_OK


def test_jdsa_host_validation():
    """hs2_jdsa refuses sizes outside its limits and missing buffers before any launch."""
    lib = _lib.load()
    args = [1, 6, 1, 6, 12, 16, 1, 1, 1, 1, 1, 6, 1, 6, 2, 2, 1, 1, 1, 1, 1, 22, 1, 6, 0.01, 1, 1, 1, 1, None, 1, None]
    for idx, val, what in ((14, 1, b"hs"),                 # a 2x2 cell needs hs, ws >= 2
                           (15, 9, b"hs*ws"),              # 2 x 9 = 18 scale unknowns > 16
                           (4, 5000, b"ht"),               # grid axes staged in shared memory
                           (23, 0, b"source frames"),      # the reference indexes kx[0]
                           (23, 23, b"source frames"),     # more source frames than edges
                           (16, None, b"null"),            # grid_y
                           (27, None, b"null")):           # dso
        bad = list(args)
        bad[idx] = val
        assert lib.hs2_jdsa(*bad) == _lib.HS2_ERR_INVALID, (idx, val)
        assert what in lib.hs2_last_error(), (idx, lib.hs2_last_error())


def test_jdsa_wrapper_checks_inputs_on_cpu():
    from hislam2_b200 import mono
    p = {k: torch.zeros(1) for k in ("target", "weight", "eta", "poses", "disps", "intrinsics", "disps_prior",
                                     "dscales")}
    ii = torch.zeros(1, dtype=torch.int64)
    with pytest.raises(RuntimeError, match="CUDA tensor"):
        mono.JDSA(p["target"], p["weight"], p["eta"], torch.zeros(2, 7), torch.zeros(1, 2, 4, 4),
                  torch.zeros(4), torch.zeros(2, 4, 4), torch.ones(2, 2, 2), ii, ii, 0.01)


def test_pgo_host_validation():
    lib = _lib.load()
    assert lib.hs2_pgo_constraints(1, -1, 1, 1, 1, 1, 4, 1e-3, 1, 1, 1, 1, None) == _lib.HS2_ERR_INVALID
    assert lib.hs2_pgo_constraints(1, 8, 1, 1, 1, 1, -2, 1e-3, 1, 1, 1, 1, None) == _lib.HS2_ERR_INVALID
    assert lib.hs2_pgo_constraints(1, 8, 1, 1, 1, 1, 4, 1e-3, 1, 1, 1, None, None) == _lib.HS2_ERR_INVALID
    assert b"info" in lib.hs2_last_error()
    assert lib.hs2_sim3_retr(1, 8, 1, 2, 9, None) == _lib.HS2_ERR_INVALID      # t1 beyond the poses
    assert lib.hs2_sim3_retr(1, 8, 1, 5, 4, None) == _lib.HS2_ERR_INVALID      # t1 < t0
    assert b"window" in lib.hs2_last_error()
    assert lib.hs2_sim3_retr(None, 8, None, 3, 3, None) == _lib.HS2_OK         # empty window: nothing to do
