"""ctypes binding of ``libhislam2_b200.so`` (declared in ``include/hislam2_b200.h``).

The library is the only implementation of the operators: there is no CPU or
PyTorch fallback.  Loading fails loudly when the shared object is missing.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhislam2_b200.so")

HS2_OK, HS2_ERR_INVALID, HS2_ERR_CUDA, HS2_ERR_WORKSPACE, HS2_ERR_DTYPE = range(5)
HS2_F32, HS2_F16, HS2_BF16, HS2_F64 = range(4)
HS2_CV_NATIVE, HS2_CV_E4M3 = range(2)
HS2_DEV_BAD_INDEX = 1
HS2_DEV_BAD_ETA = 2
HS2_DEV_TIMEOUT = 4
HS2_DEV_LIMIT = 8
HS2_DEV_NOT_PD = 16

_p = ctypes.c_void_p
_i32 = ctypes.c_int
_i64 = ctypes.c_int64
_f32 = ctypes.c_float
_sz = ctypes.c_size_t

# name -> argtypes, exactly the order of include/hislam2_b200.h
SIGNATURES = {
    "hs2_last_error": [],
    "hs2_version": [],
    "hs2_frame_distance": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _i64, _f32, _p, _p, _p],
    "hs2_corr_index_forward": [_p, _i32, _i64, _i32, _i32, _i32, _i32, _p, _i32, _p, _p],
    "hs2_corr_index_backward": [_p, _p, _i32, _i64, _i32, _i32, _i32, _i32, _i32, _p, _p],
    "hs2_corr_volume_workspace_size": [_i64, _i64, _i32, _i32, _i32, _i32, _i32, ctypes.POINTER(_sz)],
    "hs2_corr_volume": [_p, _i64, _p, _i64, _i32, _i32, _i32, _i32, _p, _p, _i64, _i32, _i32, _p, _p, _p, _sz,
                        _p],
    "hs2_altcorr_forward": [_p, _p, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _p, _p, _p,
                            _i32, _i32, _p, _p, _p],
    "hs2_altcorr_pack_workspace_size": [_i32, _i32, _i32, _i32, _i32, _i32, ctypes.POINTER(_sz)],
    "hs2_altcorr_pack": [_p, _i32, _i32, _i32, _i32, _i32, _i32, _p, _i32, _p, _sz, _p],
    "hs2_altcorr_forward_packed": [_p, _p, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _p, _p, _p,
                                   _i32, _i32, _p, _p, _p],
    "hs2_altcorr_backward_workspace_size": [_i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32,
                                            ctypes.POINTER(_sz)],
    "hs2_altcorr_backward": [_p, _p, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _p, _p, _p,
                             _i32, _p, _i32, _f32, _p, _p, _p, _p, _sz, _p],
    "hs2_ba_workspace_size": [_i64, _i64, _i32, _i32, _i64, _i32, _i32, _i32, ctypes.POINTER(_sz)],
    "hs2_ba": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _i64, _p, _p, _i64, _i32, _i32, _i32,
               _f32, _f32, _i32, _p, _p, _i64, _p, _p, _sz, _p],
    "hs2_ba_noalloc": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _i64, _p, _p, _i64, _i32, _i32, _i32,
                       _f32, _f32, _i32, _p, _p, _i64, _p, _p],
    "hs2_ba_reduced_system": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _i64, _p, _p, _i64, _i32, _i32,
                              _i32, _p, _p, _p, _p, _sz, _p],
    "hs2_ba_set_schur_path": [_i32],
    "hs2_ba_set_gram_precision": [_i32],
    "hs2_ba_adjoint_workspace_size": [_i64, _i64, _i32, _i32, _i64, _i32, _i32, ctypes.POINTER(_sz)],
    "hs2_ba_adjoint": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _i64, _p, _p, _i64, _i32, _i32, _f32, _f32,
                       _p, _p, _p, _i64, _p, _p, _p, _p, _p, _p, _sz, _p],
    "hs2_pgba_workspace_size": [_i64, _i64, _i32, _i32, _i64, _i32, _i32, ctypes.POINTER(_sz)],
    "hs2_pgba": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _i64, _p, _p, _p, _p, _i64, _p, _p, _i64, _i32,
                 _i32, _f32, _f32, _p, _p, _i64, _p, _p, _sz, _p],
    "hs2_iproj": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p],
    "hs2_proj_trans": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _p, _p, _i64, _i64, _p, _p, _p, _p],
    "hs2_bi_inter": [_p, _i64, _i32, _i32, _p, _i32, _i32, _p, _p, _p, _p],
    "hs2_pgo_constraints": [_p, _i64, _p, _p, _p, _p, _i64, ctypes.c_double, _p, _p, _p, _p, _p],
    "hs2_sim3_retr": [_p, _i64, _p, _i64, _i64, _p],
    "hs2_jdsa": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _p, _p,
                 _i64, _p, _i64, _f32, _p, _p, _p, _p, _p, _p, _p],
    "hs2_covis_distance": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _i64, _p, _p, _p],
    "hs2_depth_filter": [_p, _i64, _p, _i64, _i32, _i32, _p, _p, _p, _i64, _p, _p, _p],
    "hs2_profile_enable": [_i32],
    "hs2_launch_count": [],
    "hs2_profile_report": [ctypes.c_char_p, _sz, _i32],
    "hs2_ba_keys": [_i64, _i64, _i32, _i32, _p, _p, _i64, _i32, _i32, _p, _p, _p, _p, _p, _p, _sz, _p],
}

class BaWindow(ctypes.Structure):
    """``hs2_ba_window`` of include/hislam2_b200.h (one window of hs2_ba_batch)."""
    _fields_ = [("poses", _p), ("num_poses", _i64), ("disps", _p), ("num_disps", _i64), ("ht", _i32),
                ("wd", _i32), ("intrinsics", _p), ("targets", _p), ("weights", _p), ("eta", _p),
                ("eta_rows", _i64), ("ii", _p), ("jj", _p), ("num_edges", _i64), ("t0", _i32), ("t1", _i32),
                ("dx", _p), ("dz", _p), ("dz_rows", _i64), ("info", _p)]


SIGNATURES.update({
    "hs2_corr_reproject_lookup": [_p, _i64, _p, _i64, _p, _p, _i32, _i32, _i64, _i32, _i32, _i32, _p, _p, _i64,
                                  _i32, _p, _p, _p, _p],
    "hs2_corr_reproject_lookup_packed": [_p, _i64, _p, _i64, _p, _p, _i32, _i32, _i64, _i32, _i32, _i32, _p, _p,
                                         _i64, _i32, _p, _p, _p, _p],
    "hs2_ba_batch_workspace_size": [ctypes.POINTER(BaWindow), _i32, ctypes.POINTER(_sz)],
    "hs2_ba_batch_prepare": [ctypes.POINTER(BaWindow), _i32, _i32, _i32, _p, _sz, ctypes.POINTER(_i32), _p],
    "hs2_ba_batch_run": [_p, _i32, _i32, _i32, _f32, _f32, _p],
    "hs2_ba_batch_set_wait_test": [ctypes.c_uint, _i32],
})

_lib = None


def load():
    """Loads the library once; raises ``RuntimeError`` if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "hislam2_b200: %s is missing; build it with `python hi-slam2_b200/hislam2_b200/build.py` "
            "(there is no CPU fallback)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = {"hs2_last_error": ctypes.c_char_p, "hs2_profile_enable": None,
                      "hs2_launch_count": ctypes.c_longlong}.get(name, ctypes.c_int)
    _lib = lib
    return lib


def check(rc, what):
    """Maps a non-zero status to ``RuntimeError`` with the library's message."""
    if rc != HS2_OK:
        msg = load().hs2_last_error().decode(errors="replace")
        raise RuntimeError("%s failed (status %d): %s" % (what, rc, msg))


def profile_enable(on=True):
    load().hs2_profile_enable(int(bool(on)))


def profile_report(reset=True):
    """{kernel name: (launches, total_ms)} of the launches recorded since the last reset."""
    buf = ctypes.create_string_buffer(1 << 16)
    load().hs2_profile_report(buf, len(buf), int(bool(reset)))
    out = {}
    for line in buf.value.decode().splitlines():
        name, n, ms = line.split()
        out[name] = (int(n), float(ms))
    return out


def launch_count():
    """Kernels launched by the library so far in this process."""
    return int(load().hs2_launch_count())


def set_gram_precision(precision):
    """1: 3xTF32 tensor-core Gram (FP32-accurate, default); 0: one TF32 product (mixed form)."""
    check(load().hs2_ba_set_gram_precision(int(precision)), "ba_set_gram_precision")


def set_schur_path(path):
    """0: tensor-core Gram over stored E rows (default), 1: SIMT FP32 Gram,
    2: fused per-frame linearisation + tensor-core Gram."""
    check(load().hs2_ba_set_schur_path(int(path)), "ba_set_schur_path")
