"""The ``droid_backends`` operator surface of HI-SLAM2, on the B200 kernels.

Same names, positional signatures, return conventions and contiguity errors as
the reference binding (``src/droid.cpp:116-341``); every op validates dtype,
device and shape as well (the reference leaves those undefined) and launches
on the current PyTorch stream.  All compute runs in ``libhislam2_b200.so``.
"""

import ctypes

import torch

from . import _lib

_DTYPES = {torch.float32: _lib.HS2_F32, torch.float16: _lib.HS2_F16,
           torch.bfloat16: _lib.HS2_BF16, torch.float64: _lib.HS2_F64}


def _contig(name, t):
    # message of the reference's CHECK_CONTIGUOUS (src/droid.cpp:116)
    if not t.is_contiguous():
        raise RuntimeError("%s must be contiguous" % name)


def _cuda(name, t, device=None):
    if not isinstance(t, torch.Tensor):
        raise RuntimeError("%s must be a torch.Tensor" % name)
    if not t.is_cuda:
        raise RuntimeError("%s must be a CUDA tensor" % name)
    if device is not None and t.device != device:
        raise RuntimeError("%s is on %s, expected %s" % (name, t.device, device))


def _dtype(name, t, *dtypes):
    if t.dtype not in dtypes:
        raise RuntimeError("%s must have dtype %s (got %s)" % (name, " or ".join(map(str, dtypes)), t.dtype))


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


def _raise_device_errors(bits, op, indices="ii/jj outside the buffers or >= t1"):
    if bits & _lib.HS2_DEV_BAD_INDEX:
        raise RuntimeError("%s: an edge index is out of range (%s)" % (op, indices))
    if bits & _lib.HS2_DEV_BAD_ETA:
        raise RuntimeError("%s: eta must have M or 1 rows (M = number of distinct depth frames)" % op)
    if bits & _lib.HS2_DEV_TIMEOUT:
        raise RuntimeError("%s: a bounded in-kernel wait timed out; the results are not valid" % op)
    if bits & _lib.HS2_DEV_LIMIT:
        raise RuntimeError("%s: a kernel size limit was exceeded; the results are not valid" % op)


# --------------------------------------------------------------------------- ba
def ba_workspace_bytes(num_poses, num_disps, ht, wd, num_edges, t0, t1, motion_only):
    n = ctypes.c_size_t(0)
    _lib.check(_lib.load().hs2_ba_workspace_size(num_poses, num_disps, ht, wd, num_edges, t0, t1,
                                                 int(bool(motion_only)), ctypes.byref(n)),
               "ba_workspace_size")
    return n.value


def _ba_check(poses, disps, intrinsics, targets, weights, eta, ii, jj):
    for name, t in (("targets", targets), ("weights", weights), ("poses", poses), ("disps", disps),
                    ("intrinsics", intrinsics), ("ii", ii), ("jj", jj)):
        _contig(name, t)
    dev = poses.device
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("targets", targets),
                    ("weights", weights), ("eta", eta), ("ii", ii), ("jj", jj)):
        _cuda(name, t, dev)
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("targets", targets),
                    ("weights", weights), ("eta", eta)):
        _dtype(name, t, torch.float32)
    _dtype("ii", ii, torch.int64)
    _dtype("jj", jj, torch.int64)
    if poses.dim() != 2 or poses.shape[1] != 7:
        raise RuntimeError("poses must be [N, 7] (got %s)" % tuple(poses.shape))
    if disps.dim() != 3:
        raise RuntimeError("disps must be [N, H, W] (got %s)" % tuple(disps.shape))
    if intrinsics.numel() < 4:
        raise RuntimeError("intrinsics must hold fx, fy, cx, cy")
    E = ii.numel()
    ht, wd = disps.shape[1], disps.shape[2]
    if jj.numel() != E:
        raise RuntimeError("ii and jj must have the same length")
    for name, t in (("targets", targets), ("weights", weights)):
        if tuple(t.shape) != (E, 2, ht, wd):
            raise RuntimeError("%s must be [num_edges, 2, H, W] = %s (got %s)" % (name, (E, 2, ht, wd),
                                                                                 tuple(t.shape)))
    if eta.numel() % (ht * wd) != 0:
        raise RuntimeError("eta must hold whole [H, W] maps (got %s)" % tuple(eta.shape))


def ba(poses, disps, intrinsics, *args, disps_sens=None):
    """Dense bundle adjustment, ``droid_backends.ba`` (reference ``src/droid.cpp:141-168``).

    ``ba(poses, disps, intrinsics, targets, weights, eta, ii, jj, t0, t1, iterations,
    lm, ep, motion_only) -> [dx, dz, dzcov]``; the 15-argument form with
    ``disps_sens`` after ``intrinsics`` is accepted with ``disps_sens=None``.
    ``poses`` and ``disps`` are updated in place.  ``dz`` is None when
    ``motion_only``; ``dzcov`` is always None (undefined in the reference).
    """
    if len(args) == 12:
        disps_sens, args = args[0], args[1:]
    if len(args) != 11:
        raise TypeError("ba() takes 14 positional arguments (15 with disps_sens), got %d" % (3 + len(args)))
    targets, weights, eta, ii, jj, t0, t1, iterations, lm, ep, motion_only = args
    if disps_sens is not None:
        raise RuntimeError("ba: disps_sens is not part of HI-SLAM2's bundle adjustment; pass None")
    _ba_check(poses, disps, intrinsics, targets, weights, eta, ii, jj)
    eta = eta.contiguous()
    dev = poses.device
    t0, t1, iterations = int(t0), int(t1), int(iterations)
    motion_only = bool(motion_only)
    K, (Kd, ht, wd), E = poses.shape[0], disps.shape, ii.numel()
    P = t1 - t0
    ws_bytes = ba_workspace_bytes(K, Kd, ht, wd, E, t0, t1, motion_only)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    S = max(1, min(min(K, Kd), P + E))
    dx = torch.zeros(max(P, 0), 6, dtype=torch.float32, device=dev)
    dz = torch.zeros(S, ht * wd, dtype=torch.float32, device=dev)
    info = torch.zeros(4, dtype=torch.int32, device=dev)
    lib = _lib.load()
    _lib.check(lib.hs2_ba(_ptr(poses), K, _ptr(disps), Kd, ht, wd, _ptr(intrinsics), _ptr(targets),
                          _ptr(weights), _ptr(eta), eta.numel() // (ht * wd), _ptr(ii), _ptr(jj), E, t0, t1,
                          iterations, float(lm), float(ep), int(motion_only), _ptr(dx), _ptr(dz), S,
                          _ptr(info), _ptr(ws), ws_bytes, _stream(dev)), "ba")
    h = info.cpu()
    _raise_device_errors(int(h[0]), "ba")
    M = int(h[1])
    return [dx, None if motion_only else dz[:M], None]


def ba_adjoint(poses, disps, intrinsics, targets, weights, eta, ii, jj, t0, t1, lm, ep, dx, grad_dx, grad_dz):
    """Gradients of one ``ba`` iteration (motion_only = False) w.r.t. targets, weights, eta.

    ``poses``/``disps`` are the linearisation point (the state before the step), ``dx``
    the step's pose update, ``grad_dx`` [t1-t0, 6] and ``grad_dz`` [M, H*W] the incoming
    gradients of dx and dz.  Returns ``[grad_targets, grad_weights, grad_eta, lam]``
    (``lam`` [t1-t0, 6]: the adjoint solution of the damped reduced system).  No
    counterpart in the reference's operator set (its BA is differentiated only on
    the pure-PyTorch path, hislam2/geom/chol.py:8-22).
    """
    _ba_check(poses, disps, intrinsics, targets, weights, eta, ii, jj)
    eta = eta.contiguous()
    dev = poses.device
    t0, t1 = int(t0), int(t1)
    K, (Kd, ht, wd), E = poses.shape[0], disps.shape, ii.numel()
    P = t1 - t0
    for name, t in (("dx", dx), ("grad_dx", grad_dx), ("grad_dz", grad_dz)):
        _cuda(name, t, dev)
        _dtype(name, t, torch.float32)
    dx, grad_dx, grad_dz = dx.contiguous(), grad_dx.contiguous(), grad_dz.contiguous()
    if tuple(dx.shape) != (P, 6) or tuple(grad_dx.shape) != (P, 6) or grad_dz.dim() != 2 \
            or grad_dz.shape[1] != ht * wd:
        raise RuntimeError("ba_adjoint: dx, grad_dx must be [t1-t0, 6] and grad_dz [M, H*W]")
    lib = _lib.load()
    n = ctypes.c_size_t(0)
    _lib.check(lib.hs2_ba_adjoint_workspace_size(K, Kd, ht, wd, E, t0, t1, ctypes.byref(n)),
               "ba_adjoint_workspace_size")
    ws = torch.empty(n.value, dtype=torch.uint8, device=dev)
    gt = torch.empty_like(targets)
    gw = torch.empty_like(weights)
    eta_rows = eta.numel() // (ht * wd)
    ge = torch.empty(eta_rows, ht, wd, dtype=torch.float32, device=dev)
    lam = torch.zeros(max(P, 0), 6, dtype=torch.float32, device=dev)
    info = torch.zeros(4, dtype=torch.int32, device=dev)
    _lib.check(lib.hs2_ba_adjoint(_ptr(poses), K, _ptr(disps), Kd, ht, wd, _ptr(intrinsics), _ptr(targets),
                                  _ptr(weights), _ptr(eta), eta_rows, _ptr(ii), _ptr(jj), E, t0, t1, float(lm),
                                  float(ep), _ptr(dx), _ptr(grad_dx), _ptr(grad_dz), grad_dz.shape[0], _ptr(gt),
                                  _ptr(gw), _ptr(ge), _ptr(lam), _ptr(info), _ptr(ws), n.value, _stream(dev)),
               "ba_adjoint")
    h = info.cpu()
    _raise_device_errors(int(h[0]), "ba_adjoint")
    if int(h[1]) != grad_dz.shape[0]:
        raise RuntimeError("ba_adjoint: grad_dz has %d rows, the step has %d depth frames"
                           % (grad_dz.shape[0], int(h[1])))
    return [gt, gw, ge.reshape(eta.shape), lam]


class BABatch:
    """Many independent ``ba`` windows solved together (``hs2_ba_batch_*``).

    ``windows``: a list of dicts with the tensors of a ``ba`` call (``poses``,
    ``disps``, ``intrinsics``, ``targets``, ``weights``, ``eta``, ``ii``, ``jj``) and
    ``t0``, ``t1``; every window may have its own grid, keyframe and edge count.
    ``prepare`` (at construction) builds the keys of every window once;
    :meth:`run` enqueues ``iterations`` LM iterations -- one persistent launch per
    iteration over all windows -- updating each window's poses / disps in place, and
    can be captured in a CUDA graph (:meth:`graph`).  The tensors must stay alive and
    keep their storage while the object is used.  ``gram_split`` / ``ctas_per_sm``
    are the launch-shape knobs that ``hislam2_b200.autotune`` tunes.
    """

    def __init__(self, windows, lm, ep, gram_split=4, ctas_per_sm=0):
        if not windows:
            raise RuntimeError("ba_batch: no windows")
        dev = windows[0]["poses"].device
        self.device, self.lm, self.ep = dev, float(lm), float(ep)
        self.windows = windows
        arr = (_lib.BaWindow * len(windows))()
        self.dx, self.dz, self.info = [], [], []
        for k, w in enumerate(windows):
            _ba_check(w["poses"], w["disps"], w["intrinsics"], w["targets"], w["weights"], w["eta"], w["ii"], w["jj"])
            if w["poses"].device != dev:
                raise RuntimeError("ba_batch: every window must be on %s" % dev)
            K, (Kd, ht, wd), E = w["poses"].shape[0], w["disps"].shape, w["ii"].numel()
            t0, t1 = int(w["t0"]), int(w["t1"])
            P = t1 - t0
            S = max(1, min(min(K, Kd), P + E))
            dx = torch.zeros(max(P, 0), 6, dtype=torch.float32, device=dev)
            dz = torch.zeros(S, ht * wd, dtype=torch.float32, device=dev)
            info = torch.zeros(4, dtype=torch.int32, device=dev)
            self.dx.append(dx)
            self.dz.append(dz)
            self.info.append(info)
            eta = w["eta"]
            arr[k] = _lib.BaWindow(_ptr(w["poses"]), K, _ptr(w["disps"]), Kd, ht, wd, _ptr(w["intrinsics"]),
                                   _ptr(w["targets"]), _ptr(w["weights"]), _ptr(eta), eta.numel() // (ht * wd),
                                   _ptr(w["ii"]), _ptr(w["jj"]), E, t0, t1, _ptr(dx), _ptr(dz), S, _ptr(info))
        self._arr = arr
        lib = _lib.load()
        n = ctypes.c_size_t(0)
        _lib.check(lib.hs2_ba_batch_workspace_size(arr, len(windows), ctypes.byref(n)), "ba_batch_workspace_size")
        self.ws = torch.empty(n.value, dtype=torch.uint8, device=dev)
        grid = ctypes.c_int(0)
        _lib.check(lib.hs2_ba_batch_prepare(arr, len(windows), int(gram_split), int(ctas_per_sm), _ptr(self.ws),
                                            n.value, ctypes.byref(grid), _stream(dev)), "ba_batch_prepare")
        self.grid = grid.value
        self.check()

    def run(self, iterations):
        _lib.check(_lib.load().hs2_ba_batch_run(_ptr(self.ws), len(self.windows), self.grid, int(iterations), self.lm,
                                                self.ep, _stream(self.device)), "ba_batch_run")

    def graph(self, iterations):
        """A CUDA graph of `iterations` LM iterations (replay with ``.replay()``)."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            g.capture_begin()
            _lib.check(_lib.load().hs2_ba_batch_run(_ptr(self.ws), len(self.windows), self.grid, int(iterations),
                                                    self.lm, self.ep, _stream(self.device)), "ba_batch_run")
            g.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(s)
        return g

    def check(self):
        """Raises on device-detected errors of any window; returns each window's M."""
        out = []
        for k, info in enumerate(self.info):
            h = info.cpu()
            _raise_device_errors(int(h[0]), "ba_batch window %d" % k)
            out.append(int(h[1]))
        return out

    def results(self):
        """[dx, dz] of every window after the last iteration (dz trimmed to M rows)."""
        Ms = self.check()
        return [[dx, dz[:M]] for dx, dz, M in zip(self.dx, self.dz, Ms)]


def pgba_workspace_bytes(num_poses, num_disps, ht, wd, num_edges, t0, t1):
    n = ctypes.c_size_t(0)
    _lib.check(_lib.load().hs2_pgba_workspace_size(num_poses, num_disps, ht, wd, num_edges, t0, t1,
                                                   ctypes.byref(n)), "pgba_workspace_size")
    return n.value


def pgba(poses, disps, intrinsics, targets, weights, eta, Hsp, vsp, ii, jj, iip, jjp, t0, t1, lm, ep):
    """Sim3 pose-graph bundle adjustment, ``droid_backends.pgba`` (reference
    ``src/droid.cpp:171-196``): one damped Gauss-Newton step -> ``[dx, dz]``.

    ``poses`` [N, 8] (t, q xyzw, s) are not modified (``dx`` [t1-t0, 7] is for the
    caller's Sim3 retraction, as ``hislam2/depth_video.py:cuda_pgba`` does);
    ``disps`` is updated in place.  ``Hsp`` [4, ..., Np, 7, 7] and ``vsp`` [2, ..., Np, 7]
    are the relative-pose factors at ``iip`` / ``jjp`` (``pgo_buffer.py``'s
    ``global_relative_posesim3_constraints`` layout).
    """
    for name, t in (("poses", poses), ("disps", disps), ("ii", ii), ("jj", jj)):
        _contig(name, t)
    dev = poses.device
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("targets", targets),
                    ("weights", weights), ("eta", eta), ("Hsp", Hsp), ("vsp", vsp), ("ii", ii), ("jj", jj),
                    ("iip", iip), ("jjp", jjp)):
        _cuda(name, t, dev)
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("targets", targets),
                    ("weights", weights), ("eta", eta), ("Hsp", Hsp), ("vsp", vsp)):
        _dtype(name, t, torch.float32)
    for name, t in (("ii", ii), ("jj", jj), ("iip", iip), ("jjp", jjp)):
        _dtype(name, t, torch.int64)
    if poses.dim() != 2 or poses.shape[1] != 8:
        raise RuntimeError("poses must be [N, 8] Sim3 (got %s)" % tuple(poses.shape))
    if disps.dim() != 3:
        raise RuntimeError("disps must be [N, H, W] (got %s)" % tuple(disps.shape))
    if intrinsics.numel() < 4:
        raise RuntimeError("intrinsics must hold fx, fy, cx, cy")
    E, Np = ii.numel(), iip.numel()
    ht, wd = disps.shape[1], disps.shape[2]
    if jj.numel() != E or jjp.numel() != Np:
        raise RuntimeError("ii/jj and iip/jjp must have matching lengths")
    for name, t in (("targets", targets), ("weights", weights)):
        if tuple(t.shape) != (E, 2, ht, wd):
            raise RuntimeError("%s must be [num_edges, 2, H, W] = %s (got %s)" % (name, (E, 2, ht, wd),
                                                                                 tuple(t.shape)))
    if Hsp.numel() != 4 * Np * 49 or vsp.numel() != 2 * Np * 7:
        raise RuntimeError("Hsp must hold 4 x %d blocks 7x7 and vsp 2 x %d rows of 7 (got %s, %s)"
                           % (Np, Np, tuple(Hsp.shape), tuple(vsp.shape)))
    if eta.numel() % (ht * wd) != 0:
        raise RuntimeError("eta must hold whole [H, W] maps (got %s)" % tuple(eta.shape))
    targets, weights, eta = targets.contiguous(), weights.contiguous(), eta.contiguous()
    Hsp, vsp, iip, jjp = Hsp.contiguous(), vsp.contiguous(), iip.contiguous(), jjp.contiguous()
    intrinsics = intrinsics.contiguous()
    t0, t1 = int(t0), int(t1)
    K, Kd = poses.shape[0], disps.shape[0]
    P = t1 - t0
    ws_bytes = pgba_workspace_bytes(K, Kd, ht, wd, E, t0, t1)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    S = max(1, min(min(K, Kd), P + E))
    dx = torch.zeros(max(P, 0), 7, dtype=torch.float32, device=dev)
    dz = torch.zeros(S, ht * wd, dtype=torch.float32, device=dev)
    info = torch.zeros(4, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_pgba(
        _ptr(poses), K, _ptr(disps), Kd, ht, wd, _ptr(intrinsics), _ptr(targets), _ptr(weights), _ptr(eta),
        eta.numel() // (ht * wd), _ptr(Hsp), _ptr(vsp), _ptr(iip), _ptr(jjp), Np, _ptr(ii), _ptr(jj), E, t0, t1,
        float(lm), float(ep), _ptr(dx), _ptr(dz), S, _ptr(info), _ptr(ws), ws_bytes, _stream(dev)), "pgba")
    h = info.cpu()
    _raise_device_errors(int(h[0]), "pgba", "ii/jj outside the buffers or >= t1, or iip/jjp >= t1")
    return [dx, dz[:int(h[1])]]


def ba_reduced_system(poses, disps, intrinsics, targets, weights, eta, ii, jj, t0, t1, motion_only=False):
    """The reduced camera system (A - S, b - v) of one linearisation at the given state,
    before damping, as float64 CUDA tensors ``[6P, 6P]`` and ``[6P]`` (diagnostic)."""
    _ba_check(poses, disps, intrinsics, targets, weights, eta, ii, jj)
    eta = eta.contiguous()
    dev = poses.device
    K, (Kd, ht, wd), E = poses.shape[0], disps.shape, ii.numel()
    t0, t1 = int(t0), int(t1)
    n = 6 * (t1 - t0)
    ws_bytes = ba_workspace_bytes(K, Kd, ht, wd, E, t0, t1, motion_only)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    A = torch.zeros(n, n, dtype=torch.float64, device=dev)
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    info = torch.zeros(4, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_ba_reduced_system(
        _ptr(poses), K, _ptr(disps), Kd, ht, wd, _ptr(intrinsics), _ptr(targets), _ptr(weights), _ptr(eta),
        eta.numel() // (ht * wd), _ptr(ii), _ptr(jj), E, t0, t1, int(bool(motion_only)), _ptr(A), _ptr(b),
        _ptr(info), _ptr(ws), ws_bytes, _stream(dev)), "ba_reduced_system")
    _raise_device_errors(int(info[0].item()), "ba_reduced_system")
    return A, b


def ba_keys(poses, disps, ii, jj, t0, t1):
    """Integer keys of ``ba`` (unique depth frames, inverse index, Schur row lists).

    Returns ``(kx, kk_exp, rows_ptr, rows)`` as int64 CPU tensors; see
    ``hs2_ba_keys`` in ``include/hislam2_b200.h``.
    """
    _cuda("ii", ii)
    _cuda("jj", jj, ii.device)
    _dtype("ii", ii, torch.int64)
    _dtype("jj", jj, torch.int64)
    dev = ii.device
    K, Kd, (ht, wd), E = poses.shape[0], disps.shape[0], disps.shape[1:], ii.numel()
    P = t1 - t0
    ws_bytes = ba_workspace_bytes(K, Kd, ht, wd, E, t0, t1, False)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    S = max(1, min(min(K, Kd), P + E))
    kx = torch.zeros(S, dtype=torch.int32, device=dev)
    kk = torch.zeros(max(1, P + E), dtype=torch.int32, device=dev)
    rptr = torch.zeros(S + 1, dtype=torch.int32, device=dev)
    rows = torch.zeros(max(1, P + E), dtype=torch.int32, device=dev)
    info = torch.zeros(4, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_ba_keys(K, Kd, ht, wd, _ptr(ii), _ptr(jj), E, t0, t1, _ptr(kx), _ptr(kk),
                                       _ptr(rptr), _ptr(rows), _ptr(info), _ptr(ws), ws_bytes, _stream(dev)),
               "ba_keys")
    h = info.cpu()
    _raise_device_errors(int(h[0]), "ba_keys")
    M = int(h[1])
    rptr = rptr[: M + 1].cpu().long()
    return kx[:M].cpu().long(), kk[: P + E].cpu().long(), rptr, rows[: int(rptr[-1])].cpu().long()


# -------------------------------------------------------------- frame_distance
def frame_distance(poses, disps, intrinsics, ii, jj, beta):
    """``droid_backends.frame_distance`` (reference ``src/droid.cpp:200-216``) -> dist [E]."""
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("ii", ii), ("jj", jj)):
        _contig(name, t)
    dev = poses.device
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("ii", ii), ("jj", jj)):
        _cuda(name, t, dev)
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)):
        _dtype(name, t, torch.float32)
    _dtype("ii", ii, torch.int64)
    _dtype("jj", jj, torch.int64)
    if poses.dim() != 2 or poses.shape[1] != 7 or disps.dim() != 3:
        raise RuntimeError("frame_distance: poses must be [N,7] and disps [N,H,W]")
    if ii.numel() != jj.numel():
        raise RuntimeError("frame_distance: ii and jj must have the same length")
    E = ii.numel()
    dist = torch.zeros(E, dtype=torch.float32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_frame_distance(_ptr(poses), poses.shape[0], _ptr(disps), disps.shape[0],
                                              disps.shape[1], disps.shape[2], _ptr(intrinsics), _ptr(ii),
                                              _ptr(jj), E, float(beta), _ptr(dist), _ptr(info), _stream(dev)),
               "frame_distance")
    if E:
        _raise_device_errors(int(info.item()), "frame_distance")
    return dist


# ------------------------------------------------------ iproj / covis / depth_filter
def _geo_inputs(op, poses, disps, intrinsics, extra=()):
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)) + tuple(extra):
        _contig(name, t)
    dev = poses.device
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)) + tuple(extra):
        _cuda(name, t, dev)
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)):
        _dtype(name, t, torch.float32)
    if poses.dim() != 2 or poses.shape[1] != 7 or disps.dim() != 3:
        raise RuntimeError("%s: poses must be [N,7] and disps [N,H,W]" % op)
    return dev


def iproj(poses, disps, intrinsics):
    """``droid_backends.iproj`` (reference ``src/droid.cpp:233-242``) -> points [N,H,W,3]: every
    pixel of every disparity frame b back-projected and moved by poses[b]."""
    dev = _geo_inputs("iproj", poses, disps, intrinsics)
    N, H, W = disps.shape
    points = torch.zeros((N, H, W, 3), dtype=torch.float32, device=dev)
    _lib.check(_lib.load().hs2_iproj(_ptr(poses), poses.shape[0], _ptr(disps), N, H, W, _ptr(intrinsics),
                                     _ptr(points), _stream(dev)), "iproj")
    return points


def covis_distance(poses, disps, intrinsics, ii):
    """``droid_backends.covis_distance`` (reference ``src/droid.cpp:218-231``) -> dist [N]: for
    i = ii[n], the fraction of frame i's pixels outside the image under both neighbours i-1, i+1."""
    dev = _geo_inputs("covis_distance", poses, disps, intrinsics, (("ii", ii),))
    _dtype("ii", ii, torch.int64)
    n = ii.numel()
    dist = torch.zeros(n, dtype=torch.float32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_covis_distance(_ptr(poses), poses.shape[0], _ptr(disps), disps.shape[0],
                                              disps.shape[1], disps.shape[2], _ptr(intrinsics), _ptr(ii), n,
                                              _ptr(dist), _ptr(info), _stream(dev)), "covis_distance")
    if n and int(info.item()) & _lib.HS2_DEV_BAD_INDEX:
        raise RuntimeError("covis_distance: every ii must have both neighbours ii-1 and ii+1 in the buffers")
    return dist


def depth_filter(poses, disps, intrinsics, ix, thresh):
    """``droid_backends.depth_filter`` (reference ``src/droid.cpp:308-322``) -> counter [N,H,W]:
    per pixel of frame ix[b], how many of the neighbours ix-1, ix-2, ix-3, ix+3, ix+4, ix+5
    agree with its depth to within thresh[b] (reprojected inverse depth)."""
    dev = _geo_inputs("depth_filter", poses, disps, intrinsics, (("ix", ix), ("thresh", thresh)))
    _dtype("ix", ix, torch.int64)
    _dtype("thresh", thresh, torch.float32)
    n = ix.numel()
    if thresh.numel() < n:
        raise RuntimeError("depth_filter: thresh needs one value per ix entry")
    N, H, W = disps.shape
    counter = torch.empty((n, H, W), dtype=torch.float32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_depth_filter(_ptr(poses), poses.shape[0], _ptr(disps), N, H, W, _ptr(intrinsics),
                                            _ptr(ix), _ptr(thresh), n, _ptr(counter), _ptr(info), _stream(dev)),
               "depth_filter")
    if n and int(info.item()) & _lib.HS2_DEV_BAD_INDEX:
        raise RuntimeError("depth_filter: ix outside the disparity buffer")
    return counter


def proj_trans(poses, disps, intrinsics, targets, weights, ii, jj):
    """``droid_backends.proj_trans`` (reference ``src/droid.cpp:121-139``) -> [C, w], each
    [M, H*W] for the M = len(unique(ii)) source frames in ascending order: the depth-only
    Schur terms of the mono-prior alignment (``hislam2/geom/ba.py:178``)."""
    dev = _geo_inputs("proj_trans", poses, disps, intrinsics,
                      (("targets", targets), ("weights", weights), ("ii", ii), ("jj", jj)))
    for name, t in (("targets", targets), ("weights", weights)):
        _dtype(name, t, torch.float32)
    _dtype("ii", ii, torch.int64)
    _dtype("jj", jj, torch.int64)
    E = ii.numel()
    N, H, W = disps.shape
    if jj.numel() != E or targets.shape != (E, 2, H, W) or weights.shape != (E, 2, H, W):
        raise RuntimeError("proj_trans: targets/weights must be [E,2,H,W] and jj as long as ii")
    if intrinsics.numel() < 4:
        raise RuntimeError("proj_trans: intrinsics needs 4 values")
    kx, slot = torch.unique(ii, sorted=True, return_inverse=True)
    M = kx.numel()
    C = torch.empty((M, H * W), dtype=torch.float32, device=dev)
    w = torch.empty((M, H * W), dtype=torch.float32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    slot = slot.contiguous()
    _lib.check(_lib.load().hs2_proj_trans(_ptr(poses), poses.shape[0], _ptr(disps), N, H, W, _ptr(intrinsics),
                                          _ptr(targets), _ptr(weights), _ptr(ii), _ptr(jj), _ptr(slot), E, M,
                                          _ptr(C), _ptr(w), _ptr(info), _stream(dev)), "proj_trans")
    if E and int(info.item()) & _lib.HS2_DEV_BAD_INDEX:
        raise RuntimeError("proj_trans: an edge index is outside the pose/disparity buffers")
    return [C, w]


def bi_inter(scales, grids):
    """``droid_backends.bi_inter`` (reference ``src/droid.cpp:244-251``) -> [outputs [N,H,W],
    jacobians [N,H,W,hs,ws]]: bilinear interpolation of each frame's scale grid at grids[b,i,j]
    = (x, y) and its dense Jacobian (``hislam2/geom/ba.py:161-167``)."""
    for name, t in (("scales", scales), ("grids", grids)):
        _contig(name, t)
        _cuda(name, t, scales.device)
        _dtype(name, t, torch.float32)
    if scales.dim() != 3 or grids.dim() != 4 or grids.shape[-1] != 2 or grids.shape[0] > scales.shape[0]:
        raise RuntimeError("bi_inter: scales must be [N,hs,ws] and grids [N,H,W,2]")
    dev = scales.device
    N, H, W, _ = grids.shape
    hs, ws = scales.shape[1:]
    out = torch.zeros((N, H, W), dtype=torch.float32, device=dev)
    jac = torch.empty((N, H, W, hs, ws), dtype=torch.float32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_bi_inter(_ptr(scales), N, hs, ws, _ptr(grids), H, W, _ptr(out), _ptr(jac),
                                        _ptr(info), _stream(dev)), "bi_inter")
    if N and int(info.item()) & _lib.HS2_DEV_BAD_INDEX:
        raise RuntimeError("bi_inter: a grid point's interpolation cell leaves the scale grid")
    return [out, jac]


# ------------------------------------------------------------------ corr_index
def _corr_dtype(name, t):
    if t.dtype not in _DTYPES:
        raise RuntimeError("%s: unsupported dtype %s" % (name, t.dtype))
    return _DTYPES[t.dtype]


def corr_index_forward(volume, coords, radius):
    """``droid_backends.corr_index_forward`` (reference ``src/droid.cpp:254-264``) -> [corr]."""
    _contig("volume", volume)
    _contig("coords", coords)
    _cuda("volume", volume)
    _cuda("coords", coords, volume.device)
    _dtype("coords", coords, torch.float32)
    dt = _corr_dtype("volume", volume)
    if volume.dim() != 5 or coords.dim() != 4 or coords.shape[1] != 2 or coords.shape[0] != volume.shape[0] \
            or tuple(coords.shape[2:]) != tuple(volume.shape[1:3]):
        raise RuntimeError("corr_index_forward: volume [N,H1,W1,H2,W2] and coords [N,2,H1,W1] expected, got %s "
                           "and %s" % (tuple(volume.shape), tuple(coords.shape)))
    n, h1, w1, h2, w2 = volume.shape
    r = int(radius)
    corr = torch.empty(n, 2 * r + 1, 2 * r + 1, h1, w1, dtype=volume.dtype, device=volume.device)
    _lib.check(_lib.load().hs2_corr_index_forward(_ptr(volume), dt, n, h1, w1, h2, w2, _ptr(coords), r,
                                                  _ptr(corr), _stream(volume.device)), "corr_index_forward")
    return [corr]


def corr_index_backward(volume, coords, corr_grad, radius):
    """``droid_backends.corr_index_backward`` (reference ``src/droid.cpp:266-275``) -> [volume_grad]."""
    _contig("volume", volume)
    _contig("coords", coords)
    _contig("corr_grad", corr_grad)
    _cuda("volume", volume)
    _cuda("coords", coords, volume.device)
    _cuda("corr_grad", corr_grad, volume.device)
    _dtype("coords", coords, torch.float32)
    dt = _corr_dtype("volume", volume)
    _dtype("corr_grad", corr_grad, volume.dtype)
    n, h1, w1, h2, w2 = volume.shape
    r = int(radius)
    if tuple(corr_grad.shape) != (n, 2 * r + 1, 2 * r + 1, h1, w1):
        raise RuntimeError("corr_index_backward: corr_grad must be %s (got %s)"
                           % ((n, 2 * r + 1, 2 * r + 1, h1, w1), tuple(corr_grad.shape)))
    volume_grad = torch.empty_like(volume)
    _lib.check(_lib.load().hs2_corr_index_backward(_ptr(coords), _ptr(corr_grad), dt, n, h1, w1, h2, w2, r,
                                                   _ptr(volume_grad), _stream(volume.device)),
               "corr_index_backward")
    return [volume_grad]


# ----------------------------------------------------------------- corr_volume
def corr_volume(fmap1, fmap2, ii=None, jj=None, num_levels=4, precision="native"):
    """All-pairs correlation pyramid of HI-SLAM2's ``CorrBlock`` on the tensor cores.

    Replaces the caller-side ``CorrBlock.corr`` + ``avg_pool2d`` pyramid
    (``hislam2/modules/corr.py:29-38,63-71``).  ``fmap1`` [K1,128,H,W] and ``fmap2``
    [K2,128,H,W] (float16 or bfloat16; a leading [B,N] is flattened); pair e
    correlates frame ``ii[e]`` of fmap1 with frame ``jj[e]`` of fmap2 (default: frame
    e with frame e, K1 == K2).  Returns ``num_levels`` tensors [E, H, W, H>>l, W>>l]
    of the fmaps' dtype: level 0 = (f1/4)^T (f2/4), level l = 2x2 average of level l-1
    computed as avg_pool2d does.  ``precision="e4m3"`` contracts FP8 e4m3 features with
    one scale per pixel instead of the 16-bit values.
    """
    if fmap1.dim() == 5:
        fmap1 = fmap1.reshape(-1, *fmap1.shape[2:])
    if fmap2.dim() == 5:
        fmap2 = fmap2.reshape(-1, *fmap2.shape[2:])
    _contig("fmap1", fmap1)
    _contig("fmap2", fmap2)
    _cuda("fmap1", fmap1)
    dev = fmap1.device
    _cuda("fmap2", fmap2, dev)
    _dtype("fmap1", fmap1, torch.float16, torch.bfloat16)
    _dtype("fmap2", fmap2, fmap1.dtype)
    if fmap1.dim() != 4 or fmap2.dim() != 4 or tuple(fmap1.shape[1:]) != tuple(fmap2.shape[1:]):
        raise RuntimeError("corr_volume: fmaps [K,C,H,W] of equal C,H,W expected, got %s and %s"
                           % (tuple(fmap1.shape), tuple(fmap2.shape)))
    K1, C, H, W = fmap1.shape
    K2 = fmap2.shape[0]
    if ii is None or jj is None:
        if K1 != K2:
            raise RuntimeError("corr_volume: without ii/jj both fmaps need the same number of frames")
        ii = jj = torch.arange(K1, device=dev)
    for name, t in (("ii", ii), ("jj", jj)):
        _cuda(name, t, dev)
        _dtype(name, t, torch.int64)
    ii, jj = ii.contiguous(), jj.contiguous()
    if ii.numel() != jj.numel():
        raise RuntimeError("corr_volume: ii and jj differ in length")
    prec = {"native": _lib.HS2_CV_NATIVE, "e4m3": _lib.HS2_CV_E4M3}.get(precision)
    if prec is None:
        raise RuntimeError("corr_volume: precision must be 'native' or 'e4m3'")
    L = int(num_levels)
    E = ii.numel()
    dt = _DTYPES[fmap1.dtype]
    lib = _lib.load()
    nbytes = ctypes.c_size_t(0)
    _lib.check(lib.hs2_corr_volume_workspace_size(K1, K2, C, H, W, dt, prec, ctypes.byref(nbytes)),
               "corr_volume_workspace_size")
    pyr = [torch.empty(E, H, W, H >> l, W >> l, dtype=fmap1.dtype, device=dev) for l in range(L)]
    if E == 0:
        return pyr
    ws = torch.empty(max(1, nbytes.value), dtype=torch.uint8, device=dev)
    ptrs = (ctypes.c_void_p * 4)(*[p.data_ptr() if p.numel() else 0 for p in pyr] + [0] * (4 - L))
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.hs2_corr_volume(_ptr(fmap1), K1, _ptr(fmap2), K2, C, H, W, dt, _ptr(ii), _ptr(jj), E, prec, L,
                                   ptrs, _ptr(info), _ptr(ws), nbytes.value, _stream(dev)), "corr_volume")
    bits = int(info.item())
    if bits:
        _raise_device_errors(bits, "corr_volume", "ii/jj outside the frames of fmap1/fmap2")
    return pyr


def corr_reproject_lookup(fmap_levels, poses, disps, intrinsics, ii, jj, radius, return_coords=True, *,
                          path="auto"):
    """Reprojection + multi-level correlation lookup in one launch.

    Fuses ``DepthVideo.reproject(ii, jj)`` (``hislam2/depth_video.py:170-178``) with the
    ``AltCorrBlock`` lookup (``hislam2/modules/corr.py:90-117``): ``fmap_levels`` is the
    list of pooled features [K, C, H>>l, W>>l] (level 0 the features themselves),
    ``poses`` [K,7], ``disps`` [K,H,W], ``intrinsics`` [4] float32.  Returns ``corr``
    [E, L*(2r+1)^2, H, W] (the fmaps' dtype) and, with ``return_coords``, the level-0
    ``coords1`` [E, H, W, 2] (float32).  float16 / bfloat16 features with 128 channels and
    radius <= 8 take the channel-last tensor-core path (the frames of ii / jj packed per
    level first) unless ``path="direct"``.
    """
    L = len(fmap_levels)
    f0 = fmap_levels[0]
    dev = f0.device
    for l, f in enumerate(fmap_levels):
        _contig("fmap_levels[%d]" % l, f)
        _cuda("fmap_levels[%d]" % l, f, dev)
        _dtype("fmap_levels[%d]" % l, f, f0.dtype)
        if f.dim() != 4 or f.shape[:2] != f0.shape[:2] or tuple(f.shape[2:]) != (f0.shape[2] >> l,
                                                                               f0.shape[3] >> l):
            raise RuntimeError("corr_reproject_lookup: level %d must be [K, C, H>>%d, W>>%d]" % (l, l, l))
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)):
        _contig(name, t)
        _cuda(name, t, dev)
        _dtype(name, t, torch.float32)
    for name, t in (("ii", ii), ("jj", jj)):
        _cuda(name, t, dev)
        _dtype(name, t, torch.int64)
    ii, jj = ii.contiguous(), jj.contiguous()
    K, C, H, W = f0.shape
    if tuple(disps.shape[1:]) != (H, W) or poses.dim() != 2 or poses.shape[1] != 7:
        raise RuntimeError("corr_reproject_lookup: disps [K,H,W] on the features' grid and poses [K,7] expected")
    E, r = ii.numel(), int(radius)
    corr = torch.empty(E, L * (2 * r + 1) ** 2, H, W, dtype=f0.dtype, device=dev)
    coords = torch.empty(E, H, W, 2, dtype=torch.float32, device=dev) if return_coords else None
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    if path not in ("auto", "direct", "packed"):
        raise RuntimeError("corr_reproject_lookup: path is auto, direct or packed")
    packable = f0.dtype in (torch.float16, torch.bfloat16) and C == 128 and r <= 8
    if path == "packed" and not packable:
        raise RuntimeError("corr_reproject_lookup: the packed path takes float16 / bfloat16 features, C = 128, r <= 8")
    if packable and path != "direct":
        both = torch.cat([ii, jj])
        packed = [PackedFeatures(f[None], both if lvl == 0 else jj) for lvl, f in enumerate(fmap_levels)]
        pptrs = (ctypes.c_void_p * 4)(*[pk.buf.data_ptr() for pk in packed] + [0] * (4 - L))
        _lib.check(_lib.load().hs2_corr_reproject_lookup_packed(
            _ptr(poses), poses.shape[0], _ptr(disps), disps.shape[0], _ptr(intrinsics), pptrs, L, _DTYPES[f0.dtype],
            K, C, H, W, _ptr(ii), _ptr(jj), E, r, _ptr(corr), _ptr(coords), _ptr(info), _stream(dev)),
            "corr_reproject_lookup")
        return (corr, coords) if return_coords else corr
    ptrs = (ctypes.c_void_p * 4)(*[f.data_ptr() for f in fmap_levels] + [0] * (4 - L))
    _lib.check(_lib.load().hs2_corr_reproject_lookup(_ptr(poses), poses.shape[0], _ptr(disps), disps.shape[0],
                                                     _ptr(intrinsics), ptrs, L, _DTYPES[f0.dtype], K, C, H, W,
                                                     _ptr(ii), _ptr(jj), E, r, _ptr(corr), _ptr(coords), _ptr(info),
                                                     _stream(dev)), "corr_reproject_lookup")
    return (corr, coords) if return_coords else corr


# --------------------------------------------------------------------- altcorr
def _altcorr_check(fmap1, fmap2, coords, ii, jj):
    _contig("fmap1", fmap1)
    _contig("fmap2", fmap2)
    _contig("coords", coords)
    dev = fmap1.device
    for name, t in (("fmap1", fmap1), ("fmap2", fmap2), ("coords", coords), ("ii", ii), ("jj", jj)):
        _cuda(name, t, dev)
    _dtype("fmap2", fmap2, fmap1.dtype)
    _dtype("coords", coords, torch.float32)
    _dtype("ii", ii, torch.int64)
    _dtype("jj", jj, torch.int64)
    if fmap1.dim() != 5 or fmap2.dim() != 5 or coords.dim() != 5 or coords.shape[2] != 2:
        raise RuntimeError("altcorr: fmaps [B,N,C,H,W] and coords [B,M,2,H,W] expected")
    B, M = coords.shape[0], coords.shape[1]
    if fmap1.shape[0] != B or fmap2.shape[0] != B or fmap1.shape[2] != fmap2.shape[2] \
            or tuple(fmap1.shape[3:]) != tuple(coords.shape[3:]) or ii.numel() != M or jj.numel() != M:
        raise RuntimeError("altcorr: inconsistent shapes fmap1 %s fmap2 %s coords %s ii %s jj %s" % (
            tuple(fmap1.shape), tuple(fmap2.shape), tuple(coords.shape), tuple(ii.shape), tuple(jj.shape)))
    return _corr_dtype("fmap1", fmap1)


PACKED_CHANNELS = (32, 64, 128, 256)


class PackedFeatures:
    """Channel-last copy ([B, N, H*W, C]) of a [B, N, C, H, W] float16 / bfloat16 feature
    tensor for :func:`altcorr_forward_packed`; only the listed frames are written."""

    def __init__(self, fmap, frames=None):
        _contig("fmap", fmap)
        dt = _corr_dtype("fmap", fmap)
        if dt not in (_lib.HS2_F16, _lib.HS2_BF16) or fmap.dim() != 5:
            raise RuntimeError("altcorr_pack: [B,N,C,H,W] float16 or bfloat16 features expected")
        B, N, C, H, W = fmap.shape
        n = ctypes.c_size_t(0)
        lib = _lib.load()
        _lib.check(lib.hs2_altcorr_pack_workspace_size(dt, B, N, C, H, W, ctypes.byref(n)), "altcorr_pack")
        self.buf = torch.empty(n.value, dtype=torch.uint8, device=fmap.device)
        if frames is not None:
            frames = frames.contiguous()
            _cuda("frames", frames, fmap.device)
            _dtype("frames", frames, torch.int64)
        _lib.check(lib.hs2_altcorr_pack(_ptr(fmap), dt, B, N, C, H, W, _ptr(frames) if frames is not None else None,
                                        0 if frames is None else frames.numel(), _ptr(self.buf), n.value,
                                        _stream(fmap.device)), "altcorr_pack")
        self.dtype, self.torch_dtype, self.shape, self.device = dt, fmap.dtype, tuple(fmap.shape), fmap.device


def altcorr_forward_packed(packed1, packed2, coords, ii, jj, radius):
    """:func:`altcorr_forward` on :class:`PackedFeatures` (float16 / bfloat16, C in 32..256)."""
    _contig("coords", coords)
    ii, jj = ii.contiguous(), jj.contiguous()
    dev = packed1.device
    for name, t in (("coords", coords), ("ii", ii), ("jj", jj)):
        _cuda(name, t, dev)
    _dtype("coords", coords, torch.float32)
    B, N1, C, H, W = packed1.shape
    _, N2, C2, H2, W2 = packed2.shape
    if packed2.dtype != packed1.dtype or C2 != C or packed2.shape[0] != B or coords.dim() != 5 \
            or tuple(coords.shape[:1]) != (B,) or tuple(coords.shape[2:]) != (2, H, W):
        raise RuntimeError("altcorr_forward_packed: inconsistent shapes %s %s %s" % (
            packed1.shape, packed2.shape, tuple(coords.shape)))
    M = coords.shape[1]
    if ii.numel() != M or jj.numel() != M:
        raise RuntimeError("altcorr_forward_packed: ii/jj must have %d entries" % M)
    r = int(radius)
    corr = torch.empty(B, M, 2 * r + 1, 2 * r + 1, H, W, dtype=packed1.torch_dtype, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_altcorr_forward_packed(_ptr(packed1.buf), _ptr(packed2.buf), packed1.dtype, B, N1, N2,
                                                      C, H, W, H2, W2, _ptr(coords), _ptr(ii), _ptr(jj), M, r,
                                                      _ptr(corr), _ptr(info), _stream(dev)), "altcorr_forward_packed")
    return [corr]


def altcorr_forward(fmap1, fmap2, coords, ii, jj, radius, *, path="auto"):
    """``droid_backends.altcorr_forward`` (reference ``src/droid.cpp:277-289``) -> [corr].

    corr is [B, M, 2r+1, 2r+1, H, W] with dim 2 along x, returned contiguous
    (the reference returns the same values as a permuted view).  float16 / bfloat16
    features with C in 32..256 take the channel-last path (the frames of ii / jj packed
    first) unless ``path="direct"``.
    """
    dt = _altcorr_check(fmap1, fmap2, coords, ii.contiguous(), jj.contiguous())
    ii, jj = ii.contiguous(), jj.contiguous()
    B, N1, C, H, W = fmap1.shape
    N2, H2, W2 = fmap2.shape[1], fmap2.shape[3], fmap2.shape[4]
    M = coords.shape[1]
    r = int(radius)
    if path not in ("auto", "direct", "packed"):
        raise RuntimeError("altcorr_forward: path is auto, direct or packed")
    packable = dt in (_lib.HS2_F16, _lib.HS2_BF16) and C in PACKED_CHANNELS
    if path == "packed" and not packable:
        raise RuntimeError("altcorr_forward: the packed path takes float16 / bfloat16 features with C in %s"
                           % (PACKED_CHANNELS,))
    if packable and path != "direct":
        return altcorr_forward_packed(PackedFeatures(fmap1, ii), PackedFeatures(fmap2, jj), coords, ii, jj, r)
    corr = torch.empty(B, M, 2 * r + 1, 2 * r + 1, H, W, dtype=fmap1.dtype, device=fmap1.device)
    info = torch.zeros(1, dtype=torch.int32, device=fmap1.device)
    _lib.check(_lib.load().hs2_altcorr_forward(_ptr(fmap1), _ptr(fmap2), dt, B, N1, N2, C, H, W, H2, W2,
                                               _ptr(coords), _ptr(ii), _ptr(jj), M, r, _ptr(corr), _ptr(info),
                                               _stream(fmap1.device)), "altcorr_forward")
    return [corr]


def altcorr_backward(fmap1, fmap2, coords, ii, jj, grad, radius, scale=1.0):
    """``droid_backends.altcorr_backward`` -> [fmap1_grad, fmap2_grad].

    Positional order as HI-SLAM2 calls it (``hislam2/modules/corr.py:86``, which
    the binding's swapped parameter names in ``src/droid.cpp:291-305`` cancel).
    ``scale=1`` reproduces the reference operator, which leaves out the forward's
    1/16; ``scale=1/16`` is the exact adjoint of :func:`altcorr_forward`.
    """
    dt = _altcorr_check(fmap1, fmap2, coords, ii, jj)
    if dt == _lib.HS2_F64:
        raise RuntimeError("altcorr_backward: float64 feature maps are not supported")
    ii, jj = ii.contiguous(), jj.contiguous()
    _cuda("grad", grad, fmap1.device)
    _dtype("grad", grad, torch.float32)
    grad = grad.contiguous()
    B, N1, C, H, W = fmap1.shape
    N2, H2, W2 = fmap2.shape[1], fmap2.shape[3], fmap2.shape[4]
    M = coords.shape[1]
    r = int(radius)
    if tuple(grad.shape) != (B, M, 2 * r + 1, 2 * r + 1, H, W):
        raise RuntimeError("altcorr_backward: grad must be %s" % ((B, M, 2 * r + 1, 2 * r + 1, H, W),))
    lib = _lib.load()
    nbytes = ctypes.c_size_t(0)
    _lib.check(lib.hs2_altcorr_backward_workspace_size(dt, B, N1, N2, C, H, W, H2, W2, ctypes.byref(nbytes)),
               "altcorr_backward_workspace_size")
    ws = torch.empty(max(1, nbytes.value), dtype=torch.uint8, device=fmap1.device)
    g1 = torch.empty_like(fmap1)
    g2 = torch.empty_like(fmap2)
    info = torch.zeros(1, dtype=torch.int32, device=fmap1.device)
    _lib.check(lib.hs2_altcorr_backward(_ptr(fmap1), _ptr(fmap2), dt, B, N1, N2, C, H, W, H2, W2, _ptr(coords),
                                        _ptr(ii), _ptr(jj), M, _ptr(grad), r, float(scale), _ptr(g1), _ptr(g2),
                                        _ptr(info), _ptr(ws), nbytes.value, _stream(fmap1.device)),
               "altcorr_backward")
    return [g1, g2]
