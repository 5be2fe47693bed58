"""The pose-graph terms around ``droid_backends.pgba`` on the B200 kernels.

``global_relative_posesim3_constraints`` keeps the signature and results of HI-SLAM2's
``hislam2/pgo_buffer.py:39-63`` (Hsp [4,1,Np,7,7], vsp [2,1,Np,7], chi2, chi2_scaled),
computed in one launch (``hs2_pgo_constraints``) instead of lietorch's 28 batched
exp / mul / log passes and a dozen float32 matmuls.  ``sim3_retr_`` is the Sim3 pose
retraction that ``hislam2/depth_video.py:267`` applies after each pgba step
(``pose_retr``, lietorch's ``retr``), in place on the pose data.  With both, the loop
of ``DepthVideo.cuda_pgba`` runs without lietorch::

    for _ in range(itrs):
        Hsp, vsp, _, _ = global_relative_posesim3_constraints(iip, jjp, poses, rel_poses, infos, pw=1e-3)
        dx, dz = droid_backends.pgba(poses, disps, ...)
        sim3_retr_(poses, dx, t0, t1)
"""

import torch

from . import _lib
from .backends import _contig, _cuda, _dtype, _ptr, _stream


def _data(x):
    return x.data if hasattr(x, "data") and not isinstance(x, torch.Tensor) else x


def global_relative_posesim3_constraints(ii, jj, poses, rel_poses, infos, pw=1e-5, verbose=False):
    """Relative Sim3 pose factors -> ``(Hsp [4,1,Np,7,7], vsp [2,1,Np,7], chi2, chi2_scaled)``.

    poses: Sim3 group element (``.data`` [1, N, 8]) or tensor [N, 8] / [1, N, 8]; rel_poses:
    SE3 element or tensor [Np, 7] / [1, Np, 7]; infos [Np, 7, 7] (or [1, Np, 7, 7]); ii, jj
    [Np] int64.  ``verbose`` is accepted for the reference's signature (it prints nothing
    there either)."""
    P = _data(poses).reshape(-1, 8)
    R = _data(rel_poses).reshape(-1, 7)
    W = infos.reshape(-1, 7, 7)
    dev = P.device
    for name, t in (("poses", P), ("rel_poses", R), ("infos", W), ("ii", ii), ("jj", jj)):
        _cuda(name, t, dev)
        _contig(name, t)
    for name, t in (("poses", P), ("rel_poses", R), ("infos", W)):
        _dtype(name, t, torch.float32)
    _dtype("ii", ii, torch.int64)
    _dtype("jj", jj, torch.int64)
    Np = ii.numel()
    if jj.numel() != Np or R.shape[0] != Np or W.shape[0] != Np:
        raise RuntimeError("global_relative_posesim3_constraints: ii, jj, rel_poses and infos need one entry "
                           "per factor")
    Hsp = torch.empty((4, 1, Np, 7, 7), dtype=torch.float32, device=dev)
    vsp = torch.empty((2, 1, Np, 7), dtype=torch.float32, device=dev)
    chi = torch.empty((Np, 2), dtype=torch.float32, device=dev)
    info = torch.empty(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hs2_pgo_constraints(_ptr(P), P.shape[0], _ptr(ii), _ptr(jj), _ptr(R), _ptr(W), Np,
                                               float(pw), _ptr(Hsp), _ptr(vsp), _ptr(chi), _ptr(info),
                                               _stream(dev)), "pgo_constraints")
    if Np and int(info.item()) & _lib.HS2_DEV_BAD_INDEX:
        raise RuntimeError("global_relative_posesim3_constraints: a factor's ii / jj is outside the poses")
    chi2 = chi.sum(0)
    return Hsp, vsp, chi2[0], chi2[1]


def sim3_retr_(poses, dx, t0, t1):
    """poses[t0 + k] <- exp(dx[k]) poses[t0 + k] in place (``pose_retr(poses, dx[None],
    arange(t0, t1))`` on Sim3 poses).  poses: Sim3 element or tensor [N, 8] / [1, N, 8]
    (float32, contiguous); dx [t1 - t0, 7].  Returns poses."""
    P = _data(poses)
    P2 = P.reshape(-1, 8)
    dev = P2.device
    for name, t in (("poses", P2), ("dx", dx)):
        _cuda(name, t, dev)
        _contig(name, t)
        _dtype(name, t, torch.float32)
    if P2.data_ptr() != P.data_ptr() or not P.is_contiguous():
        raise RuntimeError("sim3_retr_: poses must be a contiguous [N, 8] buffer")
    if dx.numel() != 7 * (t1 - t0):
        raise RuntimeError("sim3_retr_: dx must be [t1 - t0, 7]")
    _lib.check(_lib.load().hs2_sim3_retr(_ptr(P2), P2.shape[0], _ptr(dx), int(t0), int(t1), _stream(dev)),
               "sim3_retr")
    return poses
