"""HI-SLAM2's mono-prior depth / scale alignment step, ``geom.ba.JDSA``, on the B200 kernels.

``JDSA`` keeps the reference's signature and results (``hislam2/geom/ba.py:170-219``):
one step that aligns the disparities of the source frames kx = unique(ii) to the
monocular prior ``disps_prior`` through per-frame bilinear scale grids ``dscales``
[N, hs, ws], after ``droid_backends.ba`` (its caller is ``hislam2/depth_video.py:234-240``).
The reference forms a dense Jacobian [M,H,W,hs,ws], E [M*hs*ws, M*H*W] and a dense
Cholesky; ``hs2_jdsa`` solves the same block-diagonal system frame by frame in one pass
(``csrc/jdsa.cu``).  Returns ``(disps [1,P,H,W], dscales, dzcov [M, H*W])`` with
``dscales`` updated in place, as the reference does.
"""

import torch

from . import _lib
from .backends import _contig, _cuda, _dtype, _ptr, _stream

_GRIDS = {}


def grid_axes(ht, wd, hs, ws, device):
    """The sampling grid of ``get_prior_depth_aligned`` (``hislam2/geom/ba.py:161-163``) as its
    two axes, gy [ht] = linspace(0, hs-1-1e-6, ht) and gx [wd] = linspace(0, ws-1-1e-6, wd):
    computed by ``torch.linspace`` on the host in float32 as the reference does, copied to
    the device once per shape."""
    key = (ht, wd, hs, ws, str(device))
    if key not in _GRIDS:
        gy = torch.linspace(0, hs - 1 - 1e-6, ht)
        gx = torch.linspace(0, ws - 1 - 1e-6, wd)
        _GRIDS[key] = (gy.to(device), gx.to(device))
    return _GRIDS[key]


def JDSA(target, weight, eta, poses, disps, intrinsics, disps_prior, dscales, ii, jj, alpha, with_dzcov=True):
    """One alignment step (reference ``JDSA``).

    target, weight [E, 2, H, W]; eta with M*H*W values (M = len(unique(ii))); poses an SE3
    group element whose ``.data`` is [1, P, 7] or a tensor [P, 7] / [1, P, 7]; disps
    [1, P, H, W] or [P, H, W]; intrinsics [..., 4] (the first camera is used, as the
    reference's ``proj_trans`` does); disps_prior [>= max(ii)+1, H, W]; dscales [>= P, hs, ws]
    (updated in place); ii, jj [E] int64; alpha the prior weight (``mono_depth_alpha``).
    ``with_dzcov=False`` skips the depth covariance (the reference always computes it and
    its caller discards it) and returns None in its place.

    Raises ``torch.linalg.LinAlgError`` when the reduced scale system is not positive
    definite (the reference raises there too) and ``RuntimeError`` for indices outside the
    buffers; in both cases ``dscales`` is left unchanged.
    """
    pdata = poses.data if hasattr(poses, "data") and not isinstance(poses, torch.Tensor) else poses
    pdata = pdata.reshape(-1, 7)
    batched = disps.dim() == 4
    d3 = disps[0] if batched else disps
    dev = d3.device
    intr = intrinsics.reshape(-1, 4)[0].contiguous()
    for name, t in (("target", target), ("weight", weight), ("eta", eta), ("poses", pdata), ("disps", d3),
                    ("intrinsics", intr), ("disps_prior", disps_prior), ("dscales", dscales), ("ii", ii),
                    ("jj", jj)):
        _cuda(name, t, dev)
        _contig(name, t)
    for name, t in (("target", target), ("weight", weight), ("eta", eta), ("poses", pdata), ("disps", d3),
                    ("intrinsics", intr), ("disps_prior", disps_prior), ("dscales", dscales)):
        _dtype(name, t, torch.float32)
    _dtype("ii", ii, torch.int64)
    _dtype("jj", jj, torch.int64)
    if d3.dim() != 3 or disps_prior.dim() != 3 or dscales.dim() != 3:
        raise RuntimeError("JDSA: disps must be [1,P,H,W], disps_prior [N,H,W] and dscales [N,hs,ws]")
    P, H, W = d3.shape
    E = ii.numel()
    if E == 0:
        raise RuntimeError("JDSA: no edges (the reference indexes kx[0] of an empty unique(ii))")
    if jj.numel() != E or target.shape != (E, 2, H, W) or weight.shape != (E, 2, H, W):
        raise RuntimeError("JDSA: target/weight must be [E,2,H,W] and jj as long as ii")
    if disps_prior.shape[1:] != (H, W):
        raise RuntimeError("JDSA: disps_prior must have the disparities' H, W")
    kx, slot = torch.unique(ii, sorted=True, return_inverse=True)
    M = kx.numel()
    if eta.numel() != M * H * W:
        raise RuntimeError("JDSA: eta needs M*H*W values (M = %d distinct source frames)" % M)
    hs, ws = dscales.shape[1:]
    D = hs * ws
    gy, gx = grid_axes(H, W, hs, ws, dev)
    C = torch.empty((M, H * W), dtype=torch.float32, device=dev)
    w = torch.empty_like(C)
    dso = torch.empty((M, D), dtype=torch.float32, device=dev)
    out = torch.empty_like(d3)
    dzcov = torch.empty((M, H * W), dtype=torch.float32, device=dev) if with_dzcov else None
    info = torch.empty(1, dtype=torch.int32, device=dev)
    slot = slot.contiguous()
    _lib.check(_lib.load().hs2_jdsa(_ptr(pdata), pdata.shape[0], _ptr(d3), P, H, W, _ptr(intr), _ptr(target),
                                    _ptr(weight), _ptr(eta), _ptr(disps_prior), disps_prior.shape[0],
                                    _ptr(dscales), dscales.shape[0], hs, ws, _ptr(gy), _ptr(gx), _ptr(ii),
                                    _ptr(jj), _ptr(slot), E, _ptr(kx), M, float(alpha), _ptr(C), _ptr(w),
                                    _ptr(dso), _ptr(out), _ptr(dzcov), _ptr(info), _stream(dev)), "jdsa")
    bits = int(info.item())
    if bits & _lib.HS2_DEV_BAD_INDEX:
        raise RuntimeError("JDSA: an edge or source frame lies outside the pose / disparity / prior / scale "
                           "buffers")
    if bits & _lib.HS2_DEV_NOT_PD:
        raise torch.linalg.LinAlgError("JDSA: the reduced scale system is not positive definite")
    return (out[None] if batched else out), dscales, dzcov
