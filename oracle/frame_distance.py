"""``droid_backends.frame_distance`` restated in float64 numpy.

Follows HI-SLAM2 ``src/droid_kernels.cu:860-994`` (``frame_distance_kernel``) and
``:2047-2069`` (host wrapper).  Test infrastructure only.
"""

import numpy as np

from . import se3

MIN_DEPTH = 0.25  # src/droid_kernels.cu:26


def frame_distance(poses, disps, intrinsics, ii, jj, beta, chunk=256):
    """Per edge: beta-blend of the mean flow under the full relative pose and under
    translation only, over pixels whose transformed depth is > MIN_DEPTH (:920-973);
    1000 when the valid fraction is below 0.75 (:992)."""
    poses = np.asarray(poses, dtype=np.float64)
    disps = np.asarray(disps, dtype=np.float64)
    intr = np.asarray(intrinsics, dtype=np.float64)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    E = ii.shape[0]
    _, ht, wd = disps.shape
    HW = ht * wd
    vv, uu = np.meshgrid(np.arange(ht, dtype=np.float64), np.arange(wd, dtype=np.float64), indexing="ij")
    uu = uu.reshape(-1)[None]
    vv = vv.reshape(-1)[None]
    out = np.zeros(E)
    for s in range(0, E, chunk):
        e = slice(s, min(E, s + chunk))
        ie, je = ii[e], jj[e]
        tij, qij = se3.rel_se3(poses[ie, :3], poses[ie, 3:], poses[je, :3], poses[je, 3:])
        tij = tij[:, None]
        qij = qij[:, None]
        Xi = se3.iproj(uu, vv, disps[ie].reshape(-1, HW), intr)
        # full relative pose
        Xj = se3.act_se3(tij, qij, Xi)
        xp, yp = se3.proj(Xj, intr)
        d1 = np.sqrt((xp - uu) ** 2 + (yp - vv) ** 2)
        ok1 = Xj[..., 2] > MIN_DEPTH
        # translation only
        Xt = Xi[..., :3] + Xi[..., 3:4] * tij
        xt, yt = se3.proj(Xt, intr)
        d2 = np.sqrt((xt - uu) ** 2 + (yt - vv) ** 2)
        ok2 = Xt[..., 2] > MIN_DEPTH
        accum = beta * np.where(ok1, d1, 0.0).sum(-1) + (1 - beta) * np.where(ok2, d2, 0.0).sum(-1)
        valid = beta * ok1.sum(-1) + (1 - beta) * ok2.sum(-1)
        total = np.full(valid.shape, HW * (beta + (1 - beta)))
        with np.errstate(divide="ignore", invalid="ignore"):
            out[e] = np.where(valid / (total + 1e-8) < 0.75, 1000.0, accum / valid)
    return out
