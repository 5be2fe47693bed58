"""``droid_backends.iproj``, ``covis_distance``, ``depth_filter``, ``proj_trans`` and
``bi_inter`` restated in float64 numpy.

Follows HI-SLAM2 ``src/droid_kernels.cu``: ``covis_distance_kernel`` (:996-1090),
``depth_filter_kernel`` (:1094-1204), ``iproj_kernel`` (:1208-1272),
``projective_transform2_kernel`` (:246-362), ``bi_inter_kernel`` (:1275-1316) and their
host wrappers (:1781-1818, :2071-2175).  Test infrastructure only.
"""

import numpy as np

from . import se3


def _pixels(ht, wd):
    vv, uu = np.meshgrid(np.arange(ht, dtype=np.float64), np.arange(wd, dtype=np.float64), indexing="ij")
    return uu.reshape(-1), vv.reshape(-1)


def iproj(poses, disps, intrinsics):
    """Per frame b and pixel: X = (xn, yn, 1, d) moved by poses[b] (actSE3), returned as
    X[:3] / X[3] (:1246-1270) -> points [N, H, W, 3]."""
    poses = np.asarray(poses, dtype=np.float64)
    disps = np.asarray(disps, dtype=np.float64)
    intr = np.asarray(intrinsics, dtype=np.float64)
    nm, ht, wd = disps.shape
    uu, vv = _pixels(ht, wd)
    X = se3.iproj(uu[None], vv[None], disps.reshape(nm, -1), intr)            # [nm, HW, 4]
    Y = se3.act_se3(poses[:nm, None, :3], poses[:nm, None, 3:], X)
    with np.errstate(divide="ignore", invalid="ignore"):
        pts = Y[..., :3] / Y[..., 3:4]
    return pts.reshape(nm, ht, wd, 3)


def covis_distance(poses, disps, intrinsics, ii):
    """Per entry i = ii[n]: the fraction of frame i's pixels that project outside the image
    under both Gij with j = i-1 and j = i+1 (:1040-1089)."""
    poses = np.asarray(poses, dtype=np.float64)
    disps = np.asarray(disps, dtype=np.float64)
    intr = np.asarray(intrinsics, dtype=np.float64)
    ii = np.asarray(ii, dtype=np.int64)
    _, ht, wd = disps.shape
    uu, vv = _pixels(ht, wd)
    out = np.zeros(ii.shape[0])
    for n, i in enumerate(ii):
        X = se3.iproj(uu, vv, disps[i].reshape(-1), intr)
        outside = np.ones(ht * wd, dtype=bool)
        for j in (i - 1, i + 1):
            tij, qij = se3.rel_se3(poses[i, :3], poses[i, 3:], poses[j, :3], poses[j, 3:])
            xp, yp = se3.proj(se3.act_se3(tij, qij, X), intr)
            outside &= (xp < 0) | (xp >= wd) | (yp < 0) | (yp >= ht)
        out[n] = outside.sum() / (ht * wd)
    return out


# neighbour offsets of depth_filter_kernel: jx = ix - n - 1 for n < 3, else ix + n (:1116)
DEPTH_FILTER_OFFSETS = (-1, -2, -3, 3, 4, 5)


def depth_filter(poses, disps, intrinsics, ix, thresh):
    """Per frame i = ix[b] and pixel: the number of neighbours j = i + offset (inside the
    buffer) in which the reprojected inverse depth lies within thresh[b] of one of the four
    disparities around the reprojection, tested in the order d00, d01, d10, d11
    (:1143-1203) -> counter [N, H, W]."""
    poses = np.asarray(poses, dtype=np.float64)
    disps = np.asarray(disps, dtype=np.float64)
    intr = np.asarray(intrinsics, dtype=np.float64)
    ix = np.asarray(ix, dtype=np.int64)
    thresh = np.asarray(thresh, dtype=np.float64)
    num, ht, wd = disps.shape
    uu, vv = _pixels(ht, wd)
    counter = np.zeros((ix.shape[0], ht * wd))
    for b, i in enumerate(ix):
        X = se3.iproj(uu, vv, disps[i].reshape(-1), intr)
        for off in DEPTH_FILTER_OFFSETS:
            j = i + off
            if j < 0 or j >= num:
                continue
            tij, qij = se3.rel_se3(poses[i, :3], poses[i, 3:], poses[j, :3], poses[j, 3:])
            Xj = se3.act_se3(tij, qij, X)
            uj, vj = se3.proj(Xj, intr)
            with np.errstate(divide="ignore", invalid="ignore"):
                dj = Xj[:, 3] / Xj[:, 2]
            u0 = np.floor(uj)
            v0 = np.floor(vj)
            ok = (u0 >= 0) & (v0 >= 0) & (u0 < wd - 1) & (v0 < ht - 1)
            u0i = np.where(ok, u0, 0).astype(np.int64)
            v0i = np.where(ok, v0, 0).astype(np.int64)
            dj_ = disps[j]
            with np.errstate(divide="ignore", invalid="ignore"):
                inv = 1.0 / dj
                hit = np.zeros(ht * wd, dtype=bool)
                for dv, du in ((0, 0), (0, 1), (1, 0), (1, 1)):
                    hit |= np.abs(inv - 1.0 / dj_[v0i + dv, u0i + du]) < thresh[b]
            counter[b] += ok & hit
    return counter.reshape(ix.shape[0], ht, wd)


MIN_DEPTH = 0.25  # src/droid_kernels.cu:26


def proj_trans(poses, disps, intrinsics, targets, weights, ii, jj):
    """``proj_trans_cuda`` (:1781-1818) with ``projective_transform2_kernel`` (:246-362): per
    edge and pixel the depth-only Schur terms C = wu Jzu^2 + wv Jzv^2 and w = wu ru Jzu +
    wv rv Jzv, summed over the edges leaving each frame of kx = unique(ii) (``accum_cuda``)
    -> (C [M, HW], w [M, HW]).  ``intrinsics`` may be [4] or [N, 4] (row 0 is used)."""
    poses = np.asarray(poses, dtype=np.float64)
    disps = np.asarray(disps, dtype=np.float64)
    intr = np.asarray(intrinsics, dtype=np.float64).reshape(-1, 4)[0]
    targets = np.asarray(targets, dtype=np.float64)
    weights = np.asarray(weights, dtype=np.float64)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    _, ht, wd = disps.shape
    HW = ht * wd
    kx, kk = np.unique(ii, return_inverse=True)
    uu, vv = _pixels(ht, wd)
    fx, fy = intr[0], intr[1]
    C = np.zeros((len(kx), HW))
    w = np.zeros((len(kx), HW))
    for e in range(len(ii)):
        tij, qij = se3.rel_se3(poses[ii[e], :3], poses[ii[e], 3:], poses[jj[e], :3], poses[jj[e], 3:])
        X = se3.iproj(uu, vv, disps[ii[e]].reshape(-1), intr)
        Xj = se3.act_se3(tij, qij, X)
        xp, yp = se3.proj(Xj, intr)
        ok = Xj[:, 2] >= MIN_DEPTH
        with np.errstate(divide="ignore", invalid="ignore"):
            d = np.where(ok, 1.0 / Xj[:, 2], 0.0)
        wu = np.where(ok, 0.001 * weights[e, 0].reshape(-1), 0.0)
        wv = np.where(ok, 0.001 * weights[e, 1].reshape(-1), 0.0)
        ru = targets[e, 0].reshape(-1) - xp
        rv = targets[e, 1].reshape(-1) - yp
        Jzu = fx * d * tij[0] + fx * (-Xj[:, 0] * d * d) * tij[2]
        Jzv = fy * d * tij[1] + fy * (-Xj[:, 1] * d * d) * tij[2]
        C[kk[e]] += wu * Jzu * Jzu + wv * Jzv * Jzv
        w[kk[e]] += np.where(wu != 0, wu * ru * Jzu, 0.0) + np.where(wv != 0, wv * rv * Jzv, 0.0)
    return C, w


def bi_inter(scales, grids):
    """``bi_inter_kernel`` (:1275-1316): bilinear interpolation of scales[b] at grids[b, i, j] =
    (x, y) and the dense Jacobian of each output w.r.t. the scale grid -> (outputs [N, H, W],
    jacobians [N, H, W, hs, ws])."""
    scales = np.asarray(scales, dtype=np.float64)
    grids = np.asarray(grids, dtype=np.float64)
    nm, ht, wd, _ = grids.shape
    hs, ws = scales.shape[1:]
    out = np.zeros((nm, ht, wd))
    jac = np.zeros((nm, ht, wd, hs, ws))
    for b in range(nm):
        for i in range(ht):
            for j in range(wd):
                x, y = grids[b, i, j]
                x0, y0 = int(np.floor(x)), int(np.floor(y))
                x1, y1 = x0 + 1, y0 + 1
                wa, wb = (x1 - x) * (y1 - y), (x1 - x) * (y - y0)
                wc, wdd = (x - x0) * (y1 - y), (x - x0) * (y - y0)
                out[b, i, j] = (wa * scales[b, y0, x0] + wb * scales[b, y1, x0] + wc * scales[b, y0, x1]
                                + wdd * scales[b, y1, x1])
                jac[b, i, j, y0, x0] = wa
                jac[b, i, j, y1, x0] = wb
                jac[b, i, j, y0, x1] = wc
                jac[b, i, j, y1, x1] = wdd
    return out, jac
