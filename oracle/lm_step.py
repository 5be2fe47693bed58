"""One Levenberg-Marquardt step of ``droid_backends.ba`` as a differentiable float64
PyTorch function (TEST INFRASTRUCTURE ONLY: the autograd reference for the
hand-written LM-step adjoint).

It restates the same operator as ``oracle/ba.py`` -- ``projective_transform_kernel``
(``src/droid_kernels.cu:364-606``: MIN_DEPTH 0.25 on the transformed depth, the
0.001 weight scale, self-edges keeping only their depth terms), the keyed
assembly (:1882-1889), the Schur complement over rows sharing a depth frame
(:1689-1779), the damped solve ``diag += ep + lm diag`` (:1660-1680) and the
back-substitution that skips the rows of the first window pose (:1562-1582,
:1920) -- with dense tensors, so that ``torch.autograd`` differentiates dx and dz
with respect to targets, weights and eta.  Poses and disparities (the
linearisation point) are constants.  Small problems only: the E matrix is dense
[6P, M*H*W].
"""

import numpy as np
import torch

from . import ba as oba
from . import se3

MIN_DEPTH = 0.25


def _jacobians(poses, disps, intr, ii, jj):
    """Per edge-pixel projection, validity and Jacobians in float64 (numpy, constants)."""
    K, ht, wd = disps.shape
    HW = ht * wd
    fx, fy = intr[0], intr[1]
    vv, uu = np.meshgrid(np.arange(ht, dtype=np.float64), np.arange(wd, dtype=np.float64), indexing="ij")
    uu, vv = uu.reshape(-1), vv.reshape(-1)
    tij, qij = se3.rel_se3(poses[ii, :3], poses[ii, 3:], poses[jj, :3], poses[jj, 3:])
    tij, qij = tij[:, None, :], qij[:, None, :]
    Xi = se3.iproj(uu[None], vv[None], disps[ii].reshape(-1, HW), intr)
    Xj = se3.act_se3(tij, qij, Xi)
    xp, yp = se3.proj(Xj, intr)
    bad = Xj[..., 2] < MIN_DEPTH
    x, y, h = Xj[..., 0], Xj[..., 1], Xj[..., 3]
    z = np.where(bad, 0.0, Xj[..., 2])
    d = np.where(bad, 0.0, 1.0 / np.where(bad, 1.0, Xj[..., 2]))
    d2 = d * d
    Jp = [fx * d, np.zeros_like(d), fx * (-x * d2), np.zeros_like(d), fy * d, fy * (-y * d2)]
    Jj_u = np.stack([Jp[0] * h, Jp[1] * h, Jp[2] * h,
                     -Jp[1] * z + Jp[2] * y, Jp[0] * z - Jp[2] * x, -Jp[0] * y + Jp[1] * x], -1)
    Jj_v = np.stack([Jp[3] * h, Jp[4] * h, Jp[5] * h,
                     -Jp[4] * z + Jp[5] * y, Jp[3] * z - Jp[5] * x, -Jp[3] * y + Jp[4] * x], -1)
    Jz_u = Jp[0] * tij[..., 0] + Jp[1] * tij[..., 1] + Jp[2] * tij[..., 2]
    Jz_v = Jp[3] * tij[..., 0] + Jp[4] * tij[..., 1] + Jp[5] * tij[..., 2]
    Ji_u = -se3.adj_se3(tij, qij, Jj_u)
    Ji_v = -se3.adj_se3(tij, qij, Jj_v)
    proj = np.stack([xp, yp], 1)                            # [E, 2, HW]
    Ji = np.stack([Ji_u, Ji_v], 1)                          # [E, 2, HW, 6]
    Jj = np.stack([Jj_u, Jj_v], 1)
    Jz = np.stack([Jz_u, Jz_v], 1)                          # [E, 2, HW]
    valid = (~bad)[:, None, :].repeat(2, 1)                 # [E, 2, HW]
    return proj, Ji, Jj, Jz, valid


def lm_step(poses, disps, intrinsics, targets, weights, eta, ii, jj, t0, t1, lm, ep):
    """dx [P, 6], dz [M, H*W] of one iteration of ``ba`` (motion_only = False).

    ``targets``, ``weights`` [E, 2, H, W] and ``eta`` [M or 1, H, W] are float64 torch
    tensors (they may require grad); the rest are numpy arrays / ints.
    """
    poses = np.asarray(poses, np.float64)
    disps = np.asarray(disps, np.float64)
    intr = np.asarray(intrinsics, np.float64)
    ii = np.asarray(ii, np.int64)
    jj = np.asarray(jj, np.int64)
    oba.validate(min(len(poses), len(disps)), ii, jj, t0, t1)
    E = len(ii)
    K, ht, wd = disps.shape
    HW = ht * wd
    P = t1 - t0
    proj, Ji, Jj, Jz, valid = _jacobians(poses, disps, intr, ii, jj)
    T = lambda a: torch.as_tensor(a, dtype=torch.float64)  # noqa: E731
    proj, Ji, Jj, Jz, valid = T(proj), T(Ji), T(Jj), T(Jz), T(valid.astype(np.float64))
    r = targets.reshape(E, 2, HW) - proj
    wd_ = 0.001 * weights.reshape(E, 2, HW) * valid          # depth terms: every edge
    selfe = T((ii == jj).astype(np.float64))[:, None, None]
    wp = wd_ * (1.0 - selfe)                                 # pose terms: self-edges dropped

    kx, kk_exp, ii_exp = oba.keys(ii, t0, t1)
    M = len(kx)
    slot = np.searchsorted(kx, ii)                           # depth frame slot of each edge
    a = ii - t0
    b = jj - t0
    n = 6 * P
    # pose block A, rhs b
    A = torch.zeros(n, n, dtype=torch.float64)
    bv = torch.zeros(n, dtype=torch.float64)
    Jfull = torch.zeros(E, 2, HW, n, dtype=torch.float64)
    for e in range(E):
        if 0 <= a[e] < P:
            Jfull[e, :, :, 6 * a[e]:6 * a[e] + 6] += Ji[e]
        if 0 <= b[e] < P:
            Jfull[e, :, :, 6 * b[e]:6 * b[e] + 6] += Jj[e]
    A = torch.einsum("ecpx,ecp,ecpy->xy", Jfull, wp, Jfull)
    bv = torch.einsum("ecpx,ecp,ecp->x", Jfull, wp, r)
    # depth blocks: C, gd per depth pixel; E couplings
    C = torch.zeros(M, HW, dtype=torch.float64)
    gd = torch.zeros(M, HW, dtype=torch.float64)
    C = C.index_add(0, T(slot).long(), (wd_ * Jz * Jz).sum(1))
    gd = gd.index_add(0, T(slot).long(), (wd_ * Jz * r).sum(1))
    Em = torch.zeros(n, M, HW, dtype=torch.float64)
    contrib = torch.einsum("ecpx,ecp,ecp->exp", Jfull, wp, Jz)  # [E, n, HW]
    Em = Em.index_add(1, T(slot).long(), contrib.permute(1, 0, 2))
    etaf = eta.reshape(-1, HW).expand(M, HW)
    Q = 1.0 / (C + etaf)
    Ef = Em.reshape(n, M * HW)
    Qf = Q.reshape(-1)
    R = A - (Ef * Qf) @ Ef.t()
    y = bv - Ef @ (Qf * gd.reshape(-1))
    Rd = R + torch.diag(ep + lm * torch.diagonal(R))
    L = torch.linalg.cholesky(Rd)
    dx = torch.cholesky_solve(y[:, None], L)[:, 0]
    # back-substitution without the rows of window pose 0
    keep = torch.ones(n, dtype=torch.float64)
    keep[:6] = 0.0
    dz = Q * (gd - ((Ef * keep[:, None]).t() @ dx).reshape(M, HW))
    return dx.reshape(P, 6), dz


def lm_step_adjoint(poses, disps, intrinsics, targets, weights, eta, ii, jj, t0, t1, lm, ep, gdx, gdz):
    """Closed-form adjoint of :func:`lm_step` (float64 numpy): given dL/ddx [P,6] and
    dL/ddz [M,HW], returns dL/dtargets, dL/dweights [E,2,H,W] and dL/deta (eta's shape).

    With M_d the damped system solved by the step (pose block A + ep + lm diag(R),
    R = A - E Q E^T, depth block C + eta), lam = R_d^-1 (gdx - E~ Q gdz) and the
    rank-2 + diagonal adjoint of R_d, every per-pixel term reduces to the scalars
    s_lam = E_k . lam, s_x = E_k . dx (E_k = column k of the pose/depth coupling);
    this is the formula the GPU adjoint kernels implement.
    """
    poses = np.asarray(poses, np.float64)
    disps = np.asarray(disps, np.float64)
    intr = np.asarray(intrinsics, np.float64)
    ii = np.asarray(ii, np.int64)
    jj = np.asarray(jj, np.int64)
    targets = np.asarray(targets, np.float64)
    weights = np.asarray(weights, np.float64)
    eta = np.asarray(eta, np.float64)
    E = len(ii)
    K, ht, wd = disps.shape
    HW = ht * wd
    P = t1 - t0
    n = 6 * P
    proj, Ji, Jj, Jz, valid = _jacobians(poses, disps, intr, ii, jj)
    r = targets.reshape(E, 2, HW) - proj
    wd_ = 0.001 * weights.reshape(E, 2, HW) * valid
    wp = wd_ * (ii != jj)[:, None, None]
    kx, _, _ = oba.keys(ii, t0, t1)
    M = len(kx)
    slot = np.searchsorted(kx, ii)
    a, b = ii - t0, jj - t0
    ina, inb = (a >= 0) & (a < P), (b >= 0) & (b < P)
    # forward quantities
    A = np.zeros((n, n))
    bv = np.zeros(n)
    Em = np.zeros((n, M, HW))
    C = np.zeros((M, HW))
    gd = np.zeros((M, HW))
    for e in range(E):
        Jf = np.zeros((2, HW, n))
        if ina[e]:
            Jf[:, :, 6 * a[e]:6 * a[e] + 6] += Ji[e]
        if inb[e]:
            Jf[:, :, 6 * b[e]:6 * b[e] + 6] += Jj[e]
        A += np.einsum("cpx,cp,cpy->xy", Jf, wp[e], Jf)
        bv += np.einsum("cpx,cp,cp->x", Jf, wp[e], r[e])
        Em[:, slot[e]] += np.einsum("cpx,cp,cp->xp", Jf, wp[e], Jz[e])
        C[slot[e]] += (wd_[e] * Jz[e] ** 2).sum(0)
        gd[slot[e]] += (wd_[e] * Jz[e] * r[e]).sum(0)
    etaf = np.broadcast_to(eta.reshape(-1, HW), (M, HW))
    Q = 1.0 / (C + etaf)
    Ef = Em.reshape(n, M * HW)
    R = A - (Ef * Q.reshape(-1)) @ Ef.T
    Rd = R + np.diag(ep + lm * np.diag(R))
    y = bv - Ef @ (Q * gd).reshape(-1)
    Lc = np.linalg.cholesky(Rd)
    dx = np.linalg.solve(Lc.T, np.linalg.solve(Lc, y))
    keep = np.ones(n)
    keep[:6] = 0.0
    Et = Ef * keep[:, None]
    gdz = np.asarray(gdz, np.float64).reshape(M, HW)
    gdx = np.asarray(gdx, np.float64).reshape(n)
    # adjoint solve
    rhs = gdx - Et @ (Q * gdz).reshape(-1)
    lam = np.linalg.solve(Lc.T, np.linalg.solve(Lc, rhs))
    s_l = (Ef * lam[:, None]).sum(0).reshape(M, HW)
    s_x = (Ef * dx[:, None]).sum(0).reshape(M, HW)
    s_xt = (Et * dx[:, None]).sum(0).reshape(M, HW)
    ld = lam * dx
    s_e2 = ((Ef ** 2) * ld[:, None]).sum(0).reshape(M, HW)
    gQ = gdz * (gd - s_xt) - s_l * gd + s_l * s_x + lm * s_e2
    ggd = Q * (gdz - s_l)
    gC = -(Q ** 2) * gQ
    # per edge-pixel
    gw = np.zeros((E, 2, HW))
    gt = np.zeros((E, 2, HW))
    for e in range(E):
        k = slot[e]
        for c in range(2):
            u = np.zeros(HW)
            v = np.zeros(HW)
            vt = np.zeros(HW)
            dmp = np.zeros(HW)
            ebar = np.zeros(HW)
            for inside, blk, J in ((ina[e], a[e], Ji[e, c]), (inb[e], b[e], Jj[e, c])):
                if not inside:
                    continue
                sl = slice(6 * blk, 6 * blk + 6)
                u += J @ lam[sl]
                v += J @ dx[sl]
                if blk >= 1:
                    vt += J @ dx[sl]
                dmp += (J ** 2) @ ld[sl]
                ebar += (J * Em[sl, k].T) @ ld[sl]
            pose_w = -u * v - lm * dmp + u * r[e, c] + \
                Jz[e, c] * Q[k] * (-gdz[k] * vt - gd[k] * u + s_x[k] * u + s_l[k] * v + 2 * lm * ebar)
            depth_w = gC[k] * Jz[e, c] ** 2 + ggd[k] * Jz[e, c] * r[e, c]
            selfe = ii[e] == jj[e]
            gw[e, c] = 0.001 * valid[e, c] * ((0.0 if selfe else pose_w) + depth_w)
            gt[e, c] = (0.0 if selfe else 1.0) * wp[e, c] * u + ggd[k] * wd_[e, c] * Jz[e, c]
    geta = gC if eta.reshape(-1, HW).shape[0] == M else gC.sum(0, keepdims=True)
    return gt.reshape(E, 2, ht, wd), gw.reshape(E, 2, ht, wd), geta.reshape(eta.shape)
