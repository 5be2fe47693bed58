"""HI-SLAM2's mono-prior depth/scale alignment step ``JDSA`` restated in float64 numpy.

TEST INFRASTRUCTURE ONLY (the checker of ``hs2_jdsa``; never on a product path).

Follows ``hislam2/geom/ba.py:JDSA`` (:170-219), ``get_prior_depth_aligned`` (:159-167)
and ``hislam2/geom/chol.py:schur_solve_mono_prior`` (:80-107) literally, in their own
dense form: the scale Jacobian ``Jso`` [M, HW, D] from ``bi_inter``, ``Hs``/``Es``/``vs``
scattered with ``safe_scatter_add_mat/vec`` (:13-19, keys ``kx - kx[0]``, out-of-range
keys dropped), ``C`` and ``w`` from ``proj_trans`` plus the prior terms, the damped
``H + (ep + lm H) I`` with ep = 0.1 and lm = 1e-4, the Schur complement over all M*HW
depth unknowns, one Cholesky of the [M*D, M*D] system, ``dz = Q (w - E^T dso)``,
``dzcov = sum((L^-1 E Q)^2) + Q``, then ``disps[kx] += dz``, ``dscales[kx] += dso``,
``disps > 10 -> 0`` and ``clamp(min=0.001)`` over the whole window.  The operators
``proj_trans`` and ``bi_inter`` are ``oracle.geometry``'s (pinned to the reference's
compiled kernels by the ``geo_*`` fixtures).

The sampling grid is ``torch.linspace(0, hs-1-1e-6, ht)`` x ``linspace(0, ws-1-1e-6,
wd)`` in float32, as the reference builds it; ``grid_axes`` returns both axes.
"""

import numpy as np
import torch

from . import geometry

EP = 0.1      # schur_solve_mono_prior default (hislam2/geom/chol.py:80)
LM = 0.0001


def grid_axes(ht, wd, hs, ws):
    """(gy [ht], gx [wd]) float32: the grid of ``get_prior_depth_aligned`` (:161-163)."""
    gy = torch.linspace(0, hs - 1 - 1e-6, ht).numpy()
    gx = torch.linspace(0, ws - 1 - 1e-6, wd).numpy()
    return gy, gx


def jdsa(targets, weights, eta, poses, disps, intrinsics, disps_prior, dscales, ii, jj, alpha):
    """One JDSA step.  disps [P, H, W] (the reference's ``disps[0]``), dscales [P, hs, ws],
    disps_prior [>= max(ii)+1, H, W], eta with M*H*W elements (M = len(unique(ii))).
    Returns dict(disps [P,H,W], dscales [P,hs,ws], dzcov [M,HW], dso [M,D], dz [M,HW],
    kx [M]).  Raises ``np.linalg.LinAlgError`` when the reduced system is not positive
    definite (the reference's ``torch.linalg.inv`` of the zero factor raises there)."""
    disps = np.asarray(disps, dtype=np.float64)
    dscales = np.asarray(dscales, dtype=np.float64)
    prior_all = np.asarray(disps_prior, dtype=np.float64)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    P, ht, wd = disps.shape
    HW = ht * wd
    C, w = geometry.proj_trans(poses, disps, intrinsics, targets, weights, ii, jj)       # :179
    kx = np.unique(ii)                                                                   # :181
    M = len(kx)
    prior = prior_all[kx]                                                                # :184
    m = (prior > 0).astype(np.float64).reshape(M, HW)                                    # :185
    hs, ws = dscales.shape[1:]
    gy, gx = grid_axes(ht, wd, hs, ws)
    grid = np.stack(np.broadcast_arrays(gx[None, :], gy[:, None]), -1)                  # (x, y)
    sbi, Jbi = geometry.bi_inter(dscales[kx], np.broadcast_to(grid, (M, ht, wd, 2)))    # :165
    disps_bi = prior * sbi                                                               # :166
    rd = (disps[kx] - disps_bi).reshape(M, HW)                                           # :190
    Jd = np.ones((M, HW))
    D = hs * ws
    Jso = -m[..., None] * prior.reshape(M, HW)[..., None] * Jbi.reshape(M, HW, D)       # :193
    a = float(alpha)
    # safe_scatter_add_mat(A, kx', kx', M, M) with kx' = kx - kx[0] (:198-203)
    kxr = kx - kx[0]
    keep = (kxr >= 0) & (kxr < M)
    Hs = np.zeros((M, D, D))
    Es = np.zeros((M, D, HW))
    vs = np.zeros((M, D))
    for f in np.nonzero(keep)[0]:
        b = kxr[f]
        Hs[b] += np.einsum("pk,pl->kl", a * Jso[f], Jso[f])
        Es[b] += (a * Jso[f]).T * Jd[f][None]
        vs[b] += -(a * Jso[f]).T @ rd[f]
    Cf = C + m * a * Jd * Jd + (1 - m) * np.asarray(eta, dtype=np.float64).reshape(M, HW)   # :206
    wf = w - m * a * rd * Jd                                                             # :207
    # schur_solve_mono_prior (chol.py:80-107), dense
    Q = 1.0 / Cf.reshape(-1)
    H = np.zeros((M * D, M * D))
    E = np.zeros((M * D, M * HW))
    for b in range(M):
        H[b * D:(b + 1) * D, b * D:(b + 1) * D] = Hs[b]
        E[b * D:(b + 1) * D, b * HW:(b + 1) * HW] = Es[b]
    H = H + np.diag(EP + LM * np.diag(H))
    S = H - (E * Q[None]) @ E.T
    v = vs.reshape(-1) - E @ (Q * wf.reshape(-1))
    L = np.linalg.cholesky(S)
    dso = np.linalg.solve(L.T, np.linalg.solve(L, v))
    dz = Q * (wf.reshape(-1) - E.T @ dso)
    F = np.linalg.solve(L, E * Q[None])
    dzcov = (F * F).sum(0) + Q
    # retraction and clean-up (:214-219)
    out = disps.copy()
    out[kx] += dz.reshape(M, ht, wd)
    sc = dscales.copy()
    sc[kx] += dso.reshape(M, hs, ws)
    out = np.where(out > 10, 0.0, out)
    out = np.where(out < 0.001, 0.001, out)
    return dict(disps=out, dscales=sc, dzcov=dzcov.reshape(M, HW), dso=dso.reshape(M, D),
                dz=dz.reshape(M, HW), kx=kx)
