"""The per-frame block form that ``csrc/jdsa.cu`` computes equals the reference's dense JDSA.

``hislam2/geom/ba.py:198-203`` scatters H and E with keys (kx', kx'), kx' = kx - kx[0], so
the [M*D, M*D] system of ``schur_solve_mono_prior`` is block diagonal.  This test restates
the kernel's algorithm in float64 numpy -- per block b the prior terms of frame kx[0] + b
(if it is a source frame) with row b of C, w, eta and the mask; S = sum alpha a^2 (1 - alpha
Q) w w^T + diag(0.1 + 1e-4 diag H); v = sum alpha a w (rd + Q w'); dz = Q (w' + alpha a
w.dso); dzcov = (alpha a Q)^2 w^T S^-1 w + Q -- and checks it against the dense oracle
(``oracle/jdsa.py``, pinned to the reference's own JDSA) on every fixture, including the
gapped source sets and the case whose block is not positive definite."""

import glob
import os

import numpy as np
import pytest

from oracle import geometry
from oracle import jdsa as ojdsa

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "jdsa_*.npz")))


def block_form(g):
    disps = g["disps"].astype(np.float64)
    prior = g["disps_prior"].astype(np.float64)
    dsc = g["dscales"].astype(np.float64)
    P, ht, wd = disps.shape
    HW = ht * wd
    hs, ws = dsc.shape[1:]
    D = hs * ws
    alpha = float(g["alpha"])
    C, w = geometry.proj_trans(g["poses"], g["disps"], g["intrinsics"], g["targets"], g["weights"], g["ii"], g["jj"])
    kx = np.unique(g["ii"])
    M = len(kx)
    eta = g["eta"].reshape(M, HW).astype(np.float64)
    gy, gx = ojdsa.grid_axes(ht, wd, hs, ws)
    yy, xx = np.meshgrid(gy.astype(np.float64), gx.astype(np.float64), indexing="ij")
    y, x = yy.reshape(-1), xx.reshape(-1)
    cy, cx = np.floor(y).astype(int), np.floor(x).astype(int)
    wt = np.stack([(cx + 1 - x) * (cy + 1 - y), (cx + 1 - x) * (y - cy), (x - cx) * (cy + 1 - y), (x - cx) * (y - cy)])
    pos = np.stack([cy * ws + cx, (cy + 1) * ws + cx, cy * ws + cx + 1, (cy + 1) * ws + cx + 1])
    interp = lambda sc: (wt * sc.reshape(-1)[pos]).sum(0)  # noqa: E731

    out = np.where(disps > 10, 0.0, disps)
    out = np.where(out < 0.001, 0.001, out)
    dso_all, cov = np.zeros((M, D)), np.zeros((M, HW))
    for b in range(M):
        fr = kx[b]
        src = np.nonzero(kx == kx[0] + b)[0]
        pr = prior[fr].reshape(-1)
        m = (pr > 0).astype(np.float64)
        rd = disps[fr].reshape(-1) - pr * interp(dsc[fr])
        Q = 1.0 / (C[b] + m * alpha + (1 - m) * eta[b])
        wq = w[b] - m * alpha * rd
        if len(src):
            fs = kx[src[0]]
            ps = prior[fs].reshape(-1)
            a = np.where(ps > 0, ps, 0.0)
            rds = disps[fs].reshape(-1) - ps * interp(dsc[fs])
        else:
            a, rds = np.zeros(HW), np.zeros(HW)
        Jw = np.zeros((HW, D))                      # the four bilinear weights at their positions
        np.put_along_axis(Jw, pos.T, wt.T, axis=1)
        S = np.einsum("p,pk,pl->kl", alpha * a * a * (1 - alpha * Q), Jw, Jw)
        Hd = np.einsum("p,pk->k", alpha * a * a, Jw * Jw)
        v = np.einsum("p,pk->k", alpha * a * (rds + Q * wq), Jw)
        S = S + np.diag(0.1 + 1e-4 * Hd)
        L = np.linalg.cholesky(S)                   # raises where the dense system does
        dso = np.linalg.solve(S, v)
        dso_all[b] = dso
        dz = Q * (wq + alpha * a * (Jw @ dso))
        cov[b] = (alpha * a * Q) ** 2 * np.einsum("pk,kl,pl->p", Jw, np.linalg.inv(L @ L.T), Jw) + Q
        d = disps[fr].reshape(-1) + dz
        d = np.where(d > 10, 0.0, d)
        out[fr] = np.where(d < 0.001, 0.001, d).reshape(ht, wd)
    sc = dsc.copy()
    sc.reshape(sc.shape[0], -1)[kx] += dso_all
    return dict(disps=out, dscales=sc, dzcov=cov, dso=dso_all)


@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_block_form_equals_dense_form(path):
    z = np.load(path)
    g = {k: z[k] for k in z.files}
    if bool(g["raised"]):
        with pytest.raises(np.linalg.LinAlgError):
            block_form(g)
        return
    r = block_form(g)
    d = ojdsa.jdsa(g["targets"], g["weights"], g["eta"], g["poses"], g["disps"], g["intrinsics"], g["disps_prior"],
                   g["dscales"], g["ii"], g["jj"], float(g["alpha"]))
    for k in ("disps", "dscales", "dzcov", "dso"):
        np.testing.assert_allclose(r[k], d[k], rtol=1e-9, atol=1e-12 * max(1.0, np.abs(d[k]).max()), err_msg=k)
