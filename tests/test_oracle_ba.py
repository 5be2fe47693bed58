"""The BA oracle checked by identities that do not depend on its own code path.

* Jacobians, gradients and the depth blocks of ``oracle.ba.linearize`` against
  central finite differences of an independently written reprojection residual.
* The Schur step (dx from the reduced camera system, dz by back-substitution)
  against the residual of the full joint (pose + depth) damped normal equations.
* Keys against ``np.unique``; the per-frame Schur rows against the reference's
  quadruple loop (``schur_pairs``).
"""

import numpy as np
import pytest
import torch

from hislam2_b200 import synth
from oracle import ba as oba
from oracle import se3


def small_problem(name="frontend_small", seed=0, crop=(12, 16), edges=None):
    p = synth.make_ba_problem(name, seed)
    h, w = crop
    out = {k: v for k, v in p.items()}
    out["disps"] = p["disps"][:, :h, :w].contiguous()
    out["targets"] = p["targets"][:, :, :h, :w].contiguous()
    out["weights"] = p["weights"][:, :, :h, :w].contiguous()
    out["eta"] = p["eta"][:, :h, :w].contiguous()
    if edges is not None:
        for k in ("ii", "jj", "targets", "weights"):
            out[k] = out[k][edges]
    out = {k: (v.numpy().astype(np.float64) if isinstance(v, torch.Tensor) and v.is_floating_point() else
               (v.numpy() if isinstance(v, torch.Tensor) else v)) for k, v in out.items()}
    # unit quaternions in float64, so that any rotation formula agrees to rounding
    q = out["poses"][:, 3:]
    out["poses"][:, 3:] = q / np.linalg.norm(q, axis=1, keepdims=True)
    return out


def project(poses, disps, intr, ii, jj):
    """Independent restatement: pixel grid of ii mapped into jj; returns x, y, z [E,HW]."""
    K, h, w = disps.shape
    fx, fy, cx, cy = intr
    v, u = np.meshgrid(np.arange(h, dtype=np.float64), np.arange(w, dtype=np.float64), indexing="ij")
    u, v = u.reshape(-1), v.reshape(-1)
    X = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u)], -1)
    out = []
    for a, b in zip(ii, jj):
        # world<-camera conventions do not matter here: Gij = Gj Gi^-1 built by composition
        Ri = quat_to_R(poses[a, 3:])
        Rj = quat_to_R(poses[b, 3:])
        R = Rj @ Ri.T
        t = poses[b, :3] - R @ poses[a, :3]
        d = disps[a].reshape(-1)
        Y = X @ R.T + d[:, None] * t
        out.append(Y)
    Y = np.stack(out)
    return fx * Y[..., 0] / Y[..., 2] + cx, fy * Y[..., 1] / Y[..., 2] + cy, Y[..., 2]


def quat_to_R(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def perturb(poses, k, xi):
    out = poses.copy()
    t, q = se3.retr_se3(xi, poses[k, :3], poses[k, 3:])
    out[k, :3], out[k, 3:] = t, q
    return out


def test_linearize_matches_finite_differences():
    p = small_problem(edges=[0, 4, 9, 17])
    P, D, I = p["poses"], p["disps"], p["intrinsics"]
    ii, jj = p["ii"], p["jj"]
    lin = oba.linearize(P, D, I, p["targets"], p["weights"], ii, jj)
    HW = D.shape[1] * D.shape[2]
    x0, y0, z0 = project(P, D, I, ii, jj)
    valid = z0 >= oba.MIN_DEPTH
    wgt = 0.001 * p["weights"].reshape(len(ii), 2, HW) * valid[:, None]
    res = p["targets"].reshape(len(ii), 2, HW) - np.stack([x0, y0], 1)
    eps = 1e-6
    for e, (a, b) in enumerate(zip(ii, jj)):
        Jj = np.zeros((2, HW, 6))
        Ji = np.zeros((2, HW, 6))
        for k in range(6):
            xi = np.zeros(6)
            xi[k] = eps
            xp, yp, _ = project(perturb(P, b, xi), D, I, [a], [b])
            xm, ym, _ = project(perturb(P, b, -xi), D, I, [a], [b])
            Jj[0, :, k], Jj[1, :, k] = (xp[0] - xm[0]) / (2 * eps), (yp[0] - ym[0]) / (2 * eps)
            xp, yp, _ = project(perturb(P, a, xi), D, I, [a], [b])
            xm, ym, _ = project(perturb(P, a, -xi), D, I, [a], [b])
            Ji[0, :, k], Ji[1, :, k] = (xp[0] - xm[0]) / (2 * eps), (yp[0] - ym[0]) / (2 * eps)
        Dp = D.copy()
        Dp[a] += eps
        Dm = D.copy()
        Dm[a] -= eps
        xp, yp, _ = project(P, Dp, I, [a], [b])
        xm, ym, _ = project(P, Dm, I, [a], [b])
        Jz = np.stack([(xp[0] - xm[0]) / (2 * eps), (yp[0] - ym[0]) / (2 * eps)])  # [2,HW]
        we, re = wgt[e], res[e]
        Hjj = np.einsum("cp,cpa,cpb->ab", we, Jj, Jj)
        Hij = np.einsum("cp,cpa,cpb->ab", we, Ji, Jj)
        Hii = np.einsum("cp,cpa,cpb->ab", we, Ji, Ji)
        scale = np.abs(Hjj).max()
        np.testing.assert_allclose(lin["Hs"][3, e], Hjj, atol=1e-6 * scale)
        np.testing.assert_allclose(lin["Hs"][1, e], Hij, atol=1e-6 * scale)
        np.testing.assert_allclose(lin["Hs"][2, e], Hij.T, atol=1e-6 * scale)
        np.testing.assert_allclose(lin["Hs"][0, e], Hii, atol=1e-6 * scale)
        vj = np.einsum("cp,cp,cpa->a", we, re, Jj)
        vi = np.einsum("cp,cp,cpa->a", we, re, Ji)
        np.testing.assert_allclose(lin["vs"][1, e], vj, atol=1e-6 * np.abs(vj).max())
        np.testing.assert_allclose(lin["vs"][0, e], vi, atol=1e-6 * np.abs(vi).max())
        C = (we * Jz * Jz).sum(0)
        wz = (we * re * Jz).sum(0)
        np.testing.assert_allclose(lin["Cii"][e], C, atol=1e-6 * np.abs(C).max())
        np.testing.assert_allclose(lin["wi"][e], wz, atol=1e-6 * np.abs(wz).max())
        Eij = np.einsum("cp,cp,cpa->ap", we, Jz, Jj)
        Eii = np.einsum("cp,cp,cpa->ap", we, Jz, Ji)
        np.testing.assert_allclose(lin["Eij"][e], Eij, atol=1e-6 * np.abs(Eij).max())
        np.testing.assert_allclose(lin["Eii"][e], Eii, atol=1e-6 * np.abs(Eii).max())


def test_self_edge_contributes_nothing():
    # Gii = identity: the pose terms are zeroed explicitly (droid_kernels.cu:493,525) and the
    # depth terms vanish with tij = 0
    p = small_problem(edges=[0, 1])
    p["jj"] = p["ii"].copy()
    lin = oba.linearize(p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], p["ii"], p["jj"])
    for k in ("Hs", "vs", "Eij", "Eii", "Cii", "wi"):
        assert np.all(lin[k] == 0), k


def test_schur_step_solves_joint_system():
    p = small_problem()
    t0, t1, lm, ep = p["t0"], p["t1"], p["lm"], p["ep"]
    ii, jj = p["ii"], p["jj"]
    P = t1 - t0
    lin = oba.linearize(p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], ii, jj)
    A, b = oba.assemble_pose_system(lin["Hs"], lin["vs"], ii, jj, t0, P)
    kx, kk_exp, ii_exp = oba.keys(ii, t0, t1)
    jj_exp = np.concatenate([np.arange(t0, t1), jj])
    HW = lin["Cii"].shape[1]
    C = oba.accum(lin["Cii"], ii, kx)
    w = oba.accum(lin["wi"], ii, kx)
    Dg = C + p["eta"].reshape(-1, HW)
    Q = 1.0 / Dg
    Ei = oba.accum(lin["Eii"].reshape(len(ii), -1), ii, np.arange(t0, t1)).reshape(P, 6, HW)
    E = np.concatenate([Ei, lin["Eij"]])
    S, bS = oba.schur_complement(E, Q, w, jj_exp, kk_exp, t0, t1)
    dx, ok = oba.solve(A - S, b - bS, lm, ep)
    assert ok
    dz = oba.back_substitute(E, Q, w, dx, ii_exp, jj_exp, kx, t0, P, skip_t0=False)
    # joint system [A_d B; B^T D] [dx; dz] = [b; w]; the reference damps the diagonal of the
    # reduced matrix A - S (SparseBlock::solve, droid_kernels.cu:1663-1664)
    Ad = A.copy()
    di = np.arange(6 * P)
    Ad[di, di] += ep + lm * (A - S)[di, di]
    Bdz = np.zeros((P, 6))
    BTdx = np.zeros_like(dz)
    for n in range(E.shape[0]):
        pose = jj_exp[n] - t0
        if 0 <= pose < P:
            Bdz[pose] += E[n] @ dz[kk_exp[n]]
            BTdx[kk_exp[n]] += dx[pose] @ E[n]
    r1 = Ad @ dx.reshape(-1) + Bdz.reshape(-1) - b
    r2 = BTdx + Dg * dz - w
    assert np.abs(r1).max() < 1e-9 * max(1.0, np.abs(b).max())
    assert np.abs(r2).max() < 1e-9 * max(1.0, np.abs(w).max())


def test_reference_skip_of_first_window_pose():
    """back_substitute keeps the reference's ix <= 0 skip (droid_kernels.cu:1572)."""
    rng = np.random.default_rng(0)
    P, HW = 3, 5
    E = rng.standard_normal((P + 2, 6, HW))
    Q = rng.random((2, HW)) + 0.5
    w = rng.standard_normal((2, HW))
    dx = rng.standard_normal((P, 6))
    ii_exp = np.array([4, 5, 6, 4, 5])
    jj_exp = np.array([4, 5, 6, 5, 4])
    kx = np.array([4, 5, 6])
    Qk = np.concatenate([Q, Q[:1]])
    wk = np.concatenate([w, w[:1]])
    dz_ref = oba.back_substitute(E, Qk, wk, dx, ii_exp, jj_exp, kx, 4, P)
    dz_all = oba.back_substitute(E, Qk, wk, dx, ii_exp, jj_exp, kx, 4, P, skip_t0=False)
    # rows with pose t0 (n = 0 and n = 4) only enter dz_all
    diff = dz_all - dz_ref
    np.testing.assert_allclose(diff[0], -Qk[0] * (E[0].T @ dx[0]), atol=1e-12)
    np.testing.assert_allclose(diff[1], -Qk[1] * (E[4].T @ dx[0]), atol=1e-12)


def test_keys_and_schur_rows_match_reference_loops():
    p = synth.make_ba_problem("frontend", seed=3)
    ii, jj = p["ii"].numpy(), p["jj"].numpy()
    t0, t1 = 2, 25
    kx, kk_exp, ii_exp = oba.keys(ii, t0, t1)
    u, inv = np.unique(np.concatenate([np.arange(t0, t1), ii]), return_inverse=True)
    assert np.array_equal(kx, u) and np.array_equal(kk_exp, inv)
    jj_exp = np.concatenate([np.arange(t0, t1), jj])
    pairs = oba.schur_pairs(jj_exp, kk_exp, t0, t1)
    rows = oba.schur_rows(jj_exp, kk_exp, t0, t1)
    from_rows = []
    for k, rr in rows.items():
        for a in rr:
            for b in rr:
                from_rows.append((jj_exp[a] - t0, jj_exp[b] - t0, a, b, k))
    assert sorted(pairs) == sorted(from_rows)


def test_assemble_matches_direct_loop():
    rng = np.random.default_rng(1)
    E, t0, P = 7, 2, 4
    ii = np.array([0, 2, 3, 5, 2, 4, 1])
    jj = np.array([2, 3, 4, 4, 5, 1, 0])
    Hs = rng.standard_normal((4, E, 6, 6))
    vs = rng.standard_normal((2, E, 6))
    A, b = oba.assemble_pose_system(Hs, vs, ii, jj, t0, P)
    A2 = np.zeros((6 * P, 6 * P))
    b2 = np.zeros(6 * P)
    keys_r = np.concatenate([ii, ii, jj, jj]) - t0
    keys_c = np.concatenate([ii, jj, ii, jj]) - t0
    H = Hs.reshape(-1, 6, 6)
    for n in range(len(keys_r)):
        i, j = keys_r[n], keys_c[n]
        if i >= 0 and j >= 0:
            A2[6 * i:6 * i + 6, 6 * j:6 * j + 6] += H[n]
    for n, i in enumerate(np.concatenate([ii, jj]) - t0):
        if i >= 0:
            b2[6 * i:6 * i + 6] += vs.reshape(-1, 6)[n]
    np.testing.assert_allclose(A, A2)
    np.testing.assert_allclose(b, b2)


def test_failed_factorisation_gives_zero_update():
    A = -np.eye(12)
    dx, ok = oba.solve(A, np.ones(12), 1e-4, 0.1)
    assert not ok and np.all(dx == 0)


def test_ba_reduces_reprojection_error_and_motion_only():
    p = small_problem(crop=(24, 32))
    args = (p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], p["eta"], p["ii"], p["jj"],
            p["t0"], p["t1"])

    def cost(poses, disps):
        x, y, z = project(poses, disps, p["intrinsics"], p["ii"], p["jj"])
        HW = x.shape[1]
        wgt = 0.001 * p["weights"].reshape(len(x), 2, HW) * (z >= oba.MIN_DEPTH)[:, None]
        r = p["targets"].reshape(len(x), 2, HW) - np.stack([x, y], 1)
        return float((wgt * r * r).sum())

    c0 = cost(p["poses"], p["disps"])
    r = oba.ba(*args, 2, p["lm"], p["ep"])
    assert cost(r.poses, r.disps) < c0
    assert r.dz.shape == (len(r.kx), 24 * 32)
    rm = oba.ba(*args, 2, p["lm"], p["ep"], motion_only=True)
    assert rm.dz is None
    np.testing.assert_array_equal(rm.disps, p["disps"])
    assert np.abs(rm.poses[p["t0"]:] - p["poses"][p["t0"]:]).max() > 0
    np.testing.assert_array_equal(rm.poses[:p["t0"]], p["poses"][:p["t0"]])


def test_validation_rejects_out_of_window_indices():
    p = small_problem()
    with pytest.raises(ValueError):
        oba.validate(8, p["ii"], p["jj"], 2, 6)        # edges reach frame 7 >= t1
    with pytest.raises(ValueError):
        oba.validate(8, np.array([-1]), np.array([0]), 0, 8)


def test_empty_window_and_no_edges():
    p = small_problem()
    r = oba.ba(p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], p["eta"], p["ii"], p["jj"],
               8, 8, 1, p["lm"], p["ep"])
    assert r.dx.shape == (0, 6) and r.dz.shape[0] == 8
    e = np.zeros(0, dtype=np.int64)
    r = oba.ba(p["poses"], p["disps"], p["intrinsics"], p["targets"][:0], p["weights"][:0], p["eta"][2:], e, e,
               2, 8, 1, p["lm"], p["ep"])
    assert np.all(r.dx == 0) and np.all(r.dz == 0)
