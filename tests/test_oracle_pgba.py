"""The pgba oracle checked by identities that do not depend on its own code path.

* Jj, the depth column, Hjj, vj, C, w and Eij of ``oracle.pgba.linearize_sim3`` against
  central finite differences of an independently written Sim3 reprojection.
* Ji against the reference's map written independently as a 7x7 matrix
  (``adjSim3``, ``src/droid_kernels.cu:122-145``); that map is NOT the derivative of
  the reprojection in its rotation and scale columns, which is recorded here as the
  reference behaviour kept for parity.
* The Schur step (with relative-pose factors) against the joint damped normal
  equations; the factor blocks against a direct loop with keys below t0 dropped.
"""

import numpy as np
import pytest

from hislam2_b200 import synth
from oracle import ba as oba
from oracle import pgba as opg
from oracle import se3


def small(seed=0, crop=(12, 16), edges=None, num_factors=None):
    p = synth.make_pgba_problem("frontend_small", seed, num_factors=num_factors)
    h, w = crop
    out = dict(p)
    out["disps"] = p["disps"][:, :h, :w]
    out["targets"] = p["targets"][:, :, :h, :w]
    out["weights"] = p["weights"][:, :, :h, :w]
    out["eta"] = p["eta"][:, :h, :w]
    if edges is not None:
        for k in ("ii", "jj", "targets", "weights"):
            out[k] = out[k][edges]
    out = {k: (v.numpy().astype(np.float64) if hasattr(v, "is_floating_point") and v.is_floating_point() else
               (v.numpy() if hasattr(v, "numpy") else v)) for k, v in out.items()}
    q = out["poses"][:, 3:7]
    out["poses"][:, 3:7] = q / np.linalg.norm(q, axis=1, keepdims=True)
    return out


def quat_to_R(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def rot(phi):
    th = np.linalg.norm(phi)
    if th < 1e-15:
        return np.eye(3)
    k = phi / th
    Kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(th) * Kx + (1 - np.cos(th)) * Kx @ Kx


def project(G, disps, intr, a, b):
    """Pixels of frame a mapped into frame b under Gab = Gb Ga^-1, Sim3 G = (R, t, s):
    Y = sab Rab X + d tab.  Returns x, y, z [HW]."""
    h, w = disps.shape[1:]
    fx, fy, cx, cy = intr
    v, u = np.meshgrid(np.arange(h, dtype=np.float64), np.arange(w, dtype=np.float64), indexing="ij")
    X = np.stack([(u.reshape(-1) - cx) / fx, (v.reshape(-1) - cy) / fy, np.ones(h * w)], -1)
    (Ra, ta, sa), (Rb, tb, sb) = G[a], G[b]
    R = Rb @ Ra.T
    s = sb / sa
    t = tb - s * R @ ta
    Y = s * X @ R.T + disps[a].reshape(-1)[:, None] * t
    return fx * Y[:, 0] / Y[:, 2] + cx, fy * Y[:, 1] / Y[:, 2] + cy, Y[:, 2]


def sim3_of(poses):
    return [(quat_to_R(p[3:7]), p[:3].copy(), float(p[7])) for p in poses]


def perturb(G, k, delta):
    """Left perturbation exp(delta) * G_k, delta = [tau, phi, sigma] along one axis."""
    out = list(G)
    R, t, s = G[k]
    dR, ds = rot(delta[3:6]), np.exp(delta[6])
    out[k] = (dR @ R, ds * dR @ t + delta[:3], ds * s)
    return out


def adj_matrix(t, q, s):
    """The reference's adjSim3 as a matrix M (Y = M X): rows [s R^T, 0, 0],
    [-s R^T [t]x, s R^T, t], [0, 0, 1]."""
    R = quat_to_R(q)
    tx = np.array([[0, -t[2], t[1]], [t[2], 0, -t[0]], [-t[1], t[0], 0]])
    M = np.zeros((7, 7))
    M[:3, :3] = s * R.T
    M[3:6, :3] = -s * R.T @ tx
    M[3:6, 3:6] = s * R.T
    M[3:6, 6] = t
    M[6, 6] = 1.0
    return M


def fd_jacobians(p, a, b, eps=1e-6):
    G = sim3_of(p["poses"])
    D, I = p["disps"], p["intrinsics"]
    HW = D.shape[1] * D.shape[2]
    Jj, Ji = np.zeros((2, HW, 7)), np.zeros((2, HW, 7))
    for k in range(7):
        dl = np.zeros(7)
        dl[k] = eps
        for J, f in ((Jj, b), (Ji, a)):
            xp, yp, _ = project(perturb(G, f, dl), D, I, a, b)
            xm, ym, _ = project(perturb(G, f, -dl), D, I, a, b)
            J[0, :, k], J[1, :, k] = (xp - xm) / (2 * eps), (yp - ym) / (2 * eps)
    Dp, Dm = D.copy(), D.copy()
    Dp[a] += eps
    Dm[a] -= eps
    xp, yp, _ = project(G, Dp, I, a, b)
    xm, ym, _ = project(G, Dm, I, a, b)
    Jz = np.stack([(xp - xm) / (2 * eps), (yp - ym) / (2 * eps)])
    return Jj, Ji, Jz


def test_sim3_linearization_matches_finite_differences_and_reference_map():
    p = small(edges=[0, 4, 9, 17])
    P, D, I = p["poses"], p["disps"], p["intrinsics"]
    ii, jj = p["ii"], p["jj"]
    lin = opg.linearize_sim3(P, D, I, p["targets"], p["weights"], ii, jj)
    HW = D.shape[1] * D.shape[2]
    G = sim3_of(P)
    for e, (a, b) in enumerate(zip(ii, jj)):
        x0, y0, z0 = project(G, D, I, a, b)
        we = 0.001 * p["weights"][e].reshape(2, HW) * (z0 >= opg.MIN_DEPTH)
        re = p["targets"][e].reshape(2, HW) - np.stack([x0, y0])
        Jj, _, Jz = fd_jacobians(p, a, b)
        tab, qab, sab = se3.rel_sim3(P[a, :3], P[a, 3:7], P[a, 7], P[b, :3], P[b, 3:7], P[b, 7])
        M = adj_matrix(tab, qab, sab)
        Ji = -np.einsum("rk,cpk->cpr", M, Jj)          # the reference's Ji = -adjSim3(Jj)
        Hjj = np.einsum("cp,cpa,cpb->ab", we, Jj, Jj)
        scale = np.abs(Hjj).max()
        np.testing.assert_allclose(lin["Hs"][3, e], Hjj, atol=1e-6 * scale)
        np.testing.assert_allclose(lin["Hs"][1, e], np.einsum("cp,cpa,cpb->ab", we, Ji, Jj), atol=1e-6 * scale)
        np.testing.assert_allclose(lin["Hs"][2, e], lin["Hs"][1, e].T, atol=1e-9 * scale)
        np.testing.assert_allclose(lin["Hs"][0, e], np.einsum("cp,cpa,cpb->ab", we, Ji, Ji),
                                   atol=1e-6 * np.abs(lin["Hs"][0, e]).max())
        vj = np.einsum("cp,cp,cpa->a", we, re, Jj)
        vi = np.einsum("cp,cp,cpa->a", we, re, Ji)
        np.testing.assert_allclose(lin["vs"][1, e], vj, atol=1e-6 * np.abs(vj).max())
        np.testing.assert_allclose(lin["vs"][0, e], vi, atol=1e-6 * np.abs(vi).max())
        C = (we * Jz * Jz).sum(0)
        wz = (we * re * Jz).sum(0)
        np.testing.assert_allclose(lin["Cii"][e], C, atol=1e-6 * np.abs(C).max())
        np.testing.assert_allclose(lin["wi"][e], wz, atol=1e-6 * np.abs(wz).max())
        Eij = np.einsum("cp,cp,cpa->ap", we, Jz, Jj)
        np.testing.assert_allclose(lin["Eij"][e], Eij, atol=1e-6 * np.abs(Eij).max())
        np.testing.assert_allclose(lin["Eii"][e], np.einsum("cp,cp,cpa->ap", we, Jz, Ji),
                                   atol=1e-6 * np.abs(lin["Eii"][e]).max())
        # the scale of frame j does not move its own projections: column 6 of Jj vanishes
        assert np.abs(Jj[..., 6]).max() < 1e-6 * np.abs(Jj).max()


def test_reference_ji_is_not_the_derivative_in_rotation_and_scale():
    # recorded reference behaviour (adjSim3 as written): the translation columns of Ji
    # are the derivative, the rotation and scale columns are not
    p = small(edges=[4])
    a, b = p["ii"][0], p["jj"][0]
    P = p["poses"]
    Jj, Ji_fd, _ = fd_jacobians(p, a, b)
    tab, qab, sab = se3.rel_sim3(P[a, :3], P[a, 3:7], P[a, 7], P[b, :3], P[b, 3:7], P[b, 7])
    Ji_ref = -np.einsum("rk,cpk->cpr", adj_matrix(tab, qab, sab), Jj)
    scale = np.abs(Ji_fd).max()
    assert np.abs(Ji_ref[..., :3] - Ji_fd[..., :3]).max() < 1e-5 * scale
    assert np.abs(Ji_ref[..., 3:] - Ji_fd[..., 3:]).max() > 1e-2 * scale


def test_self_edge_keeps_only_depth_terms():
    p = small(edges=[0, 1])
    p["jj"] = p["ii"].copy()
    lin = opg.linearize_sim3(p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], p["ii"], p["jj"])
    for k in ("Hs", "vs", "Eij", "Eii"):
        assert np.all(lin[k] == 0), k


def test_factor_blocks_match_direct_loop_with_keys_below_t0_dropped():
    p = small(num_factors=12)
    t0, t1 = p["t0"], p["t1"]
    P = t1 - t0
    Np = len(p["iip"])
    Hsp = p["Hsp"].reshape(4, Np, 7, 7)
    vsp = p["vsp"].reshape(2, Np, 7)
    A, b = oba.assemble_pose_system(Hsp, vsp, p["iip"], p["jjp"], t0, P)
    Ad = np.zeros((7 * P, 7 * P))
    bd = np.zeros(7 * P)
    assert (p["iip"] < t0).any()
    for f in range(Np):
        i, j = p["iip"][f] - t0, p["jjp"][f] - t0
        for blk, (r, c) in enumerate(((i, i), (i, j), (j, i), (j, j))):
            if r >= 0 and c >= 0:
                Ad[7 * r:7 * r + 7, 7 * c:7 * c + 7] += Hsp[blk, f]
        if i >= 0:
            bd[7 * i:7 * i + 7] += vsp[0, f]
        if j >= 0:
            bd[7 * j:7 * j + 7] += vsp[1, f]
    np.testing.assert_allclose(A, Ad, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(b, bd, rtol=1e-12, atol=1e-12)


def test_pgba_step_solves_joint_system():
    p = small()
    t0, t1, lm, ep = p["t0"], p["t1"], p["lm"], p["ep"]
    ii, jj = p["ii"], p["jj"]
    P = t1 - t0
    r = opg.pgba(p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], p["eta"], p["Hsp"],
                 p["vsp"], ii, jj, p["iip"], p["jjp"], t0, t1, lm, ep)
    assert r.ok and r.dx.shape == (P, 7)
    kx, kk_exp, ii_exp = oba.keys(ii, t0, t1)
    jj_exp = np.concatenate([np.arange(t0, t1), jj])
    HW = r.Q.shape[1]
    Np = len(p["iip"])
    A, b = oba.assemble_pose_system(r.lin["Hs"], r.lin["vs"], ii, jj, t0, P)
    Ap, bp = oba.assemble_pose_system(p["Hsp"].reshape(4, Np, 7, 7), p["vsp"].reshape(2, Np, 7), p["iip"],
                                      p["jjp"], t0, P)
    A, b = A + Ap, b + bp
    Dg = 1.0 / r.Q
    # the reference damps the diagonal of the reduced matrix A - S
    Ad = A.copy()
    di = np.arange(7 * P)
    Ad[di, di] += ep + lm * r.A[di, di]
    E = r.E
    # joint system without the reference's ix <= 0 skip in the back-substitution
    dz = r.Q * (r.w - oba.accum_fast(np.einsum("ndp,nd->np", E, np.where(
        ((jj_exp - t0 >= 0) & (jj_exp - t0 < P))[:, None], r.dx[np.clip(jj_exp - t0, 0, P - 1)], 0.0)),
        ii_exp, kx))
    Bdz = np.zeros((P, 7))
    BTdx = np.zeros_like(dz)
    for n in range(E.shape[0]):
        pose = jj_exp[n] - t0
        if 0 <= pose < P:
            Bdz[pose] += E[n] @ dz[kk_exp[n]]
            BTdx[kk_exp[n]] += r.dx[pose] @ E[n]
    r1 = Ad @ r.dx.reshape(-1) + Bdz.reshape(-1) - b
    r2 = BTdx + Dg * dz - r.w
    assert np.abs(r1).max() < 1e-8 * max(1.0, np.abs(b).max())
    assert np.abs(r2).max() < 1e-8 * max(1.0, np.abs(r.w).max())
    # disparities move by the returned dz (with the skip), poses are not touched
    np.testing.assert_allclose(r.disps.reshape(len(p["disps"]), HW)[kx],
                               p["disps"].reshape(len(p["disps"]), HW)[kx] + r.dz)


def test_validation_rejects_factor_keys_past_t1():
    p = small()
    p["jjp"] = p["jjp"].copy()
    p["jjp"][0] = p["t1"]
    with pytest.raises(ValueError, match="iip/jjp"):
        opg.pgba(p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], p["eta"], p["Hsp"],
                 p["vsp"], p["ii"], p["jj"], p["iip"], p["jjp"], p["t0"], p["t1"], p["lm"], p["ep"])
