"""The pose-graph oracle (``oracle/pgo.py``) pinned by Sim3 identities and by the reference's
own factor procedure (``tests/golden/pgo_*.npz``), and the FP64 Sim3 code that
``csrc/pgo.cu`` runs on the device (``csrc/sim3.cuh``, compiled here for the host by
``tests/sim3_host_harness.cpp``) checked against both on the CPU."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import pgo

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "hi-slam2_b200", "hislam2_b200", "csrc")


def rand_sim3(g, n, rot=0.5, trans=1.0, scale=0.3):
    xi = np.concatenate([trans * g.standard_normal((n, 3)), rot * g.standard_normal((n, 3)),
                         scale * g.standard_normal((n, 1))], 1)
    return np.stack([pgo.from_matrix(pgo.exp(x)) for x in xi])


def quat_align(q, ref):
    return np.where((np.sum(q * ref, -1) < 0)[..., None], -q, q)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("sim3") / "harness")
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", CSRC, os.path.join(HERE, "sim3_host_harness.cpp"), "-o", exe],
                   check=True)

    def run(mode, payload, nout, dtypes):
        d = tmp_path_factory.mktemp("io")
        fin, fout = str(d / "in.bin"), str(d / "out.bin")
        with open(fin, "wb") as f:
            for a in payload:
                f.write(np.ascontiguousarray(a).tobytes())
        subprocess.run([exe, mode, fin, fout], check=True)
        raw = open(fout, "rb").read()
        out, off = [], 0
        for n, dt in zip(nout, dtypes):
            a = np.frombuffer(raw, dtype=dt, count=n, offset=off)
            off += a.nbytes
            out.append(a)
        assert off == len(raw)
        return out
    return run


# ------------------------------------------------------------------ oracle identities
def test_oracle_exp_log_inverse():
    g = np.random.default_rng(0)
    for _ in range(20):
        xi = np.concatenate([g.standard_normal(3), 0.8 * g.standard_normal(3), 0.5 * g.standard_normal(1)])
        np.testing.assert_allclose(pgo.log(pgo.exp(xi)), xi, rtol=0, atol=1e-11)


def test_oracle_adjoint_definition():
    g = np.random.default_rng(1)
    G = pgo.to_matrix(rand_sim3(g, 1)[0])
    xi = 0.1 * g.standard_normal(7)
    np.testing.assert_allclose(pgo.log(G @ pgo.exp(xi) @ np.linalg.inv(G)), pgo.adjoint(G) @ xi, atol=1e-11)


def test_oracle_jacobians_at_zero_residual():
    """r = log(Gij Gi Gj^-1) = 0 -> Ji = Ad(Gij), Jj = -I (pgo_buffer.py:43-50)."""
    g = np.random.default_rng(2)
    Gi = rand_sim3(g, 1)[0]
    rel = rand_sim3(g, 1, scale=0.0)[0][:7]
    Gj = pgo.from_matrix(pgo.to_matrix(rel) @ pgo.to_matrix(Gi))
    r, Ji, Jj = pgo.factor_terms(Gi, Gj, rel)
    np.testing.assert_allclose(r, 0, atol=1e-12)
    np.testing.assert_allclose(Ji, pgo.adjoint(pgo.to_matrix(rel)), atol=1e-9)
    np.testing.assert_allclose(Jj, -np.eye(7), atol=1e-9)


def test_oracle_retract_is_left_multiplication():
    g = np.random.default_rng(3)
    P = rand_sim3(g, 5)
    dx = 0.05 * g.standard_normal((3, 7))
    out = pgo.retract(P, dx, 1, 4)
    np.testing.assert_array_equal(out[[0, 4]], P[[0, 4]])
    for k in range(3):
        np.testing.assert_allclose(pgo.to_matrix(out[1 + k]), pgo.exp(dx[k]) @ pgo.to_matrix(P[1 + k]), atol=1e-12)


# ------------------------------------------------------------------ device code on the host
def test_device_exp_log_match_oracle(harness):
    g = np.random.default_rng(4)
    unit = lambda v: v / np.linalg.norm(v)
    # rotation angles (below pi, where log inverts exp) and log-scales on both sides of the
    # series / closed-form switch at |(phi, sigma)| = 0.5, with tiny and zero angles
    cases = [np.concatenate([g.standard_normal(3), th * unit(g.standard_normal(3)), [sg]])
             for th, sg in ((0.01, 0.0), (0.2, 0.1), (0.3, -0.3), (1.5, 0.2), (2.5, -0.8), (0.0, 0.9), (1e-9, 0.7),
                            (0.35, 0.35), (0.0, 0.0), (1e-7, 1e-9), (0.4999, 0.0), (0.5001, 0.0))]
    xi = np.stack(cases)
    gmat, back = harness("explog", [np.array([len(xi)], np.int64), xi], [len(xi) * 8, len(xi) * 7],
                         [np.float64, np.float64])
    gmat, back = gmat.reshape(-1, 8), back.reshape(-1, 7)
    for k in range(len(xi)):
        np.testing.assert_allclose(pgo.to_matrix(gmat[k]), pgo.exp(xi[k]), atol=1e-12, err_msg=str(k))
    np.testing.assert_allclose(back, xi, atol=1e-12)


def factor_problem(seed, Np=40, N=12, noise=0.05):
    g = np.random.default_rng(seed)
    P = rand_sim3(g, N).astype(np.float32)
    ii = g.integers(0, N, Np)
    jj = g.integers(0, N, Np)
    rel = np.zeros((Np, 7), np.float32)
    for n in range(Np):
        M = pgo.to_matrix(P[jj[n]]) @ np.linalg.inv(pgo.to_matrix(P[ii[n]]))
        M[:3, :3] /= np.cbrt(np.linalg.det(M[:3, :3]))            # the SE3 part of the relative pose
        meas = pgo.from_matrix(pgo.exp(noise * g.standard_normal(7) * [1, 1, 1, 1, 1, 1, 0]) @ M)
        rel[n] = meas[:7]
    infos = np.zeros((Np, 7, 7), np.float32)
    d = 10.0 ** g.uniform(1, 4, (Np, 6))
    infos[:, np.arange(6), np.arange(6)] = d
    infos[:, 6, 6] = d.min(1)
    return P, ii.astype(np.int64), jj.astype(np.int64), rel, infos


def test_device_factor_terms_match_oracle(harness):
    P, ii, jj, rel, infos = factor_problem(5)
    N, Np, pw = len(P), len(ii), 1e-3
    cols, Hsp, vsp, chi = harness(
        "factors", [np.array([N, Np], np.int64), P, ii, jj, rel, infos, np.array([pw])],
        [Np * 15 * 7, 4 * Np * 49, 2 * Np * 7, 2 * Np], [np.float64, np.float32, np.float32, np.float32])
    cols = cols.reshape(Np, 15, 7)
    H, v, chi2, chi2s, r, Ji, Jj = pgo.relative_constraints(ii, jj, P, rel, infos, pw)
    # the device code uses the float quaternions as given (|q| = 1 within ~6e-8), as lietorch
    # does; the oracle normalises them
    np.testing.assert_allclose(cols[:, 14], r, rtol=0, atol=1e-6)
    # the device's central differences (step 1e-8) against the oracle's derivative
    np.testing.assert_allclose(np.transpose(cols[:, :7], (0, 2, 1)), Ji, rtol=0, atol=2e-7 * np.abs(Ji).max())
    np.testing.assert_allclose(np.transpose(cols[:, 7:14], (0, 2, 1)), Jj, rtol=0, atol=2e-7 * np.abs(Jj).max())
    Hd = Hsp.reshape(4, Np, 7, 7)
    np.testing.assert_allclose(Hd, H, rtol=0, atol=2e-6 * np.abs(H).max())
    np.testing.assert_allclose(vsp.reshape(2, Np, 7), v, rtol=0, atol=2e-6 * np.abs(v).max())
    c = chi.reshape(Np, 2).astype(np.float64).sum(0)
    np.testing.assert_allclose(c, [chi2, chi2s], rtol=1e-5)
    assert np.abs(r).max() > 1e-2                      # the factors are not at their optimum


def test_device_retraction_matches_oracle(harness):
    g = np.random.default_rng(6)
    P = rand_sim3(g, 9).astype(np.float32)
    t0, t1 = 2, 8
    dx = (0.05 * g.standard_normal((t1 - t0, 7))).astype(np.float32)
    out, = harness("retr", [np.array([9, t0, t1], np.int64), P, dx], [9 * 8], [np.float32])
    out = out.reshape(9, 8)
    ref = pgo.retract(P.astype(np.float64), dx.astype(np.float64), t0, t1)
    np.testing.assert_array_equal(out[:t0], P[:t0])
    np.testing.assert_array_equal(out[t1:], P[t1:])
    np.testing.assert_allclose(out[:, :3], ref[:, :3], atol=2e-6)
    np.testing.assert_allclose(out[:, 7], ref[:, 7], rtol=2e-6)
    np.testing.assert_allclose(quat_align(out[:, 3:7], ref[:, 3:7]), ref[:, 3:7], atol=2e-6)


# ------------------------------------------------------------------ the reference's own procedure
GOLDEN = sorted(__import__("glob").glob(os.path.join(HERE, "golden", "pgo_*.npz")))


def _golden(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def test_golden_fixtures_present():
    assert {os.path.basename(p) for p in GOLDEN} >= {"pgo_frontend_small.npz", "pgo_frontend40.npz"}


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_procedure(path):
    """oracle vs pgo_buffer.py's own num_jacobi / global_relative_posesim3_constraints
    (tests/golden/make_golden_pgo.py)."""
    g = _golden(path)
    H, v, c2, c2s, _, _, _ = pgo.relative_constraints(g["iip"], g["jjp"], g["poses"], g["rel"], g["infos"],
                                                      float(g["pw"]))
    Hf, vf = g["Hsp"][:, 0], g["vsp"][:, 0]
    assert np.abs(H - Hf).max() < 2e-6 * np.abs(Hf).max()
    assert np.abs(v - vf).max() < 2e-6 * np.abs(vf).max()
    np.testing.assert_allclose([c2, c2s], [g["chi2"], g["chi2_scaled"]], rtol=1e-6)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_device_code_matches_reference_procedure(harness, path):
    g = _golden(path)
    N, Np = len(g["poses"]), len(g["iip"])
    _, Hsp, vsp, chi = harness(
        "factors", [np.array([N, Np], np.int64), g["poses"].astype(np.float32), g["iip"].astype(np.int64),
                    g["jjp"].astype(np.int64), g["rel"].astype(np.float32), g["infos"].astype(np.float32),
                    np.array([float(g["pw"])])],
        [Np * 15 * 7, 4 * Np * 49, 2 * Np * 7, 2 * Np], [np.float64, np.float32, np.float32, np.float32])
    Hf, vf = g["Hsp"][:, 0], g["vsp"][:, 0]
    assert np.abs(Hsp.reshape(4, Np, 7, 7) - Hf).max() < 2e-6 * np.abs(Hf).max()
    assert np.abs(vsp.reshape(2, Np, 7) - vf).max() < 2e-6 * np.abs(vf).max()
    np.testing.assert_allclose(chi.reshape(Np, 2).astype(np.float64).sum(0), [g["chi2"], g["chi2_scaled"]],
                               rtol=1e-6)
