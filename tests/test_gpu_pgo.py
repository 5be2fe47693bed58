"""hs2_pgo_constraints / hs2_sim3_retr (``hislam2_b200.pgo``) against the float64 oracle
(``oracle/pgo.py``), and the pgba loop of ``DepthVideo.cuda_pgba`` on the GPU against the
oracle chain."""

import os

import numpy as np
import pytest
import torch

import droid_backends
from hislam2_b200 import pgo, synth
from oracle import pgba as opg
from oracle import pgo as opgo

pytestmark = pytest.mark.gpu


def _factors(cuda, name="frontend_small", seed=0, num_factors=None, noise=0.02):
    p = synth.make_pgba_problem(name, seed, num_factors=num_factors)
    rel, infos = synth.make_pgo_factors(p["poses"], p["iip"], p["jjp"], seed=seed, noise=noise)
    p.update(rel=rel, infos=infos)
    g = {k: (v.to(cuda) if isinstance(v, torch.Tensor) else v) for k, v in p.items()}
    return p, g


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("name,nf", [("frontend_small", None), ("frontend", 300)])
def test_constraints_match_oracle(cuda, name, nf):
    p, g = _factors(cuda, name, num_factors=nf)
    Hsp, vsp, chi2, chi2s = pgo.global_relative_posesim3_constraints(g["iip"], g["jjp"], g["poses"][None],
                                                                     g["rel"][None], g["infos"], pw=1e-3)
    torch.cuda.synchronize()
    Np = p["iip"].numel()
    assert Hsp.shape == (4, 1, Np, 7, 7) and vsp.shape == (2, 1, Np, 7)
    H, v, c2, c2s, r, Ji, Jj = opgo.relative_constraints(p["iip"].numpy(), p["jjp"].numpy(), p["poses"].numpy(),
                                                         p["rel"].numpy(), p["infos"].numpy(), 1e-3)
    assert _rel(Hsp[:, 0].cpu().numpy(), H) < 1e-5
    assert _rel(vsp[:, 0].cpu().numpy(), v) < 1e-5
    np.testing.assert_allclose([float(chi2), float(chi2s)], [c2, c2s], rtol=1e-5)
    assert np.abs(r).max() > 1e-2


def test_constraints_at_zero_residual(cuda):
    """Factors whose measurement closes the loop exactly (equal scales): Ji = Ad(Gij), Jj = -I,
    r = 0, so Hsp = pw [Ad' W Ad, -Ad' W, -W Ad, W] and vsp = 0."""
    g = np.random.default_rng(7)
    xi = np.concatenate([g.standard_normal((6, 3)), 0.5 * g.standard_normal((6, 3)), np.zeros((6, 1))], 1)
    P = np.stack([opgo.from_matrix(opgo.exp(x)) for x in xi])
    P[:, 7] = 1.3
    ii, jj = np.array([0, 1, 2, 3, 4]), np.array([1, 2, 3, 4, 5])
    rel = np.stack([opgo.from_matrix(opgo.to_matrix(P[j]) @ np.linalg.inv(opgo.to_matrix(P[i])))[:7]
                    for i, j in zip(ii, jj)])
    infos = np.tile(np.diag([100.0, 200, 300, 400, 500, 600, 100]), (5, 1, 1))
    f = lambda a, dt=torch.float32: torch.tensor(a, dtype=dt, device=cuda).contiguous()  # noqa: E731
    Hsp, vsp, chi2, _ = pgo.global_relative_posesim3_constraints(f(ii, torch.int64), f(jj, torch.int64), f(P),
                                                                 f(rel), f(infos), pw=1.0)
    assert float(chi2) < 1e-10
    assert float(vsp.abs().max()) < 1e-3
    for n in range(5):
        Ad = opgo.adjoint(opgo.to_matrix(rel[n]))
        W = infos[n]
        ref = np.stack([Ad.T @ W @ Ad, -Ad.T @ W, -W @ Ad, W])
        assert _rel(Hsp[:, 0, n].cpu().numpy(), ref) < 1e-5


def test_constraints_bad_index_raises(cuda):
    p, g = _factors(cuda)
    jjp = g["jjp"].clone()
    jjp[3] = g["poses"].shape[0]
    with pytest.raises(RuntimeError, match="outside"):
        pgo.global_relative_posesim3_constraints(g["iip"], jjp, g["poses"], g["rel"], g["infos"], pw=1e-3)


def test_sim3_retraction_matches_oracle(cuda):
    p, g = _factors(cuda)
    t0, t1 = p["t0"], p["t1"]
    gen = torch.Generator().manual_seed(11)
    dx = (0.05 * torch.randn(t1 - t0, 7, generator=gen)).to(cuda)
    poses = g["poses"].clone()
    pgo.sim3_retr_(poses, dx, t0, t1)
    out = poses.cpu().numpy()
    ref = opgo.retract(p["poses"].numpy(), dx.cpu().numpy(), t0, t1)
    np.testing.assert_array_equal(out[:t0], p["poses"].numpy()[:t0])
    np.testing.assert_array_equal(out[t1:], p["poses"].numpy()[t1:])
    sign = np.where((out[:, 3:7] * ref[:, 3:7]).sum(1) < 0, -1.0, 1.0)[:, None]
    np.testing.assert_allclose(out[:, :3], ref[:, :3], atol=3e-6)
    np.testing.assert_allclose(sign * out[:, 3:7], ref[:, 3:7], atol=3e-6)
    np.testing.assert_allclose(out[:, 7], ref[:, 7], rtol=3e-6)


def test_cuda_pgba_loop_matches_oracle_chain(cuda):
    """Two iterations of DepthVideo.cuda_pgba's loop (depth_video.py:258-267): constraints,
    pgba, Sim3 retraction -- all on the GPU -- against the same chain in the oracle."""
    p, g = _factors(cuda)
    poses, disps = g["poses"].clone(), g["disps"].clone()
    P, D = p["poses"].numpy().astype(np.float64), p["disps"].numpy().astype(np.float64)
    f64 = lambda t: t.numpy().astype(np.float64) if t.is_floating_point() else t.numpy()  # noqa: E731
    for _ in range(2):
        Hsp, vsp, _, _ = pgo.global_relative_posesim3_constraints(g["iip"], g["jjp"], poses, g["rel"], g["infos"],
                                                                  pw=1e-3)
        dx, dz = droid_backends.pgba(poses, disps, g["intrinsics"], g["targets"], g["weights"], g["eta"], Hsp, vsp,
                                     g["ii"], g["jj"], g["iip"], g["jjp"], p["t0"], p["t1"], p["lm"], p["ep"])
        pgo.sim3_retr_(poses, dx, p["t0"], p["t1"])
        H, v, _, _, _, _, _ = opgo.relative_constraints(p["iip"].numpy(), p["jjp"].numpy(), P, f64(p["rel"]),
                                                        f64(p["infos"]), 1e-3)
        ref = opg.pgba(P, D, f64(p["intrinsics"]), f64(p["targets"]), f64(p["weights"]), f64(p["eta"]), H, v,
                       p["ii"].numpy(), p["jj"].numpy(), p["iip"].numpy(), p["jjp"].numpy(), p["t0"], p["t1"],
                       p["lm"], p["ep"])
        assert ref.ok
        D = ref.disps
        P = opgo.retract(P, ref.dx, p["t0"], p["t1"])
        assert _rel(dx.cpu().numpy(), ref.dx) < 1e-3
    out = poses.cpu().numpy()
    np.testing.assert_allclose(out[:, :3], P[:, :3], atol=1e-4 * np.abs(P[:, :3]).max())
    np.testing.assert_allclose(out[:, 7], P[:, 7], rtol=1e-4)
    assert _rel(disps.cpu().numpy(), D) < 1e-3


@pytest.mark.parametrize("name", ["pgo_frontend_small", "pgo_frontend40"])
def test_constraints_match_reference_procedure(cuda, name):
    """Against pgo_buffer.py's own num_jacobi / global_relative_posesim3_constraints
    (fixtures made by tests/golden/make_golden_pgo.py)."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    f = lambda k, dt=torch.float32: torch.tensor(z[k], dtype=dt, device=cuda).contiguous()  # noqa: E731
    Hsp, vsp, chi2, chi2s = pgo.global_relative_posesim3_constraints(
        f("iip", torch.int64), f("jjp", torch.int64), f("poses")[None], f("rel")[None], f("infos"), pw=float(z["pw"]))
    assert _rel(Hsp.cpu().numpy(), z["Hsp"]) < 1e-5
    assert _rel(vsp.cpu().numpy(), z["vsp"]) < 1e-5
    np.testing.assert_allclose([float(chi2), float(chi2s)], [z["chi2"], z["chi2_scaled"]], rtol=1e-5)
