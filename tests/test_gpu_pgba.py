"""pgba on the GPU against the float64 oracle (``oracle.pgba``).

One damped Gauss-Newton step over Sim3 poses with relative-pose factors.  The kernels
linearise in FP32 and solve in FP64, as the reference does (FP32 kernels, an FP64
Cholesky); the bar is 1e-3 of the largest oracle value for dx and dz.
"""

import numpy as np
import pytest
import torch

import droid_backends
from hislam2_b200 import backends, synth
from oracle import pgba as opg

pytestmark = pytest.mark.gpu

TOL = 1e-3


def _problem(cuda, name="frontend_small", seed=0, t0=None, num_factors=None):
    p = synth.make_pgba_problem(name, seed, num_factors=num_factors)
    if t0 is not None:
        p["t0"] = t0
    g = {k: (v.to(cuda) if isinstance(v, torch.Tensor) else v) for k, v in p.items()}
    return p, g


def _run(g):
    disps = g["disps"].clone()
    dx, dz = droid_backends.pgba(g["poses"], disps, g["intrinsics"], g["targets"], g["weights"], g["eta"],
                                 g["Hsp"], g["vsp"], g["ii"], g["jj"], g["iip"], g["jjp"], g["t0"], g["t1"],
                                 g["lm"], g["ep"])
    return dx, dz, disps


def _oracle(p):
    f = lambda t: t.numpy().astype(np.float64) if t.is_floating_point() else t.numpy()  # noqa: E731
    return opg.pgba(f(p["poses"]), f(p["disps"]), f(p["intrinsics"]), f(p["targets"]), f(p["weights"]),
                    f(p["eta"]), f(p["Hsp"]), f(p["vsp"]), f(p["ii"]), f(p["jj"]), f(p["iip"]), f(p["jjp"]),
                    p["t0"], p["t1"], p["lm"], p["ep"])


def _check(p, dx, dz, disps):
    ref = _oracle(p)
    assert ref.ok
    dx, dz, disps = dx.cpu().numpy(), dz.cpu().numpy(), disps.cpu().numpy()
    assert dx.shape == ref.dx.shape and dz.shape == ref.dz.shape
    ex = np.abs(dx - ref.dx).max() / np.abs(ref.dx).max()
    ez = np.abs(dz - ref.dz).max() / np.abs(ref.dz).max()
    ed = np.abs(disps - ref.disps).max() / np.abs(ref.dz).max()
    assert ex < TOL and ez < TOL and ed < TOL, "dx %.2e dz %.2e disps %.2e" % (ex, ez, ed)


@pytest.mark.parametrize("t0", [2, 1], ids=["even_order", "odd_order_padded"])
def test_pgba_matches_oracle_small(cuda, t0):
    p, g = _problem(cuda, t0=t0)
    dx, dz, disps = _run(g)
    _check(p, dx, dz, disps)
    # poses are not moved by pgba
    assert torch.equal(g["poses"].cpu(), p["poses"])


def test_pgba_matches_oracle_frontend_window(cuda):
    p, g = _problem(cuda, name="frontend", num_factors=50)
    dx, dz, disps = _run(g)
    _check(p, dx, dz, disps)


@pytest.mark.parametrize("t0", [0, 8], ids=["whole_buffer", "empty_window"])
def test_pgba_window_edges(cuda, t0):
    # t0 = 0: the reference's back-substitution skips pose 0 (ix <= 0); t0 = t1: no pose
    # is optimised, dx is empty and dz = Q w
    p, g = _problem(cuda, t0=t0)
    dx, dz, disps = _run(g)
    assert dx.shape == (p["t1"] - t0, 7)
    if t0 == p["t1"]:
        ref = _oracle(p)
        np.testing.assert_allclose(dz.cpu().numpy(), ref.dz, rtol=1e-4, atol=1e-4 * np.abs(ref.dz).max())
    else:
        _check(p, dx, dz, disps)


def test_pgba_without_factors(cuda):
    p, g = _problem(cuda, num_factors=0)
    dx, dz, disps = _run(g)
    _check(p, dx, dz, disps)


def test_pgba_is_deterministic_across_calls(cuda):
    p, g = _problem(cuda, seed=3)
    a = _run(g)
    b = _run(g)
    for x, y in zip(a, b):
        assert np.abs((x - y).cpu().numpy()).max() <= 1e-6 * max(1.0, np.abs(x.cpu().numpy()).max())


def test_pgba_rejects_factor_key_past_t1_and_leaves_disps(cuda):
    p, g = _problem(cuda)
    g["jjp"] = g["jjp"].clone()
    g["jjp"][0] = g["t1"]
    disps = g["disps"].clone()
    with pytest.raises(RuntimeError, match="out of range"):
        droid_backends.pgba(g["poses"], disps, g["intrinsics"], g["targets"], g["weights"], g["eta"], g["Hsp"],
                            g["vsp"], g["ii"], g["jj"], g["iip"], g["jjp"], g["t0"], g["t1"], g["lm"], g["ep"])
    assert torch.equal(disps, g["disps"])


def test_pgba_is_the_backends_operator():
    assert droid_backends.pgba is backends.pgba
