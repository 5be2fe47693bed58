"""hs2_jdsa (``hislam2_b200.mono.JDSA``) against the reference's own JDSA (golden fixtures made
by ``tests/golden/make_golden_jdsa.py``) and the float64 oracle (``oracle/jdsa.py``)."""

import glob
import os

import numpy as np
import pytest
import torch

from hislam2_b200 import mono, synth
from oracle import jdsa as ojdsa

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "jdsa_*.npz")))


def rel(a, b):
    a = np.asarray(a, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def to_dev(p, cuda):
    return {k: (torch.as_tensor(v).to(cuda).contiguous() if isinstance(v, (np.ndarray, torch.Tensor)) and
                np.ndim(v) > 0 else v) for k, v in p.items()}


def run(p, cuda, **kw):
    d = to_dev(p, cuda)
    dscales = d["dscales"].clone()
    out, sc, dzcov = mono.JDSA(d["targets"], d["weights"], d["eta"], d["poses"], d["disps"][None],
                               d["intrinsics"][None, None], d["disps_prior"], dscales, d["ii"], d["jj"],
                               float(p["alpha"]), **kw)
    torch.cuda.synchronize()
    assert sc is dscales
    return out[0].cpu().numpy(), sc.cpu().numpy(), None if dzcov is None else dzcov.cpu().numpy()


@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_matches_reference_jdsa(cuda, path):
    z = np.load(path)
    g = {k: z[k] for k in z.files}
    if bool(g["raised"]):
        d = to_dev(g, cuda)
        dscales = d["dscales"].clone()
        with pytest.raises(torch.linalg.LinAlgError):
            mono.JDSA(d["targets"], d["weights"], d["eta"], d["poses"], d["disps"][None], d["intrinsics"],
                      d["disps_prior"], dscales, d["ii"], d["jj"], float(g["alpha"]))
        np.testing.assert_array_equal(dscales.cpu().numpy(), g["dscales"])     # left unchanged
        return
    out, sc, dzcov = run(g, cuda)
    # the reference ran in float32 (dense [M*D]^2 Cholesky, float32 Schur complement)
    assert rel(out, g["out_disps"]) < 1e-5
    assert rel(sc - g["dscales"], g["out_dscales"] - g["dscales"]) < 1e-3
    assert rel(dzcov, g["out_dzcov"]) < 1e-4
    r = ojdsa.jdsa(g["targets"], g["weights"], g["eta"], g["poses"], g["disps"], g["intrinsics"],
                   g["disps_prior"], g["dscales"], g["ii"], g["jj"], float(g["alpha"]))
    assert rel(out, r["disps"]) < 1e-5
    assert rel(sc - g["dscales"], r["dscales"] - g["dscales"]) < 1e-3
    assert rel(dzcov, r["dzcov"]) < 1e-4


@pytest.mark.parametrize("hs,ws,alpha", [(2, 2, 0.01), (4, 4, 0.001)])
def test_frontend_window_matches_oracle(cuda, hs, ws, alpha):
    """HI-SLAM2's frontend size: 25 keyframes at 43x77, 258 edges, 2x2 (its configuration)
    and 4x4 scale grids (16 unknowns per frame, the kernel's limit)."""
    p = synth.make_jdsa_problem("frontend", hs=hs, ws=ws, alpha=alpha)
    out, sc, dzcov = run(p, cuda)
    a = {k: (v.numpy() if isinstance(v, torch.Tensor) else v) for k, v in p.items()}
    r = ojdsa.jdsa(a["targets"], a["weights"], a["eta"], a["poses"], a["disps"], a["intrinsics"], a["disps_prior"],
                   a["dscales"], a["ii"], a["jj"], alpha)
    assert rel(out, r["disps"]) < 1e-5
    assert rel(sc - a["dscales"], r["dscales"] - a["dscales"]) < 1e-3
    assert rel(dzcov, r["dzcov"]) < 1e-4
    # the step moves the scales: the comparison is not between two unchanged buffers
    assert np.abs(r["dso"]).max() > 1e-3


def test_without_dzcov_gives_the_same_step(cuda):
    p = synth.make_jdsa_problem("tiny6")
    out1, sc1, cov = run(p, cuda)
    out2, sc2, none = run(p, cuda, with_dzcov=False)
    assert none is None and cov is not None
    np.testing.assert_allclose(out2, out1, rtol=0, atol=1e-6)
    np.testing.assert_allclose(sc2, sc1, rtol=0, atol=1e-6)


def test_bad_source_frame_raises_and_keeps_scales(cuda):
    p = synth.make_jdsa_problem("tiny6")
    d = to_dev(p, cuda)
    prior = d["disps_prior"][:4].contiguous()          # frames 4 and 5 have no prior row
    dscales = d["dscales"].clone()
    with pytest.raises(RuntimeError, match="outside"):
        mono.JDSA(d["targets"], d["weights"], d["eta"], d["poses"], d["disps"][None], d["intrinsics"], prior,
                  dscales, d["ii"], d["jj"], p["alpha"])
    np.testing.assert_array_equal(dscales.cpu().numpy(), p["dscales"].numpy())
