"""The differentiable float64 LM step (``oracle/lm_step.py``) that the adjoint tests
differentiate: its forward equals one iteration of the BA oracle (``oracle/ba.py``, pinned
to the reference's compiled ``ba``), and its closed-form adjoint equals autograd through it."""

import numpy as np
import pytest
import torch

from hislam2_b200 import synth
from oracle import ba as oba
from oracle import lm_step


@pytest.mark.parametrize("name,t0", [("tiny6", None), ("tiny6", 0), ("tiny7", None)])
def test_forward_equals_one_ba_iteration(name, t0):
    p = synth.make_ba_problem(name, seed=0)
    t0 = p["t0"] if t0 is None else t0
    M = len(np.unique(np.concatenate([np.arange(t0, p["t1"]), p["ii"].numpy()])))
    eta = p["eta"][:M].double()
    f = lambda k: p[k].numpy().astype(np.float64)  # noqa: E731
    dx, dz = lm_step.lm_step(f("poses"), f("disps"), f("intrinsics"), p["targets"].double(), p["weights"].double(),
                             eta, p["ii"].numpy(), p["jj"].numpy(), t0, p["t1"], p["lm"], p["ep"])
    r = oba.ba(f("poses"), f("disps"), f("intrinsics"), f("targets"), f("weights"), eta.numpy(), p["ii"].numpy(),
               p["jj"].numpy(), t0, p["t1"], 1, p["lm"], p["ep"])
    np.testing.assert_allclose(dx.numpy(), r.dx.reshape(dx.shape), rtol=0, atol=1e-10 * np.abs(r.dx).max())
    np.testing.assert_allclose(dz.numpy(), r.dz.reshape(dz.shape), rtol=0, atol=1e-10 * np.abs(r.dz).max())


def test_closed_form_adjoint_equals_autograd():
    p = synth.make_ba_problem("tiny6", seed=0)
    t0, t1 = p["t0"], p["t1"]
    M = len(np.unique(np.concatenate([np.arange(t0, t1), p["ii"].numpy()])))
    f = lambda k: p[k].numpy().astype(np.float64)  # noqa: E731
    tg = p["targets"].double().requires_grad_(True)
    wt = p["weights"].double().requires_grad_(True)
    et = p["eta"][:M].double().requires_grad_(True)
    dx, dz = lm_step.lm_step(f("poses"), f("disps"), f("intrinsics"), tg, wt, et, p["ii"].numpy(), p["jj"].numpy(),
                             t0, t1, p["lm"], p["ep"])
    g = torch.Generator().manual_seed(3)
    gdx = torch.randn(dx.shape, generator=g, dtype=torch.float64)
    gdz = torch.randn(dz.shape, generator=g, dtype=torch.float64)
    at, aw, ae = torch.autograd.grad((dx * gdx).sum() + (dz * gdz).sum(), [tg, wt, et])
    ct, cw, ce = lm_step.lm_step_adjoint(f("poses"), f("disps"), f("intrinsics"), f("targets"), f("weights"),
                                         p["eta"][:M].double().numpy(), p["ii"].numpy(), p["jj"].numpy(), t0, t1,
                                         p["lm"], p["ep"], gdx.numpy(), gdz.numpy())
    for a, c in ((at, ct), (aw, cw), (ae, ce)):
        np.testing.assert_allclose(np.asarray(c), a.numpy(), rtol=0, atol=1e-8 * np.abs(a.numpy()).max())
