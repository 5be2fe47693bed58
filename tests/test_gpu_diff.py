"""Differentiation form: the hand-written adjoints against float64 references.

* BAStep (one LM step of ba, adjoint kernels hs2_ba_adjoint) w.r.t. targets, weights
  and eta: against torch.autograd through the float64 PyTorch restatement of the
  same step (oracle/lm_step.py), and against float64 central finite differences
  (h = 1e-6) of the numpy oracle (oracle.ba) along random directions.
* CorrLookup (the CorrBlock lookup differentiated w.r.t. both feature maps, no
  stored pyramid) against float64 central finite differences of the oracle's
  pyramid + lookup.
Tolerance: 1e-3 relative (the kernels compute in FP32 against FP64 references;
the bar the differentiation form states).
"""

import numpy as np
import pytest
import torch

import oracle
from oracle import lm_step
from hislam2_b200 import corr as hcorr
from hislam2_b200 import diff, synth

pytestmark = pytest.mark.gpu

TOL = 1e-3


def rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.detach().double().cpu().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def problem(name, t0=None, eta_rows=None, seed=0):
    p = synth.make_ba_problem(name, seed=seed)
    t0 = p["t0"] if t0 is None else t0
    M = len(np.unique(np.concatenate([np.arange(t0, p["t1"]), p["ii"].numpy()])))
    g = torch.Generator().manual_seed(seed + 5)
    eta = p["eta"][: (M if eta_rows is None else eta_rows)] * (1 + torch.rand(
        (M if eta_rows is None else eta_rows,) + p["eta"].shape[1:], generator=g))
    p = dict(p, t0=t0, eta=eta.contiguous())
    return p, M


def gpu_grads(p, cuda, gdx, gdz):
    q = {k: (v.to(cuda) if torch.is_tensor(v) else v) for k, v in p.items()}
    tg = q["targets"].clone().requires_grad_(True)
    wt = q["weights"].clone().requires_grad_(True)
    et = q["eta"].clone().requires_grad_(True)
    dx, dz = diff.ba_step(tg, wt, et, q["poses"], q["disps"], q["intrinsics"], q["ii"], q["jj"], q["t0"], q["t1"],
                          q["lm"], q["ep"])
    L = (dx * gdx.to(cuda).float()).sum() + (dz * gdz.to(cuda).float()).sum()
    gt, gw, ge = torch.autograd.grad(L, [tg, wt, et])
    return dx, dz, gt, gw, ge


def autograd_reference(p, gdx, gdz):
    f = lambda k: p[k].double().numpy()  # noqa: E731
    tg = p["targets"].double().requires_grad_(True)
    wt = p["weights"].double().requires_grad_(True)
    et = p["eta"].double().requires_grad_(True)
    dx, dz = lm_step.lm_step(f("poses"), f("disps"), f("intrinsics"), tg, wt, et, p["ii"].numpy(), p["jj"].numpy(),
                             p["t0"], p["t1"], p["lm"], p["ep"])
    L = (dx * gdx).sum() + (dz * gdz).sum()
    return (dx.detach(), dz.detach()) + torch.autograd.grad(L, [tg, wt, et])


CASES = {
    "tiny6": dict(name="tiny6"),
    "tiny6_t0_0": dict(name="tiny6", t0=0),
    "tiny6_eta_one_row": dict(name="tiny6", eta_rows=1),
    "tiny7_window": dict(name="tiny7"),
    "frontend_small": dict(name="frontend_small"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_ba_adjoint_matches_autograd(cuda, case):
    p, M = problem(**CASES[case])
    P = p["t1"] - p["t0"]
    HW = p["disps"].shape[1] * p["disps"].shape[2]
    g = torch.Generator().manual_seed(11)
    gdx = torch.randn(P, 6, generator=g, dtype=torch.float64)
    gdz = torch.randn(M, HW, generator=g, dtype=torch.float64)
    dx, dz, gt, gw, ge = gpu_grads(p, cuda, gdx, gdz)
    rdx, rdz, rt, rw, re = autograd_reference(p, gdx, gdz)
    assert rel(dx, rdx) < 1e-4 and rel(dz, rdz) < 1e-4
    errs = (rel(gt, rt), rel(gw, rw), rel(ge, re))
    print("%s: grad rel err targets %.2e weights %.2e eta %.2e" % ((case,) + errs))
    assert max(errs) < TOL, errs


def test_ba_adjoint_matches_finite_differences(cuda):
    p, M = problem("tiny6", seed=3)
    P = p["t1"] - p["t0"]
    HW = p["disps"].shape[1] * p["disps"].shape[2]
    g = torch.Generator().manual_seed(12)
    gdx = torch.randn(P, 6, generator=g, dtype=torch.float64)
    gdz = torch.randn(M, HW, generator=g, dtype=torch.float64)
    _, _, gt, gw, ge = gpu_grads(p, cuda, gdx, gdz)
    f = lambda k: p[k].double().numpy()  # noqa: E731

    def loss(targets, weights, eta):
        r = oracle.ba.ba(f("poses"), f("disps"), f("intrinsics"), targets, weights, eta, p["ii"].numpy(),
                         p["jj"].numpy(), p["t0"], p["t1"], 1, p["lm"], p["ep"])
        return float((r.dx * gdx.numpy()).sum() + (r.dz * gdz.numpy()).sum())

    h = 1e-6
    base = dict(targets=f("targets"), weights=f("weights"), eta=f("eta"))
    for name, grad in (("targets", gt), ("weights", gw), ("eta", ge)):
        d = torch.randn(base[name].shape, generator=g, dtype=torch.float64).numpy()
        plus = dict(base, **{name: base[name] + h * d})
        minus = dict(base, **{name: base[name] - h * d})
        fd = (loss(**plus) - loss(**minus)) / (2 * h)
        an = float((grad.double().cpu().numpy() * d).sum())
        print("%s: directional derivative adjoint %.6e finite difference %.6e" % (name, an, fd))
        assert abs(an - fd) <= TOL * max(abs(fd), 1e-12), (name, an, fd)


def test_ba_adjoint_two_clips_of_seven_frames(cuda):
    """The differentiation config: 2 clips x 7 frames at 48x64, all 42 edges i != j."""
    for seed in (0, 1):
        p, M = problem("clips2x7", seed=seed)
        P = p["t1"] - p["t0"]
        HW = 48 * 64
        g = torch.Generator().manual_seed(20 + seed)
        gdx = torch.randn(P, 6, generator=g, dtype=torch.float64)
        gdz = torch.randn(M, HW, generator=g, dtype=torch.float64)
        _, _, gt, gw, ge = gpu_grads(p, cuda, gdx, gdz)
        _, _, rt, rw, re = autograd_reference(p, gdx, gdz)
        errs = (rel(gt, rt), rel(gw, rw), rel(ge, re))
        print("clips2x7 seed %d: grad rel err targets %.2e weights %.2e eta %.2e" % ((seed,) + errs))
        assert max(errs) < TOL, errs


def test_corr_lookup_gradients_match_finite_differences(cuda):
    K, C, H, W, r, L = 3, 128, 48, 64, 4, 4
    g = torch.Generator().manual_seed(4)
    f = (torch.randn(K, C, H, W, generator=g) / np.sqrt(C)).half()
    ii, jj = torch.tensor([0, 1]), torch.tensor([1, 2])
    f1 = f[ii][None].to(cuda).requires_grad_(True)
    f2 = f[jj][None].to(cuda).requires_grad_(True)
    p = synth.make_ba_problem("frontend_small", seed=0)
    coords = synth.reproject(p["poses_gt"], p["disps_gt"], p["intrinsics"], ii, jj).float()
    coords = (coords + torch.randn(coords.shape, generator=g)).to(cuda)[None]
    out = hcorr.CorrLookup.apply(f1, f2, coords, r, L)
    G = torch.randn(out.shape, generator=g).to(cuda)
    loss = (out.float() * G).sum()
    g1, g2 = torch.autograd.grad(loss, [f1, f2])

    def oracle_loss(a, b):
        pyr = oracle.corr.pyramid(a[None], b[None], L)
        o = oracle.corr.corr_block_lookup(pyr, coords.double().cpu().numpy(), r)
        return float((o * G.double().cpu().numpy()).sum())

    a0 = f1.detach().double().cpu().numpy()[0]
    b0 = f2.detach().double().cpu().numpy()[0]
    ref = oracle.corr.corr_block_lookup(oracle.corr.pyramid(a0[None], b0[None], L), coords.double().cpu().numpy(), r)
    assert rel(out, ref) < 2e-3
    h = 1e-6
    for which, grad in (("fmap1", g1), ("fmap2", g2)):
        d = torch.randn(a0.shape, generator=g, dtype=torch.float64).numpy()
        if which == "fmap1":
            fd = (oracle_loss(a0 + h * d, b0) - oracle_loss(a0 - h * d, b0)) / (2 * h)
        else:
            fd = (oracle_loss(a0, b0 + h * d) - oracle_loss(a0, b0 - h * d)) / (2 * h)
        an = float((grad.double().cpu().numpy()[0] * d).sum())
        print("%s: directional derivative adjoint %.6e finite difference %.6e" % (which, an, fd))
        assert abs(an - fd) <= TOL * abs(fd), (which, an, fd)
