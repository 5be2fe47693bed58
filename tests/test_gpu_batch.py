"""Batched BA (hs2_ba_batch: one persistent launch per LM iteration over many windows)
against the single-window operator (droid_backends.ba) on every window, and against
the float64 oracle on the small ones.

Tolerance: 1e-4 relative to the largest magnitude for poses and disparities after
several iterations and for dx and dz of a first iteration (the bar of the FP32 form;
the batch runs the same linearisation, the SIMT Gram in FP32 and a single-CTA FP64
Cholesky, so it agrees with the single-window path to FP32 rounding).  dx / dz of the
last of several iterations are not compared: converged, they are rounding noise.
"""

import numpy as np
import pytest
import torch

import droid_backends
import oracle
from hislam2_b200 import backends, synth

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.detach().double().cpu().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def on(w, dev):
    return {k: (v.to(dev).clone() if torch.is_tensor(v) else v) for k, v in w.items()}


def single(w, dev, iters):
    q = on(w, dev)
    dx, dz, _ = droid_backends.ba(q["poses"], q["disps"], q["intrinsics"], q["targets"], q["weights"], q["eta"],
                                  q["ii"], q["jj"], q["t0"], q["t1"], iters, q["lm"], q["ep"], False)
    torch.cuda.synchronize()
    return q["poses"], q["disps"], dx, dz


def mixed_windows():
    ws = [synth.make_ba_problem("tiny6"), synth.make_ba_problem("tiny7"), synth.make_ba_problem("frontend_small")]
    for w in ws:
        M = len(np.unique(np.concatenate([np.arange(w["t0"], w["t1"]), w["ii"].numpy()])))
        w["eta"] = w["eta"][:M].contiguous()
    return ws + synth.make_batch_problems(num_windows=5, seed=7)


def run_batch(ws, dev, iters, lm, ep, **kw):
    dev_ws = [on(dict(w, lm=lm, ep=ep), dev) for w in ws]
    plan = backends.BABatch(dev_ws, lm, ep, **kw)
    plan.run(iters)
    torch.cuda.synchronize()
    return dev_ws, plan.results()


@pytest.mark.parametrize("gram_split,ctas", [(1, 0), (4, 1), (8, 2)])
def test_batch_matches_single_window_operator(cuda, gram_split, ctas):
    ws = mixed_windows()
    lm, ep = 1e-4, 0.1
    dev_ws, _ = run_batch(ws, cuda, 3, lm, ep, gram_split=gram_split, ctas_per_sm=ctas)
    one_ws, res = run_batch(ws, cuda, 1, lm, ep, gram_split=gram_split, ctas_per_sm=ctas)
    for k, w in enumerate(ws):
        po, do, _, _ = single(dict(w, lm=lm, ep=ep), cuda, 3)
        assert rel(dev_ws[k]["poses"], po) < RTOL, k
        assert rel(dev_ws[k]["disps"], do) < RTOL, k
        _, _, xo, zo = single(dict(w, lm=lm, ep=ep), cuda, 1)
        assert rel(res[k][0], xo) < RTOL, k
        assert rel(res[k][1], zo) < RTOL, k


def test_batch_small_windows_match_oracle(cuda):
    ws = mixed_windows()[:3]
    lm, ep, iters = 1e-4, 0.1, 2
    dev_ws, _ = run_batch(ws, cuda, iters, lm, ep)
    _, res = run_batch(ws, cuda, 1, lm, ep)
    for k, w in enumerate(ws):
        f = lambda n: w[n].double().numpy()  # noqa: E731
        r = oracle.ba.ba(f("poses"), f("disps"), f("intrinsics"), f("targets"), f("weights"), f("eta"),
                         w["ii"].numpy(), w["jj"].numpy(), w["t0"], w["t1"], iters, lm, ep, trace=True)
        assert rel(dev_ws[k]["poses"], r.poses) < RTOL
        assert rel(dev_ws[k]["disps"], r.disps) < RTOL
        assert rel(res[k][0], r.traces[0]["dx"]) < RTOL
        assert rel(res[k][1], r.traces[0]["dz"].reshape(res[k][1].shape)) < RTOL


def test_batch_64_uneven_windows(cuda):
    """The batching configuration: 64 windows, keyframes 8..40, edges 20..500, 43x77 or 30x40."""
    ws = synth.make_batch_problems(num_windows=64, seed=0)
    lm, ep, iters = 1e-4, 0.1, 4
    dev_ws, _ = run_batch(ws, cuda, iters, lm, ep)
    _, res = run_batch(ws, cuda, 1, lm, ep)
    worst = 0.0
    for k in range(0, 64, 7):
        po, do, _, _ = single(ws[k], cuda, iters)
        _, _, xo, zo = single(ws[k], cuda, 1)
        worst = max(worst, rel(dev_ws[k]["poses"], po), rel(dev_ws[k]["disps"], do), rel(res[k][0], xo),
                    rel(res[k][1], zo))
    print("64 windows: worst relative difference to the single-window operator %.2e" % worst)
    assert worst < RTOL


def test_batch_graph_replay_matches_eager(cuda):
    ws = synth.make_batch_problems(num_windows=8, seed=2)
    lm, ep, iters = 1e-4, 0.1, 3
    eager = [on(w, cuda) for w in ws]
    BA = backends.BABatch(eager, lm, ep)
    BA.run(iters)
    torch.cuda.synchronize()
    graphed = [on(w, cuda) for w in ws]
    init = [(g["poses"].clone(), g["disps"].clone()) for g in graphed]
    plan = backends.BABatch(graphed, lm, ep)
    g = plan.graph(iters)
    for _ in range(2):
        for w, (p0, d0) in zip(graphed, init):
            w["poses"].copy_(p0)
            w["disps"].copy_(d0)
        g.replay()
        torch.cuda.synchronize()
        for a, b in zip(graphed, eager):
            assert rel(a["poses"], b["poses"]) < 1e-5 and rel(a["disps"], b["disps"]) < 1e-5


def test_batch_reports_a_bad_window(cuda):
    ws = [on(w, cuda) for w in synth.make_batch_problems(num_windows=3, seed=4)]
    ws[1]["jj"] = ws[1]["jj"].clone()
    ws[1]["jj"][0] = ws[1]["t1"]            # an edge index >= t1
    with pytest.raises(RuntimeError, match="window 1"):
        backends.BABatch(ws, 1e-4, 0.1)


def test_batch_bounded_wait_runs_out_and_reports(cuda):
    """A dependency wait that nothing can satisfy gives up after its poll limit: the
    launch drains, every window reports HS2_DEV_TIMEOUT (RuntimeError), and the context
    stays usable for the next call."""
    from hislam2_b200 import _lib
    lib = _lib.load()
    ws = [on(w, cuda) for w in synth.make_batch_problems(num_windows=4, seed=5)]
    plan = backends.BABatch(ws, 1e-4, 0.1)
    try:
        _lib.check(lib.hs2_ba_batch_set_wait_test(1000, 1), "ba_batch_set_wait_test")
        plan.run(1)
        torch.cuda.synchronize()
    finally:
        _lib.check(lib.hs2_ba_batch_set_wait_test(0, 0), "ba_batch_set_wait_test")
    with pytest.raises(RuntimeError, match="timed out"):
        plan.check()
    fresh = [on(w, cuda) for w in synth.make_batch_problems(num_windows=4, seed=5)]
    plan2 = backends.BABatch(fresh, 1e-4, 0.1)
    plan2.run(1)
    plan2.check()
    po, _, _, _ = single(synth.make_batch_problems(num_windows=4, seed=5)[0], cuda, 1)
    assert rel(fresh[0]["poses"], po) < RTOL
