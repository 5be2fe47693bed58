"""ba on the B200 kernels against the float64 oracle (parity) and, at the 300-keyframe
size, against size-independent properties.

Tolerances (FP32 kernels vs the FP64 oracle): 1e-4 relative to the largest
entry for the reduced camera system (Hessian blocks), poses and disparities,
the bar stated for the plain FP32 form; integer keys are compared bit-exactly.
"""

import numpy as np
import pytest
import torch

import droid_backends
import oracle
from hislam2_b200 import backends, synth

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def np64(t):
    return t.detach().cpu().double().numpy()


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def on(p, dev):
    return {k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in p.items()}


def subproblem(p, frames):
    """Edges of p among the first `frames` keyframes (all pose/disp buffers kept)."""
    m = (p["ii"] < frames) & (p["jj"] < frames)
    q = dict(p)
    for k in ("ii", "jj", "targets", "weights"):
        q[k] = p[k][m].contiguous()
    q["t1"] = frames
    q["eta"] = p["eta"][:frames].contiguous()
    return q


def run_gpu(p, dev, iters=None, motion_only=False, eta=None):
    q = on(p, dev)
    poses, disps = q["poses"].clone(), q["disps"].clone()
    dx, dz, dzcov = droid_backends.ba(poses, disps, q["intrinsics"], q["targets"], q["weights"],
                                      q["eta"] if eta is None else eta.to(dev), q["ii"], q["jj"], q["t0"],
                                      q["t1"], p["iters"] if iters is None else iters, q["lm"], q["ep"],
                                      motion_only)
    torch.cuda.synchronize()
    assert dzcov is None
    return poses, disps, dx, dz


def run_oracle(p, iters=None, motion_only=False, eta=None, trace=False):
    return oracle.ba.ba(np64(p["poses"]), np64(p["disps"]), np64(p["intrinsics"]), np64(p["targets"]),
                        np64(p["weights"]), np64(p["eta"] if eta is None else eta), p["ii"].numpy(),
                        p["jj"].numpy(), p["t0"], p["t1"], p["iters"] if iters is None else iters, p["lm"],
                        p["ep"], motion_only=motion_only, trace=trace)


def oracle_reduced_system(p, motion_only=False):
    r = run_oracle(p, iters=1, motion_only=motion_only, trace=True)
    it = r.traces[0]
    if motion_only:
        return it["A"], it["b"]
    return it["A"] - it["S"], it["b"] - it["bS"]


def star_problem(extra=48):
    """60 frames of the 300-kf workload plus `extra` edges out of frame 12.  With 48 its depth
    frame has 49 Schur rows, past the tensor-core Gram's limit of 42, so both Gram kernels run;
    with 24 it has about 30 (two 128-row M tiles of the tensor-core Gram)."""
    p = subproblem(synth.make_ba_problem("backend300", seed=3), 60)
    extra_j = torch.arange(13, 13 + extra) % 60
    extra_j[extra_j == 12] = 0
    extra_i = torch.full_like(extra_j, 12)
    coords = synth.reproject(p["poses_gt"], p["disps_gt"], p["intrinsics"], extra_i, extra_j)
    q = dict(p)
    q["ii"] = torch.cat([p["ii"], extra_i])
    q["jj"] = torch.cat([p["jj"], extra_j])
    q["targets"] = torch.cat([p["targets"], coords.permute(0, 3, 1, 2).float()]).contiguous()
    q["weights"] = torch.cat([p["weights"], torch.full_like(p["weights"][:extra], 0.5)]).contiguous()
    return q


CASES = {
    "frontend_small": lambda: synth.make_ba_problem("frontend_small", seed=0),
    "frontend": lambda: synth.make_ba_problem("frontend", seed=1),
    "backend40": lambda: subproblem(synth.make_ba_problem("backend300", seed=2), 40),
    "star60": star_problem,
    "wide60": lambda: star_problem(extra=24),
}


@pytest.fixture(params=[0, 1, 2], ids=["gram_tc", "gram_simt", "fused"])
def schur_path(request):
    from hislam2_b200 import _lib
    _lib.set_schur_path(request.param)
    yield request.param
    _lib.set_schur_path(0)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("motion_only", [False, True])
def test_reduced_system_matches_oracle(cuda, case, motion_only, schur_path):
    p = CASES[case]()
    q = on(p, cuda)
    A, b = backends.ba_reduced_system(q["poses"], q["disps"], q["intrinsics"], q["targets"], q["weights"],
                                      q["eta"], q["ii"], q["jj"], q["t0"], q["t1"], motion_only)
    Ao, bo = oracle_reduced_system(p, motion_only)
    assert rel(np64(A), Ao) < RTOL, rel(np64(A), Ao)
    assert rel(np64(b), bo) < RTOL, rel(np64(b), bo)
    # symmetric up to the order of the FP64 atomic sums
    assert rel(np64(A), np64(A.t())) < 1e-12


@pytest.mark.parametrize("case", list(CASES))
def test_ba_matches_oracle(cuda, case, schur_path):
    p = CASES[case]()
    poses, disps, dx, dz = run_gpu(p, cuda)
    r = run_oracle(p)
    assert rel(np64(poses), r.poses) < RTOL, rel(np64(poses), r.poses)
    assert rel(np64(disps), r.disps) < RTOL, rel(np64(disps), r.disps)
    assert dz.shape == (len(r.kx), p["disps"].shape[1] * p["disps"].shape[2])
    # the step of the first iteration (later ones shrink towards the FP32 noise floor)
    poses, disps, dx, dz = run_gpu(p, cuda, iters=1)
    r = run_oracle(p, iters=1)
    assert rel(np64(dx), r.dx) < 1e-4, rel(np64(dx), r.dx)
    assert rel(np64(dz), r.dz) < 1e-4, rel(np64(dz), r.dz)


def test_motion_only_matches_oracle(cuda):
    p = CASES["frontend"]()
    poses, disps, dx, dz = run_gpu(p, cuda, motion_only=True)
    r = run_oracle(p, motion_only=True)
    assert dz is None
    assert torch.equal(disps.cpu(), p["disps"])
    assert rel(np64(poses), r.poses) < RTOL
    poses, disps, dx, dz = run_gpu(p, cuda, iters=1, motion_only=True)
    r = run_oracle(p, iters=1, motion_only=True)
    assert rel(np64(dx), r.dx) < 1e-4


@pytest.mark.parametrize("case", ["frontend", "backend40"])
def test_keys_bit_exact(cuda, case):
    p = CASES[case]()
    q = on(p, cuda)
    kx, kk, rptr, rows = backends.ba_keys(q["poses"], q["disps"], q["ii"], q["jj"], p["t0"], p["t1"])
    okx, okk, ii_exp = oracle.ba.keys(p["ii"].numpy(), p["t0"], p["t1"])
    assert np.array_equal(kx.numpy(), okx)
    assert np.array_equal(kk.numpy(), okk)
    jj_exp = np.concatenate([np.arange(p["t0"], p["t1"]), p["jj"].numpy()])
    orows = oracle.ba.schur_rows(jj_exp, okk, p["t0"], p["t1"])
    for k in range(len(okx)):
        got = rows[rptr[k]:rptr[k + 1]].tolist()
        assert got == orows.get(k, []), k


def test_edge_cases_match_oracle(cuda):
    base = CASES["frontend_small"]()
    # (a) no edges at all: the depth frames are the window frames alone
    p = dict(base)
    p["eta"] = base["eta"][base["t0"]:].contiguous()
    for k in ("ii", "jj"):
        p[k] = base[k][:0]
    for k in ("targets", "weights"):
        p[k] = base[k][:0].contiguous()
    poses, disps, dx, dz = run_gpu(p, cuda)
    r = run_oracle(p)
    assert rel(np64(poses), r.poses) < RTOL and rel(np64(disps), r.disps) < RTOL
    # (b) empty window t0 == t1
    p = dict(base)
    p["t0"] = p["t1"] = 8
    poses, disps, dx, dz = run_gpu(p, cuda)
    r = run_oracle(p)
    assert dx.shape == (0, 6)
    assert rel(np64(disps), r.disps) < RTOL
    # (c) self edges and a duplicated edge
    p = dict(base)
    extra = torch.tensor([3, 5, 4], dtype=torch.int64)
    p["ii"] = torch.cat([base["ii"], extra])
    p["jj"] = torch.cat([base["jj"], torch.tensor([3, 5, base["jj"][0].item()])])
    p["ii"][-1] = base["ii"][0]
    for k in ("targets", "weights"):
        p[k] = torch.cat([base[k], base[k][:3]]).contiguous()
    poses, disps, dx, dz = run_gpu(p, cuda)
    r = run_oracle(p)
    assert rel(np64(poses), r.poses) < RTOL and rel(np64(disps), r.disps) < RTOL
    # (d) eta broadcast from one row
    eta1 = base["eta"][:1].clone() * 3
    poses, disps, dx, dz = run_gpu(base, cuda, eta=eta1)
    r = run_oracle(base, eta=eta1)
    assert rel(np64(disps), r.disps) < RTOL
    # (e) pose/disparity buffers longer than the frames in use
    p = dict(base)
    p["poses"] = torch.cat([base["poses"], base["poses"][:5]]).contiguous()
    p["disps"] = torch.cat([base["disps"], base["disps"][:5]]).contiguous()
    poses, disps, dx, dz = run_gpu(p, cuda)
    r = run_oracle(p)
    assert rel(np64(poses), r.poses) < RTOL and rel(np64(disps), r.disps) < RTOL
    assert torch.equal(poses[8:].cpu(), p["poses"][8:])


def test_invalid_inputs_raise_and_leave_state(cuda):
    base = on(CASES["frontend_small"](), cuda)
    poses, disps = base["poses"].clone(), base["disps"].clone()
    args = lambda ii, jj, eta, t1: (poses, disps, base["intrinsics"], base["targets"], base["weights"], eta,  # noqa
                                    ii, jj, base["t0"], t1, 2, base["lm"], base["ep"], False)
    bad = base["ii"].clone()
    bad[3] = 99
    with pytest.raises(RuntimeError, match="out of range"):
        droid_backends.ba(*args(bad, base["jj"], base["eta"], 8))
    with pytest.raises(RuntimeError, match="out of range"):
        droid_backends.ba(*args(base["ii"], base["jj"], base["eta"], 6))   # jj >= t1
    with pytest.raises(RuntimeError, match="eta"):
        droid_backends.ba(*args(base["ii"], base["jj"], base["eta"][:5].contiguous(), 8))
    assert torch.equal(poses, base["poses"]) and torch.equal(disps, base["disps"])
    with pytest.raises(RuntimeError, match="t0 <= t1"):
        droid_backends.ba(*args(base["ii"], base["jj"], base["eta"], 9))


def test_failed_factorisation_zero_update(cuda):
    p = CASES["frontend_small"]()
    p["ep"] = -1e3
    poses, disps, dx, dz = run_gpu(p, cuda)
    r = run_oracle(p)
    assert not r.ok
    assert torch.count_nonzero(dx) == 0
    assert torch.equal(poses.cpu(), p["poses"])
    assert rel(np64(disps), r.disps) < RTOL


def test_backend300_full_size_properties(cuda):
    p = synth.make_ba_problem("backend300", seed=0)
    q = on(p, cuda)
    # one step solves the damped reduced system it builds (FP64 both sides)
    A, b = backends.ba_reduced_system(q["poses"], q["disps"], q["intrinsics"], q["targets"], q["weights"],
                                      q["eta"], q["ii"], q["jj"], q["t0"], q["t1"])
    assert rel(np64(A), np64(A.t())) < 1e-12
    Ad = A.clone()
    Ad.diagonal().add_(p["ep"] + p["lm"] * A.diagonal())
    x_ref = torch.linalg.solve(Ad, b)
    poses1, disps1, dx1, dz1 = run_gpu(p, cuda, iters=1)
    assert rel(dx1.double().cpu().numpy().reshape(-1), x_ref.cpu().numpy()) < 1e-5
    # eight iterations: finite, deterministic, closer to the ground truth
    poses, disps, dx, dz = run_gpu(p, cuda)
    poses2, disps2, _, _ = run_gpu(p, cuda)
    assert torch.isfinite(poses).all() and torch.isfinite(disps).all()
    assert rel(np64(poses), np64(poses2)) < 1e-6 and rel(np64(disps), np64(disps2)) < 1e-6
    t0 = p["t0"]
    e0 = (p["poses"][t0:, :3] - p["poses_gt"][t0:, :3]).abs().max()
    e1 = (poses[t0:, :3].cpu() - p["poses_gt"][t0:, :3]).abs().max()
    assert e1 < e0
    assert torch.equal(poses[:t0].cpu(), p["poses"][:t0])
