"""The pure-PyTorch restatement of HI-SLAM2's Python bundle adjustment (oracle/torch_path.py,
the CPU baseline bench.py times): its Jacobians against central finite differences of its
own reprojection, and one iteration moving the poses toward the ground truth as the
float64 oracle of the CUDA operator does (the two differ by design: damping before the
Schur complement, MIN_DEPTH 0.2, eta + 1e-7, the final disparity clamp)."""

import numpy as np
import torch

import oracle
from oracle import torch_path as tp
from hislam2_b200 import synth


def test_projective_jacobians_match_finite_differences():
    p = synth.make_ba_problem("tiny6", seed=0)
    poses, disps, intr = p["poses"].double(), p["disps"].double(), p["intrinsics"].double()
    ii, jj = p["ii"][:4], p["jj"][:4]
    coords, valid, (Ji, Jj, Jz) = tp.projective_transform(poses, disps, intr, ii, jj)
    h = 1e-6
    for k in range(6):
        d = torch.zeros(6, dtype=torch.float64)
        d[k] = h
        for which, J in (("j", Jj), ("i", Ji)):
            pp, pm = poses.clone(), poses.clone()
            idx = jj if which == "j" else ii
            for e in range(len(idx)):
                f = int(idx[e])
                pp[f] = tp.retr(poses[f:f + 1], d[None])[0]
                pm[f] = tp.retr(poses[f:f + 1], -d[None])[0]
                cp = tp.projective_transform(pp, disps, intr, ii[e:e + 1], jj[e:e + 1])[0]
                cm = tp.projective_transform(pm, disps, intr, ii[e:e + 1], jj[e:e + 1])[0]
                fd = (cp - cm) / (2 * h)
                assert torch.allclose(J[e, ..., k], fd[0], atol=1e-5, rtol=1e-5), (which, k, e)
                pp[f], pm[f] = poses[f], poses[f]
    dp, dm = disps.clone(), disps.clone()
    dp[ii[0]] += h
    dm[ii[0]] -= h
    fd = (tp.projective_transform(poses, dp, intr, ii[:1], jj[:1])[0]
          - tp.projective_transform(poses, dm, intr, ii[:1], jj[:1])[0]) / (2 * h)
    assert torch.allclose(Jz[0, ..., 0], fd[0], atol=1e-5, rtol=1e-5)


def test_one_iteration_moves_toward_ground_truth():
    p = synth.make_ba_problem("frontend_small", seed=0)
    t0 = p["t0"]
    tg = p["targets"].permute(0, 2, 3, 1).contiguous()
    wt = p["weights"].permute(0, 2, 3, 1).contiguous()
    M = len(torch.unique(p["ii"]))
    po, di, dzcov = tp.BA(tg, wt, p["eta"][:M], p["poses"], p["disps"], p["intrinsics"], p["ii"], p["jj"], t0,
                          ep=p["ep"], lm=p["lm"])
    gt = p["poses_gt"].numpy()
    e0 = np.abs(p["poses"].numpy() - gt).max()
    assert np.abs(po.numpy() - gt).max() < 0.1 * e0
    r = oracle.ba.ba(p["poses"].numpy(), p["disps"].numpy(), p["intrinsics"].numpy(), p["targets"].numpy(),
                     p["weights"].numpy(), p["eta"].numpy(), p["ii"].numpy(), p["jj"].numpy(), t0, p["t1"], 1,
                     p["lm"], p["ep"])
    assert np.abs(po.numpy() - r.poses).max() < 0.1 * e0
    assert dzcov.shape == (M, 48 * 64) and bool((dzcov > 0).all())
    np.testing.assert_array_equal(po[:t0].numpy(), p["poses"][:t0].numpy())
