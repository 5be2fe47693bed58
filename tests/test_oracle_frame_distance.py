"""frame_distance oracle against a pure-Python loop and limiting cases."""

import numpy as np

from oracle import frame_distance as ofd
from oracle import se3


def loop_frame_distance(poses, disps, intr, ii, jj, beta):
    fx, fy, cx, cy = intr
    out = []
    for a, b in zip(ii, jj):
        tij, qij = se3.rel_se3(poses[a, :3], poses[a, 3:], poses[b, :3], poses[b, 3:])
        acc = val = tot = 0.0
        H, W = disps.shape[1:]
        for v in range(H):
            for u in range(W):
                d = disps[a, v, u]
                X = np.array([(u - cx) / fx, (v - cy) / fy, 1.0])
                Y = se3.act_so3(qij, X) + d * tij
                for wgt, P in ((beta, Y), (1 - beta, X + d * tij)):
                    tot += wgt
                    if P[2] > 0.25:
                        du = fx * P[0] / P[2] + cx - u
                        dv = fy * P[1] / P[2] + cy - v
                        acc += wgt * np.hypot(du, dv)
                        val += wgt
        out.append(1000.0 if val / (tot + 1e-8) < 0.75 else acc / val)
    return np.array(out)


def rand_poses(rng, K, sigma):
    xi = sigma * rng.standard_normal((K, 6))
    t, q = se3.exp_se3(xi)
    return np.concatenate([t, q], -1)


def test_matches_loop():
    rng = np.random.default_rng(0)
    K, H, W = 4, 5, 7
    poses = rand_poses(rng, K, 0.1)
    disps = rng.uniform(0.2, 1.0, (K, H, W))
    intr = np.array([5.0, 5.5, 3.0, 2.0])
    ii = np.array([0, 1, 2, 3, 0])
    jj = np.array([1, 2, 3, 0, 0])
    np.testing.assert_allclose(ofd.frame_distance(poses, disps, intr, ii, jj, 0.3),
                               loop_frame_distance(poses, disps, intr, ii, jj, 0.3), rtol=1e-12)


def test_limits():
    rng = np.random.default_rng(1)
    K, H, W = 2, 6, 8
    poses = np.tile(np.array([0, 0, 0, 0, 0, 0, 1.0]), (K, 1))
    disps = rng.uniform(0.2, 1.0, (K, H, W))
    intr = np.array([5.0, 5.0, 4.0, 3.0])
    d = ofd.frame_distance(poses, disps, intr, np.array([0]), np.array([1]), 0.3)
    assert abs(d[0]) < 1e-12
    poses[1, 2] = -10.0  # frame 1 far behind: every point lands behind the camera
    d = ofd.frame_distance(poses, disps, intr, np.array([0]), np.array([1]), 0.3)
    assert d[0] == 1000.0
