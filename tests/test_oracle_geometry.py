"""The iproj / covis_distance / depth_filter oracle against direct per-pixel loops written
from the reference kernels' text (src/droid_kernels.cu:996-1272), on small random cases."""

import numpy as np

import oracle
from oracle import se3


def _case(seed, K=9, ht=6, wd=8):
    rng = np.random.default_rng(seed)
    xi = 0.05 * rng.standard_normal((K, 6))
    t, q = se3.exp_se3(xi)
    poses = np.concatenate([t, q], axis=-1)
    disps = rng.uniform(0.2, 1.0, size=(K, ht, wd))
    intr = np.array([6.0, 6.5, 3.7, 2.6])
    return poses, disps, intr


def _rot(q, X):
    x, y, z, w = q
    uv = 2.0 * np.array([y * X[2] - z * X[1], z * X[0] - x * X[2], x * X[1] - y * X[0]])
    return X + w * uv + np.array([y * uv[2] - z * uv[1], z * uv[0] - x * uv[2], x * uv[1] - y * uv[0]])


def _rel(pi, pj):
    ti, qi, tj, qj = pi[:3], pi[3:], pj[:3], pj[3:]
    qij = np.array([-qj[3] * qi[0] + qj[0] * qi[3] - qj[1] * qi[2] + qj[2] * qi[1],
                    -qj[3] * qi[1] + qj[1] * qi[3] - qj[2] * qi[0] + qj[0] * qi[2],
                    -qj[3] * qi[2] + qj[2] * qi[3] - qj[0] * qi[1] + qj[1] * qi[0],
                    qj[3] * qi[3] + qj[0] * qi[0] + qj[1] * qi[1] + qj[2] * qi[2]])
    return tj - _rot(qij, ti), qij


def test_iproj_matches_loop():
    poses, disps, intr = _case(0)
    got = oracle.geometry.iproj(poses, disps, intr)
    fx, fy, cx, cy = intr
    for b in (0, 4, 8):
        for i in range(disps.shape[1]):
            for j in range(disps.shape[2]):
                d = disps[b, i, j]
                Y = _rot(poses[b, 3:], np.array([(j - cx) / fx, (i - cy) / fy, 1.0])) + d * poses[b, :3]
                np.testing.assert_allclose(got[b, i, j], Y / d, rtol=1e-12)


def test_covis_distance_matches_loop():
    poses, disps, intr = _case(1)
    poses[:, :3] *= 20.0          # large motions: some pixels leave the image
    ii = np.array([1, 4, 7])
    got = oracle.geometry.covis_distance(poses, disps, intr, ii)
    fx, fy, cx, cy = intr
    ht, wd = disps.shape[1:]
    for n, i in enumerate(ii):
        cnt = 0
        for y in range(ht):
            for x in range(wd):
                X = np.array([(x - cx) / fx, (y - cy) / fy, 1.0])
                outs = []
                for jx in (i - 1, i + 1):
                    t, q = _rel(poses[i], poses[jx])
                    Y = _rot(q, X) + disps[i, y, x] * t
                    u, v = fx * Y[0] / Y[2] + cx, fy * Y[1] / Y[2] + cy
                    outs.append(u < 0 or u >= wd or v < 0 or v >= ht)
                cnt += outs[0] and outs[1]
        assert got[n] == cnt / (ht * wd)
    assert 0 < got.max() <= 1


def test_depth_filter_matches_loop():
    poses, disps, intr = _case(2)
    disps[:] = disps[0:1]          # consistent depth across frames: many hits
    ix = np.array([0, 4, 8])
    thresh = np.array([0.4, 0.4, 0.05])
    got = oracle.geometry.depth_filter(poses, disps, intr, ix, thresh)
    fx, fy, cx, cy = intr
    num, ht, wd = disps.shape
    for b, i in enumerate(ix):
        for y in range(ht):
            for x in range(wd):
                cnt = 0
                for nb in range(6):
                    jx = i - nb - 1 if nb < 3 else i + nb
                    if jx < 0 or jx >= num:
                        continue
                    t, q = _rel(poses[i], poses[jx])
                    d = disps[i, y, x]
                    Y = _rot(q, np.array([(x - cx) / fx, (y - cy) / fy, 1.0])) + d * t
                    uj, vj, dj = fx * Y[0] / Y[2] + cx, fy * Y[1] / Y[2] + cy, d / Y[2]
                    u0, v0 = int(np.floor(uj)), int(np.floor(vj))
                    if 0 <= u0 < wd - 1 and 0 <= v0 < ht - 1:
                        ds = [disps[jx, v0, u0], disps[jx, v0, u0 + 1], disps[jx, v0 + 1, u0], disps[jx, v0 + 1, u0 + 1]]
                        cnt += any(abs(1.0 / dj - 1.0 / dd) < thresh[b] for dd in ds)
                assert got[b, y, x] == cnt
    assert got.max() >= 2


def test_proj_trans_matches_loop():
    poses, disps, intr = _case(3, K=5, ht=4, wd=5)
    rng = np.random.default_rng(3)
    ii = np.array([0, 0, 2, 3, 3, 1])
    jj = np.array([1, 2, 3, 2, 4, 1])            # includes a self edge (1 -> 1)
    E, (ht, wd) = len(ii), disps.shape[1:]
    targets = rng.uniform(0, 5, size=(E, 2, ht, wd))
    weights = rng.uniform(0, 2, size=(E, 2, ht, wd))
    C, w = oracle.geometry.proj_trans(poses, disps, intr[None], targets, weights, ii, jj)
    kx = np.unique(ii)
    assert C.shape == (len(kx), ht * wd)
    fx, fy, cx, cy = intr
    Cl, wl = np.zeros_like(C), np.zeros_like(w)
    for e in range(E):
        m = int(np.searchsorted(kx, ii[e]))
        t, q = _rel(poses[ii[e]], poses[jj[e]])
        for y in range(ht):
            for x in range(wd):
                h = disps[ii[e], y, x]
                Y = _rot(q, np.array([(x - cx) / fx, (y - cy) / fy, 1.0])) + h * t
                if Y[2] < 0.25:
                    continue
                d = 1.0 / Y[2]
                ju = fx * d * t[0] - fx * Y[0] * d * d * t[2]
                jv = fy * d * t[1] - fy * Y[1] * d * d * t[2]
                wu, wv = 0.001 * weights[e, 0, y, x], 0.001 * weights[e, 1, y, x]
                ru = targets[e, 0, y, x] - (fx * Y[0] / Y[2] + cx)
                rv = targets[e, 1, y, x] - (fy * Y[1] / Y[2] + cy)
                Cl[m, y * wd + x] += wu * ju * ju + wv * jv * jv
                wl[m, y * wd + x] += wu * ru * ju + wv * rv * jv
    np.testing.assert_allclose(C, Cl, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(w, wl, rtol=1e-12, atol=1e-15)


def test_bi_inter_properties():
    rng = np.random.default_rng(4)
    scales = rng.uniform(0.5, 2.0, size=(2, 3, 4))
    grids = np.stack([rng.uniform(0, 3 - 1e-6, size=(2, 5, 6)), rng.uniform(0, 2 - 1e-6, size=(2, 5, 6))], -1)
    grids[0, 0, 0] = (2.0, 1.0)                   # a grid node: exact value
    out, jac = oracle.geometry.bi_inter(scales, grids)
    np.testing.assert_allclose(jac.sum(axis=(-1, -2)), 1.0, rtol=1e-12)
    np.testing.assert_allclose(out, np.einsum("bijyx,byx->bij", jac, scales), rtol=1e-12)
    assert abs(out[0, 0, 0] - scales[0, 1, 2]) < 1e-12
    assert ((jac > 0).sum(axis=(-1, -2)) <= 4).all()
