"""The correlation oracle checked against independent restatements and identities."""

import numpy as np

from oracle import corr as oc


def loop_corr_index_forward(volume, coords, r):
    """Pure-Python restatement of the reference's per-thread scatter loop
    (``src/correlation_kernels.cu:44-68``); tiny inputs only."""
    N, H1, W1, H2, W2 = volume.shape
    rd = 2 * r + 1
    out = np.zeros((N, rd, rd, H1, W1))
    for n in range(N):
        for y in range(H1):
            for x in range(W1):
                x0, y0 = coords[n, 0, y, x], coords[n, 1, y, x]
                dx, dy = x0 - np.floor(x0), y0 - np.floor(y0)
                for i in range(rd + 1):
                    for j in range(rd + 1):
                        x1 = int(np.floor(x0)) - r + i
                        y1 = int(np.floor(y0)) - r + j
                        if 0 <= y1 < H2 and 0 <= x1 < W2:
                            s = volume[n, y, x, y1, x1]
                            if i > 0 and j > 0:
                                out[n, i - 1, j - 1, y, x] += s * dx * dy
                            if i > 0 and j < rd:
                                out[n, i - 1, j, y, x] += s * dx * (1 - dy)
                            if i < rd and j > 0:
                                out[n, i, j - 1, y, x] += s * (1 - dx) * dy
                            if i < rd and j < rd:
                                out[n, i, j, y, x] += s * (1 - dx) * (1 - dy)
    return out


def rand_coords(rng, N, H, W, H2, W2, spread=3.0):
    return np.stack([rng.uniform(-spread, W2 - 1 + spread, (N, H, W)),
                     rng.uniform(-spread, H2 - 1 + spread, (N, H, W))], 1)


def test_corr_index_forward_matches_scatter_loop():
    rng = np.random.default_rng(0)
    N, H1, W1, H2, W2, r = 2, 3, 4, 5, 6, 2
    vol = rng.standard_normal((N, H1, W1, H2, W2))
    crd = rand_coords(rng, N, H1, W1, H2, W2)
    np.testing.assert_allclose(oc.corr_index_forward(vol, crd, r), loop_corr_index_forward(vol, crd, r),
                               atol=1e-12)


def test_corr_index_backward_is_adjoint():
    rng = np.random.default_rng(1)
    N, H1, W1, H2, W2, r = 2, 4, 5, 6, 7, 3
    vol = rng.standard_normal((N, H1, W1, H2, W2))
    crd = rand_coords(rng, N, H1, W1, H2, W2)
    g = rng.standard_normal((N, 2 * r + 1, 2 * r + 1, H1, W1))
    lhs = np.sum(oc.corr_index_forward(vol, crd, r) * g)
    rhs = np.sum(vol * oc.corr_index_backward(vol.shape, crd, g, r))
    assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(lhs))


def test_altcorr_equals_lookup_in_all_pairs_volume():
    rng = np.random.default_rng(2)
    B, N, C, H, W, r = 1, 3, 8, 5, 6, 2
    f1 = rng.standard_normal((B, N, C, H, W))
    f2 = rng.standard_normal((B, N, C, H, W))
    ii = np.array([0, 2, 1, 0])
    jj = np.array([1, 0, 2, 2])
    M = len(ii)
    crd = np.stack([rng.uniform(-2, W + 1, (B, M, H, W)), rng.uniform(-2, H + 1, (B, M, H, W))], 2)
    out = oc.altcorr_forward(f1, f2, crd, ii, jj, r)
    vol = oc.all_pairs(f1[:, ii], f2[:, jj]).reshape(B * M, H, W, H, W)
    ref = oc.corr_index_forward(vol, crd.reshape(B * M, 2, H, W), r).reshape(out.shape)
    np.testing.assert_allclose(out, ref, atol=1e-10)


def test_altcorr_backward_adjoint_and_reference_scale():
    rng = np.random.default_rng(3)
    B, N1, N2, C, H, W, r = 2, 2, 3, 4, 4, 5, 1
    f1 = rng.standard_normal((B, N1, C, H, W))
    f2 = rng.standard_normal((B, N2, C, H, W))
    ii = np.array([0, 1, 1])
    jj = np.array([2, 0, 2])
    M = len(ii)
    crd = np.stack([rng.uniform(-2, W + 1, (B, M, H, W)), rng.uniform(-2, H + 1, (B, M, H, W))], 2)
    G = rng.standard_normal((B, M, 2 * r + 1, 2 * r + 1, H, W))
    lhs = np.sum(oc.altcorr_forward(f1, f2, crd, ii, jj, r) * G)
    g1, g2 = oc.altcorr_backward(f1, f2, crd, ii, jj, G, r, scale=1.0 / 16)
    assert abs(lhs - np.sum(f1 * g1)) < 1e-10 * max(1, abs(lhs))
    assert abs(lhs - np.sum(f2 * g2)) < 1e-10 * max(1, abs(lhs))
    r1, r2 = oc.altcorr_backward(f1, f2, crd, ii, jj, G, r)
    np.testing.assert_allclose(r1, 16 * g1, atol=1e-10)
    np.testing.assert_allclose(r2, 16 * g2, atol=1e-10)


def test_pyramid_shapes_follow_floor_pooling():
    rng = np.random.default_rng(4)
    f = rng.standard_normal((1, 2, 4, 43 // 4, 77 // 4))
    pyr = oc.pyramid(f, f, 4)
    h, w = 43 // 4, 77 // 4
    assert [p.shape[-2:] for p in pyr] == [(h, w), (h // 2, w // 2), (h // 4, w // 4), (h // 8, w // 8)]
    np.testing.assert_allclose(pyr[1][0, 0, 0, 0, 0], pyr[0][0, 0, 0, :2, :2].mean())
