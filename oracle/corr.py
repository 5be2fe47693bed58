"""Correlation operators of ``droid_backends``, restated in float64 numpy.

Follows HI-SLAM2:
  * ``src/correlation_kernels.cu:19-70``  corr_index_forward_kernel;
  * ``src/correlation_kernels.cu:73-124`` corr_index_backward_kernel;
  * ``src/altcorr_kernel.cu:25-75,132-172``  altcorr forward (+ ATen bilinear/permute);
  * ``src/altcorr_kernel.cu:79-129,175-225`` altcorr backward (reference scale: the
    forward's 1/16 is NOT applied, :124-125; ``scale`` selects the true adjoint);
  * ``hislam2/modules/corr.py:29-38,63-71``   CorrBlock all-pairs volume + pyramid.
Test infrastructure only.
"""

import numpy as np


def _window(coords_x, coords_y, r):
    fx = np.floor(coords_x)
    fy = np.floor(coords_y)
    return fx.astype(np.int64), fy.astype(np.int64), coords_x - fx, coords_y - fy


def corr_index_forward(volume, coords, r):
    """volume [N,H1,W1,H2,W2], coords [N,2,H1,W1] -> corr [N,2r+1,2r+1,H1,W1].

    corr[n,a,b] = sum of the 4 bilinear taps around (x0 - r + a, y0 - r + b); dim 1
    runs along x, dim 2 along y; taps outside [0,H2)x[0,W2) contribute 0.
    """
    vol = np.asarray(volume, dtype=np.float64)
    crd = np.asarray(coords, dtype=np.float64)
    N, H1, W1, H2, W2 = vol.shape
    rd = 2 * r + 1
    x0, y0, dx, dy = _window(crd[:, 0], crd[:, 1], r)
    # V[n, i, j, y, x] = vol[n, y, x, y0-r+j, x0-r+i]  for i, j in [0, rd]
    V = np.zeros((N, rd + 1, rd + 1, H1, W1))
    nn, yy, xx = np.meshgrid(np.arange(N), np.arange(H1), np.arange(W1), indexing="ij")
    for i in range(rd + 1):
        for j in range(rd + 1):
            x1 = x0 - r + i
            y1 = y0 - r + j
            ok = (x1 >= 0) & (x1 < W2) & (y1 >= 0) & (y1 < H2)
            V[:, i, j][ok] = vol[nn[ok], yy[ok], xx[ok], y1[ok], x1[ok]]
    dx = dx[:, None, None]
    dy = dy[:, None, None]
    return ((1 - dx) * (1 - dy) * V[:, :rd, :rd] + (1 - dx) * dy * V[:, :rd, 1:]
            + dx * (1 - dy) * V[:, 1:, :rd] + dx * dy * V[:, 1:, 1:])


def corr_index_backward(volume_shape, coords, corr_grad, r):
    """Adjoint of :func:`corr_index_forward` (``correlation_kernels.cu:73-124``)."""
    crd = np.asarray(coords, dtype=np.float64)
    g = np.asarray(corr_grad, dtype=np.float64)
    N, H1, W1, H2, W2 = volume_shape
    rd = 2 * r + 1
    x0, y0, dx, dy = _window(crd[:, 0], crd[:, 1], r)
    G = np.zeros((N, rd + 1, rd + 1, H1, W1))
    dx = dx[:, None, None]
    dy = dy[:, None, None]
    G[:, :rd, :rd] += (1 - dx) * (1 - dy) * g
    G[:, :rd, 1:] += (1 - dx) * dy * g
    G[:, 1:, :rd] += dx * (1 - dy) * g
    G[:, 1:, 1:] += dx * dy * g
    out = np.zeros((N, H1, W1, H2, W2))
    nn, yy, xx = np.meshgrid(np.arange(N), np.arange(H1), np.arange(W1), indexing="ij")
    for i in range(rd + 1):
        for j in range(rd + 1):
            x1 = x0 - r + i
            y1 = y0 - r + j
            ok = (x1 >= 0) & (x1 < W2) & (y1 >= 0) & (y1 < H2)
            # each (n,y,x) row owns distinct (y1,x1) taps: no collisions
            out[nn[ok], yy[ok], xx[ok], y1[ok], x1[ok]] += G[:, i, j][ok]
    return out


def all_pairs(fmap1, fmap2):
    """CorrBlock.corr (``modules/corr.py:63-71``): (f1/4)^T (f2/4) per (batch, num).

    fmap1/fmap2 [B,N,C,H,W] -> [B,N,H,W,H,W].
    """
    f1 = np.asarray(fmap1, dtype=np.float64)
    f2 = np.asarray(fmap2, dtype=np.float64)
    B, N, C, H, W = f1.shape
    a = f1.reshape(B * N, C, H * W) / 4.0
    b = f2.reshape(B * N, C, H * W) / 4.0
    return np.matmul(np.swapaxes(a, 1, 2), b).reshape(B, N, H, W, H, W)


def avg_pool2(x):
    """2x2 stride-2 average pool over the last two axes, floor sizes (F.avg_pool2d)."""
    h, w = x.shape[-2] // 2, x.shape[-1] // 2
    x = x[..., : 2 * h, : 2 * w]
    return 0.25 * (x[..., 0::2, 0::2] + x[..., 1::2, 0::2] + x[..., 0::2, 1::2] + x[..., 1::2, 1::2])


def pyramid(fmap1, fmap2, num_levels=4):
    """CorrBlock.__init__ (``modules/corr.py:29-38``): list of [B*N,H,W,H/2^i,W/2^i]."""
    c = all_pairs(fmap1, fmap2)
    B, N, H, W = c.shape[:4]
    c = c.reshape(B * N, H, W, H, W)
    out = []
    for _ in range(num_levels):
        out.append(c)
        c = avg_pool2(c)
    return out


def corr_block_lookup(pyr, coords, r):
    """CorrBlock.__call__ (``modules/corr.py:40-51``) for coords [B,N,H,W,2]."""
    crd = np.asarray(coords, dtype=np.float64)
    B, N, H, W, _ = crd.shape
    c = np.transpose(crd, (0, 1, 4, 2, 3)).reshape(B * N, 2, H, W)
    outs = []
    for i, vol in enumerate(pyr):
        o = corr_index_forward(vol, c / 2 ** i, r)
        outs.append(o.reshape(B, N, -1, H, W))
    return np.concatenate(outs, axis=2)


def altcorr_forward(fmap1, fmap2, coords, ii, jj, r):
    """fmap1 [B,N1,C,H,W], fmap2 [B,N2,C,H2,W2], coords [B,M,2,H,W] -> [B,M,2r+1,2r+1,H,W].

    Inner products over the D x D integer window (D = 2r+2) with the /4 /4 scaling
    (``altcorr_kernel.cu:62-71``), bilinear blend (:160-169), then dims 2/3 swapped so
    that dim 2 runs along x (:171).
    """
    f1 = np.asarray(fmap1, dtype=np.float64)
    f2 = np.asarray(fmap2, dtype=np.float64)
    crd = np.asarray(coords, dtype=np.float64)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    B, M, _, H, W = crd.shape
    H2, W2 = f2.shape[3], f2.shape[4]
    D = 2 * r + 2
    x0, y0, dx, dy = _window(crd[:, :, 0], crd[:, :, 1], r)
    corr = np.zeros((B, M, D, D, H, W))
    for b in range(B):
        for m in range(M):
            a = f1[b, ii[m]] / 4.0                       # [C,H,W]
            g = f2[b, jj[m]] / 4.0                       # [C,H2,W2]
            for p in range(D):                           # along y
                i1 = y0[b, m] + p - r
                for q in range(D):                       # along x
                    j1 = x0[b, m] + q - r
                    ok = (i1 >= 0) & (i1 < H2) & (j1 >= 0) & (j1 < W2)
                    s = np.zeros((H, W))
                    yy, xx = np.nonzero(ok)
                    s[yy, xx] = np.einsum("cn,cn->n", a[:, yy, xx], g[:, i1[yy, xx], j1[yy, xx]])
                    corr[b, m, p, q] = s
    dx = dx[:, :, None, None]
    dy = dy[:, :, None, None]
    out = ((1 - dx) * (1 - dy) * corr[:, :, :-1, :-1] + dx * (1 - dy) * corr[:, :, :-1, 1:]
           + (1 - dx) * dy * corr[:, :, 1:, :-1] + dx * dy * corr[:, :, 1:, 1:])
    return np.transpose(out, (0, 1, 3, 2, 4, 5))


def altcorr_backward(fmap1, fmap2, coords, ii, jj, grad, r, scale=1.0):
    """Gradients w.r.t. fmap1/fmap2 (``altcorr_kernel.cu:79-129,175-225``).

    ``scale=1`` reproduces the reference operator, which omits the forward's 1/16;
    ``scale=1/16`` is the true adjoint of :func:`altcorr_forward`.
    """
    f1 = np.asarray(fmap1, dtype=np.float64)
    f2 = np.asarray(fmap2, dtype=np.float64)
    crd = np.asarray(coords, dtype=np.float64)
    ii = np.asarray(ii, dtype=np.int64)
    jj = np.asarray(jj, dtype=np.int64)
    g = np.transpose(np.asarray(grad, dtype=np.float64), (0, 1, 3, 2, 4, 5))  # [B,M,y,x,H,W]
    B, M, _, H, W = crd.shape
    H2, W2 = f2.shape[3], f2.shape[4]
    D = 2 * r + 2
    x0, y0, dx, dy = _window(crd[:, :, 0], crd[:, :, 1], r)
    dx = dx[:, :, None, None]
    dy = dy[:, :, None, None]
    cg = np.zeros((B, M, D, D, H, W))
    cg[:, :, :-1, :-1] += (1 - dx) * (1 - dy) * g
    cg[:, :, :-1, 1:] += dx * (1 - dy) * g
    cg[:, :, 1:, :-1] += (1 - dx) * dy * g
    cg[:, :, 1:, 1:] += dx * dy * g
    g1 = np.zeros_like(f1)
    g2 = np.zeros_like(f2)
    for b in range(B):
        for m in range(M):
            for p in range(D):
                i1 = y0[b, m] + p - r
                for q in range(D):
                    j1 = x0[b, m] + q - r
                    ok = (i1 >= 0) & (i1 < H2) & (j1 >= 0) & (j1 < W2)
                    yy, xx = np.nonzero(ok)
                    gv = cg[b, m, p, q, yy, xx] * scale
                    g1[b, ii[m]][:, yy, xx] += gv * f2[b, jj[m]][:, i1[yy, xx], j1[yy, xx]]
                    np.add.at(g2[b, jj[m]], (slice(None), i1[yy, xx], j1[yy, xx]),
                              gv * f1[b, ii[m]][:, yy, xx])
    return g1, g2
