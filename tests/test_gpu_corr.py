"""corr_index / altcorr on the B200 kernels against the float64 oracle, against the
reference's own kernels (oracle/_ref, when built) and by adjoint identities.

Tolerances: FP32/FP64 inputs 1e-5 relative to the largest output; FP16/BF16 inputs
are compared with the same kernels on the upcast input (the rounding of the
stored output only): 2^-8 / 2^-7 relative.  Integer window positions are
exercised bit-exactly through coordinates placed on and next to integer values.
"""

import numpy as np
import pytest
import torch

import droid_backends
from hislam2_b200 import synth
from oracle import corr as oc

pytestmark = pytest.mark.gpu


def np64(t):
    return t.detach().cpu().double().numpy()


def rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def make_lookup(N, H1, W1, H2, W2, seed, dev, dtype=torch.float32, spread=4.0, integer_frac=False):
    g = torch.Generator().manual_seed(seed)
    vol = torch.randn(N, H1, W1, H2, W2, generator=g)
    x = -spread + (W2 - 1 + 2 * spread) * torch.rand(N, H1, W1, generator=g)
    y = -spread + (H2 - 1 + 2 * spread) * torch.rand(N, H1, W1, generator=g)
    if integer_frac:
        # exact integers and values just below/above them: floor() must agree bit-exactly
        x = torch.round(x) + torch.tensor([0.0, -1e-6, 1e-6])[torch.randint(0, 3, x.shape, generator=g)]
        y = torch.round(y)
    coords = torch.stack([x, y], 1).contiguous()
    return vol.to(dev, dtype).contiguous(), coords.to(dev)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("r", [0, 1, 3, 4])
def test_corr_index_forward_backward_vs_oracle(cuda, dtype, r):
    vol, crd = make_lookup(3, 5, 7, 6, 9, seed=r, dev=cuda, dtype=dtype)
    out, = droid_backends.corr_index_forward(vol, crd, r)
    ref = oc.corr_index_forward(np64(vol), np64(crd), r)
    assert out.dtype == dtype and tuple(out.shape) == (3, 2 * r + 1, 2 * r + 1, 5, 7)
    assert rel(np64(out), ref) < 1e-5
    g = torch.randn(out.shape, device=cuda, dtype=dtype)
    vg, = droid_backends.corr_index_backward(vol, crd, g, r)
    refg = oc.corr_index_backward(vol.shape, np64(crd), np64(g), r)
    assert rel(np64(vg), refg) < 1e-5


def test_corr_index_integer_coordinates(cuda):
    vol, crd = make_lookup(2, 6, 8, 7, 10, seed=7, dev=cuda, integer_frac=True)
    out, = droid_backends.corr_index_forward(vol, crd, 3)
    assert rel(np64(out), oc.corr_index_forward(np64(vol), np64(crd), 3)) < 1e-5


@pytest.mark.parametrize("dtype,tol", [(torch.float16, 2 ** -8), (torch.bfloat16, 2 ** -7)])
def test_corr_index_half_types(cuda, dtype, tol):
    vol, crd = make_lookup(2, 9, 11, 9, 11, seed=3, dev=cuda, dtype=dtype)
    out, = droid_backends.corr_index_forward(vol, crd, 4)
    ref32, = droid_backends.corr_index_forward(vol.float(), crd, 4)
    assert out.dtype == dtype
    assert rel(np64(out), np64(ref32)) < tol
    g = torch.randn(out.shape, device=cuda).to(dtype)
    vg, = droid_backends.corr_index_backward(vol, crd, g, 4)
    vg32, = droid_backends.corr_index_backward(vol.float(), crd, g.float(), 4)
    assert rel(np64(vg), np64(vg32)) < tol


def test_corr_index_adjoint_at_full_size(cuda):
    """<fwd(V), G> == <V, bwd(G)> on the 43x77 pyramid level 0, radius 4 (8 edges)."""
    c = synth.make_corr_problem("frontend", seed=0, device=cuda, num_edges=8, dtype=torch.float32)
    f = c["fmaps"]
    f1 = f[c["ii"]].flatten(2) / 4.0
    f2 = f[c["jj"]].flatten(2) / 4.0
    H, W = f.shape[2:]
    vol = torch.matmul(f1.transpose(1, 2), f2).view(-1, H, W, H, W).contiguous()
    crd = c["coords"].permute(0, 3, 1, 2).contiguous()
    out, = droid_backends.corr_index_forward(vol, crd, 4)
    g = torch.randn_like(out)
    vg, = droid_backends.corr_index_backward(vol, crd, g, 4)
    lhs = (out.double() * g.double()).sum()
    rhs = (vol.double() * vg.double()).sum()
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_corr_index_vs_reference_kernels(cuda, ref_corr):
    if ref_corr is None:
        pytest.skip("oracle/_ref not built")
    for dtype, tol in ((torch.float32, 1e-5), (torch.float16, 2 ** -7)):
        vol, crd = make_lookup(3, 8, 9, 8, 9, seed=11, dev=cuda, dtype=dtype)
        out, = droid_backends.corr_index_forward(vol, crd, 3)
        ref, = ref_corr.corr_index_forward(vol, crd, 3)
        assert rel(np64(out), np64(ref)) < tol
        g = torch.randn(out.shape, device=cuda).to(dtype)
        vg, = droid_backends.corr_index_backward(vol, crd, g, 3)
        refg, = ref_corr.corr_index_backward(vol, crd, g, 3)
        assert rel(np64(vg), np64(refg)) < tol


def make_alt(B, N1, N2, C, H, W, M, seed, dev, dtype=torch.float32):
    g = torch.Generator().manual_seed(seed)
    f1 = torch.randn(B, N1, C, H, W, generator=g)
    f2 = torch.randn(B, N2, C, H, W, generator=g)
    ii = torch.randint(0, N1, (M,), generator=g)
    jj = torch.randint(0, N2, (M,), generator=g)
    crd = torch.stack([-2 + (W + 3) * torch.rand(B, M, H, W, generator=g),
                       -2 + (H + 3) * torch.rand(B, M, H, W, generator=g)], 2)
    return (f1.to(dev, dtype), f2.to(dev, dtype), crd.to(dev).contiguous(), ii.to(dev), jj.to(dev))


@pytest.mark.parametrize("r", [1, 3, 4])
def test_altcorr_vs_oracle(cuda, r):
    f1, f2, crd, ii, jj = make_alt(2, 3, 4, 16, 6, 7, 3, seed=r, dev=cuda)
    out, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, r)
    ref = oc.altcorr_forward(np64(f1), np64(f2), np64(crd), ii.cpu().numpy(), jj.cpu().numpy(), r)
    assert tuple(out.shape) == ref.shape
    assert rel(np64(out), ref) < 1e-5
    g = torch.randn(out.shape, device=cuda)
    for scale in (1.0, 1.0 / 16):
        g1, g2 = droid_backends.altcorr_backward(f1, f2, crd, ii, jj, g, r, scale)
        r1, r2 = oc.altcorr_backward(np64(f1), np64(f2), np64(crd), ii.cpu().numpy(), jj.cpu().numpy(),
                                     np64(g), r, scale=scale)
        assert rel(np64(g1), r1) < 1e-5 and rel(np64(g2), r2) < 1e-5


def test_altcorr_vs_reference_kernels(cuda, ref_corr):
    if ref_corr is None:
        pytest.skip("oracle/_ref not built")
    f1, f2, crd, ii, jj = make_alt(1, 4, 4, 32, 8, 9, 5, seed=5, dev=cuda)
    out, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, 3)
    ref, = ref_corr.altcorr_forward(f1, f2, crd, ii, jj, 3)
    assert rel(np64(out), np64(ref)) < 1e-5
    g = torch.randn(out.shape, device=cuda)
    g1, g2 = droid_backends.altcorr_backward(f1, f2, crd, ii, jj, g, 3)
    r1, r2 = ref_corr.altcorr_backward(f1, f2, crd, ii, jj, g, 3)
    assert rel(np64(g1), np64(r1)) < 1e-5 and rel(np64(g2), np64(r2)) < 1e-5


def test_altcorr_equals_volume_lookup_fp16(cuda):
    c = synth.make_corr_problem("frontend", seed=1, device=cuda, num_edges=6, dtype=torch.float16)
    f = c["fmaps"][None]
    crd = c["coords"].permute(0, 3, 1, 2)[None].contiguous()
    out, = droid_backends.altcorr_forward(f, f, crd, c["ii"], c["jj"], 4)
    H, W = f.shape[-2:]
    f1 = f[0, c["ii"]].float().flatten(2) / 4.0
    f2 = f[0, c["jj"]].float().flatten(2) / 4.0
    vol = torch.matmul(f1.transpose(1, 2), f2).view(-1, H, W, H, W).contiguous()
    ref, = droid_backends.corr_index_forward(vol, crd[0], 4)
    assert rel(np64(out[0]), np64(ref)) < 2 ** -8


def test_altcorr_bad_index_zero_filled(cuda):
    f1, f2, crd, ii, jj = make_alt(1, 3, 3, 8, 5, 5, 2, seed=9, dev=cuda)
    ii[1] = 7
    out, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, 2)
    assert torch.count_nonzero(out[:, 1]) == 0


def make_alt_levels(B, N1, N2, C, H, W, level, M, seed, dev, dtype):
    """fmap1 at H x W, fmap2 at level `level` (H >> level, W >> level), coords at that level's
    scale spread past the borders, ii/jj over the frames (one edge index out of range
    is not included here)."""
    g = torch.Generator().manual_seed(seed)
    H2, W2 = H >> level, W >> level
    f1 = (torch.randn(B, N1, C, H, W, generator=g) / np.sqrt(C)).to(dev, dtype)
    f2 = (torch.randn(B, N2, C, H2, W2, generator=g) / np.sqrt(C)).to(dev, dtype)
    ii = torch.randint(0, N1, (M,), generator=g).to(dev)
    jj = torch.randint(0, N2, (M,), generator=g).to(dev)
    crd = torch.stack([-3 + (W2 + 6) * torch.rand(B, M, H, W, generator=g),
                       -3 + (H2 + 6) * torch.rand(B, M, H, W, generator=g)], 2)
    return f1, f2, crd.to(dev).contiguous(), ii, jj


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16], ids=["f16", "bf16"])
@pytest.mark.parametrize("C,r,level", [(128, 3, 0), (128, 3, 2), (128, 4, 1), (32, 3, 0), (64, 2, 3), (256, 3, 1)])
def test_altcorr_packed_vs_oracle(cuda, dtype, C, r, level):
    """The channel-last path (exact products, FP32 sums) against the float64 oracle on
    the same 16-bit inputs: only the rounding of the stored output differs (2^-10
    relative for float16, 2^-7 for bfloat16), and against the direct kernel."""
    f1, f2, crd, ii, jj = make_alt_levels(1, 3, 5, C, 24, 40, level, 6, seed=C + r + level, dev=cuda, dtype=dtype)
    out, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, r)
    direct, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, r, path="direct")
    ref = oc.altcorr_forward(np64(f1), np64(f2), np64(crd), ii.cpu().numpy(), jj.cpu().numpy(), r)
    tol = 2 ** -10 if dtype == torch.float16 else 2 ** -7
    assert tuple(out.shape) == ref.shape
    assert rel(np64(out), ref) < tol
    assert rel(np64(out), np64(direct)) < tol


def test_altcorr_packed_frame_subsets_and_bad_index(cuda):
    """Only the frames of ii / jj are packed; an edge whose frame is out of range is
    zero-filled and reported, like the direct kernel."""
    f1, f2, crd, ii, jj = make_alt_levels(2, 6, 6, 128, 16, 24, 0, 4, seed=3, dev=cuda, dtype=torch.float16)
    ii = torch.tensor([5, 0, 5, 9], device=cuda)
    out, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, 3)
    good = [0, 1, 2]
    ref = oc.altcorr_forward(np64(f1), np64(f2), np64(crd[:, good]), ii[good].cpu().numpy(),
                             jj[good].cpu().numpy(), 3)
    assert rel(np64(out[:, good]), ref) < 2 ** -10
    assert torch.count_nonzero(out[:, 3]) == 0


def test_altcorr_packed_frontend_size(cuda):
    """43x77, 128 channels, radius 3, the four pooled levels of AltCorrBlock: the packed
    block (pyramid packed once) against CorrLayer on the direct kernel."""
    from hislam2_b200 import corr as hcorr
    c = synth.make_corr_problem("frontend", seed=2, device=cuda, num_edges=24, dtype=torch.float16)
    f = c["fmaps"][None].contiguous()
    coords = c["coords"][None].contiguous()
    blk = hcorr.AltCorrBlock(f, num_levels=4, radius=3)
    assert blk.packed is not None
    with torch.no_grad():
        fast = blk(coords, c["ii"], c["jj"])
    blk.packed = None
    with torch.no_grad():
        slow = blk(coords, c["ii"], c["jj"])
    assert fast.shape == slow.shape == (1, 24, 4 * 49, 43, 77)
    assert rel(np64(fast), np64(slow)) < 2 ** -10


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16], ids=["f16", "bf16"])
@pytest.mark.parametrize("level,r", [(0, 3), (1, 3), (0, 4), (2, 2)])
def test_altcorr_tiled_smooth_coords_vs_oracle(cuda, dtype, level, r):
    """Smooth coordinates (a scaled, shifted pixel grid plus 0.7 px of noise): 8x8 pixel
    blocks whose windows fit the staged box take the tensor-core path, including blocks
    whose windows cross the target's borders."""
    B, N, C, H, W = 1, 3, 128, 20, 30
    g = torch.Generator().manual_seed(40 + level + r)
    H2, W2 = H >> level, W >> level
    f1 = (torch.randn(B, N, C, H, W, generator=g) / np.sqrt(C)).to(cuda, dtype)
    f2 = (torch.randn(B, N, C, H2, W2, generator=g) / np.sqrt(C)).to(cuda, dtype)
    ii = torch.tensor([0, 1, 2, 1], device=cuda)
    jj = torch.tensor([1, 2, 0, 1], device=cuda)
    v, u = torch.meshgrid(torch.arange(H, dtype=torch.float32), torch.arange(W, dtype=torch.float32), indexing="ij")
    crd = []
    for e in range(4):
        sx, sy = 1.0 / 2 ** level, 1.0 / 2 ** level
        x = (u * sx + (e - 1.5) * 1.7) + 0.7 * torch.randn(H, W, generator=g)
        y = (v * sy - (e - 1.5) * 1.1) + 0.7 * torch.randn(H, W, generator=g)
        crd.append(torch.stack([x, y], 0))
    crd = torch.stack(crd, 0)[None].contiguous().to(cuda)
    out, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, r)
    ref = oc.altcorr_forward(np64(f1), np64(f2), np64(crd), ii.cpu().numpy(), jj.cpu().numpy(), r)
    tol = 2 ** -10 if dtype == torch.float16 else 2 ** -7
    assert rel(np64(out), ref) < tol
    direct, = droid_backends.altcorr_forward(f1, f2, crd, ii, jj, r, path="direct")
    assert rel(np64(out), np64(direct)) < tol


@pytest.mark.parametrize("dtype,tol", [(torch.float16, 2 ** -10), (torch.bfloat16, 2 ** -7)])
@pytest.mark.parametrize("r", [3, 4])
@pytest.mark.parametrize("integer_frac", [False, True])
def test_corr_index_16bit_odd_planes(cuda, dtype, tol, r, integer_frac):
    """16-bit volumes with odd plane sizes and an odd element count (windows starting at
    either parity, one on the volume's very last element, taps past every border) on the
    radius-3/4 kernel against the float32 path on the same values."""
    vol, crd = make_lookup(3, 5, 7, 7, 9, seed=20 + r, dev=cuda, dtype=dtype, integer_frac=integer_frac)
    assert vol.numel() % 2 == 1
    out, = droid_backends.corr_index_forward(vol, crd, r)
    ref32, = droid_backends.corr_index_forward(vol.float(), crd, r)
    assert rel(np64(out), np64(ref32)) < tol
    # a window on the very last element of the volume
    crd2 = crd.clone()
    crd2[-1, 0, -1, -1] = 8.3
    crd2[-1, 1, -1, -1] = 6.6
    out2, = droid_backends.corr_index_forward(vol, crd2, r)
    ref2, = droid_backends.corr_index_forward(vol.float(), crd2, r)
    assert rel(np64(out2), np64(ref2)) < tol
