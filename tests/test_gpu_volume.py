"""corr_volume (tcgen05 all-pairs volume + fused pooling pyramid) against the float64
oracle (oracle.corr.pyramid), against the PyTorch construction HI-SLAM2's CorrBlock
uses (torch.matmul + F.avg_pool2d, hislam2/modules/corr.py:29-38,63-71), and
against itself: every pooled level must equal F.avg_pool2d of the kernel's own
level above bit for bit (same rounding, same summation order).

Tolerances, relative to the largest magnitude of the float64 oracle level:
float16 2e-3, bfloat16 1.6e-2 (one rounding of the F32 sum to the volume type,
plus the pooled levels' roundings); the FP8 e4m3 form is a different arithmetic
(3-bit mantissa features with one scale per pixel): its RMS error is checked
against 6% of the RMS value and its largest error against 12% of the largest
magnitude.  Against torch.matmul + avg_pool2d (the same inputs, cuBLAS with F32
accumulation) level 0 agrees within 2 units in the last place of float16.
"""

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import oracle
from hislam2_b200 import backends, synth

pytestmark = pytest.mark.gpu


def fmaps(K, H, W, dtype, dev, seed=0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(K, 128, H, W, generator=g) / np.sqrt(128.0)).to(dtype).to(dev)


def oracle_levels(f1, f2, ii, jj, L):
    a = f1[ii].float().cpu().numpy()[None]
    b = f2[jj].float().cpu().numpy()[None]
    return oracle.corr.pyramid(a, b, L)


def rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else a
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def check_pooling_exact(pyr):
    for l in range(1, len(pyr)):
        E, H, W, h, w = pyr[l - 1].shape
        if pyr[l].numel() == 0:
            continue
        ref = F.avg_pool2d(pyr[l - 1].reshape(E * H * W, 1, h, w), 2, stride=2)
        assert torch.equal(ref.reshape(pyr[l].shape), pyr[l]), "level %d" % l


@pytest.mark.parametrize("dtype,tol", [(torch.float16, 2e-3), (torch.bfloat16, 1.6e-2)], ids=["f16", "bf16"])
@pytest.mark.parametrize("H,W", [(43, 77), (48, 64), (12, 96), (5, 7)], ids=["43x77", "48x64", "12x96", "5x7"])
def test_volume_matches_oracle_and_pools_exactly(cuda, dtype, tol, H, W):
    f = fmaps(4, H, W, dtype, cuda)
    ii = torch.tensor([0, 1, 2, 3, 1], device=cuda)
    jj = torch.tensor([1, 2, 3, 0, 1], device=cuda)
    pyr = backends.corr_volume(f, f, ii, jj)
    torch.cuda.synchronize()
    ref = oracle_levels(f, f, ii.cpu(), jj.cpu(), 4)
    for l in range(4):
        assert tuple(pyr[l].shape) == ref[l].shape
        if ref[l].size:
            assert rel(pyr[l], ref[l]) < tol, (l, rel(pyr[l], ref[l]))
    check_pooling_exact(pyr)


def test_volume_matches_torch_corrblock_construction(cuda):
    """The frontend window (258 edges, 43x77, float16) against torch.matmul + avg_pool2d."""
    c = synth.make_corr_problem("frontend", seed=0, device=cuda, dtype=torch.float16)
    f, ii, jj = c["fmaps"], c["ii"], c["jj"]
    E, (H, W) = ii.numel(), f.shape[2:]
    pyr = backends.corr_volume(f, f, ii, jj)
    with torch.no_grad():
        vol = torch.matmul((f[ii].flatten(2) / 4.0).transpose(1, 2), f[jj].flatten(2) / 4.0)
    ours = pyr[0].reshape(E, H * W, H * W)
    ulp = torch.finfo(torch.float16).eps * vol.abs().float().clamp_min(2.0 ** -14)
    assert ((ours.float() - vol.float()).abs() <= 2 * ulp).all()
    del vol, ours
    check_pooling_exact(pyr)


def test_volume_gathered_pairs_and_fewer_levels(cuda):
    """CorrBlock's own call: fmap1/fmap2 already gathered per pair, [B,N,C,H,W]."""
    f = fmaps(6, 43, 77, torch.float16, cuda, seed=3)
    a, b = f[None, :3], f[None, 3:]
    pyr = backends.corr_volume(a, b, num_levels=2)
    assert len(pyr) == 2 and pyr[1].shape == (3, 43, 77, 21, 38)
    ref = oracle.corr.pyramid(a.float().cpu().numpy(), b.float().cpu().numpy(), 2)
    assert rel(pyr[0], ref[0]) < 2e-3 and rel(pyr[1], ref[1]) < 2e-3


def test_volume_fp8_error(cuda):
    f = fmaps(4, 43, 77, torch.float16, cuda, seed=1)
    ii = torch.tensor([0, 1, 2, 3], device=cuda)
    jj = torch.tensor([1, 2, 3, 0], device=cuda)
    pyr = backends.corr_volume(f, f, ii, jj, precision="e4m3")
    ref = oracle_levels(f, f, ii.cpu(), jj.cpu(), 4)
    for l in range(4):
        d = pyr[l].double().cpu().numpy() - ref[l]
        rms = np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(ref[l] ** 2))
        mx = np.abs(d).max() / np.abs(ref[l]).max()
        print("e4m3 level %d: rms rel err %.3e, max rel err %.3e" % (l, rms, mx))
        assert rms < 0.06 and mx < 0.12, (l, rms, mx)
    check_pooling_exact(pyr)


def test_volume_edge_cases(cuda):
    f = fmaps(2, 43, 77, torch.float16, cuda)
    empty = torch.zeros(0, dtype=torch.int64, device=cuda)
    pyr = backends.corr_volume(f, f, empty, empty)
    assert [p.shape[0] for p in pyr] == [0, 0, 0, 0]
    with pytest.raises(RuntimeError, match="out of range"):
        backends.corr_volume(f, f, torch.tensor([0, 2], device=cuda), torch.tensor([1, 1], device=cuda))
    with pytest.raises(RuntimeError, match="128"):
        backends.corr_volume(f[:, :64].contiguous(), f[:, :64].contiguous())
    with pytest.raises(RuntimeError, match="W=100"):
        g = fmaps(2, 8, 100, torch.float16, cuda)
        backends.corr_volume(g, g)
    with pytest.raises(RuntimeError, match="dtype"):
        backends.corr_volume(f.float(), f.float())


def test_volume_repeated_calls_are_deterministic(cuda):
    f = fmaps(3, 43, 77, torch.bfloat16, cuda, seed=2)
    ii = torch.tensor([0, 1, 2], device=cuda)
    jj = torch.tensor([2, 0, 1], device=cuda)
    a = backends.corr_volume(f, f, ii, jj)
    b = backends.corr_volume(f, f, ii, jj)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
