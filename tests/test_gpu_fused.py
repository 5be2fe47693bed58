"""corr_reproject_lookup (reprojection + 4-level lookup in one launch) against the
unfused chain it replaces: the reprojection of hislam2_b200.synth.reproject (float64,
the same formula as the reference's projective_transform), then altcorr_forward per
level at coords / 2^level, and against the float64 oracle of CorrBlock's lookup.

Tolerances: coordinates within 2e-3 px of the float64 reprojection (float32
arithmetic); the lookup 1e-5 relative to altcorr_forward fed with the kernel's own
coordinates (the same arithmetic) in float32, and 1e-4 (float32) / 2e-3 (float16)
relative to the oracle.
"""

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import oracle
from hislam2_b200 import backends, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.detach().double().cpu().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def levels_of(f, L=4):
    out = [f]
    for _ in range(1, L):
        out.append(F.avg_pool2d(out[-1], 2, stride=2))
    return [x.contiguous() for x in out]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16], ids=["f32", "f16"])
def test_fused_lookup_matches_unfused_chain(cuda, dtype):
    p = synth.make_ba_problem("frontend", seed=1)
    c = synth.make_corr_problem("frontend", seed=1, device=cuda, dtype=dtype)
    ii, jj, r = c["ii"], c["jj"], c["radius"]
    pyr = levels_of(c["fmaps"])
    poses, disps, intr = p["poses"].to(cuda), p["disps"].to(cuda), p["intrinsics"].to(cuda)
    corr, coords = backends.corr_reproject_lookup(pyr, poses, disps, intr, ii, jj, r)
    ref_coords = synth.reproject(p["poses"], p["disps"], p["intrinsics"], ii.cpu(), jj.cpu())
    assert float((coords.double().cpu() - ref_coords).abs().max()) < 2e-3
    E, H, W = ii.numel(), 43, 77
    rd2 = (2 * r + 1) ** 2
    crd = coords.permute(0, 3, 1, 2).contiguous()[None]
    for lvl in range(4):
        alt, = backends.altcorr_forward(pyr[0][None], pyr[lvl][None], (crd / 2 ** lvl).contiguous(), ii, jj, r)
        got = corr[:, lvl * rd2:(lvl + 1) * rd2].reshape(alt.shape)
        tol = 1e-5 if dtype == torch.float32 else 2e-3
        assert rel(got, alt) < tol, (lvl, rel(got, alt))
    # the CorrBlock semantics on a few edges (float64 oracle of the pooled-volume lookup)
    k = [0, 7, 131]
    f1 = c["fmaps"][ii[k]].double().cpu().numpy()[None]
    f2 = c["fmaps"][jj[k]].double().cpu().numpy()[None]
    ref = oracle.corr.corr_block_lookup(oracle.corr.pyramid(f1, f2, 4), coords[k].double().cpu().numpy()[None], r)
    tol = 1e-4 if dtype == torch.float32 else 2e-3
    assert rel(corr[k], ref[0]) < tol


def test_fused_lookup_without_coords_and_bad_index(cuda):
    p = synth.make_ba_problem("frontend_small", seed=0)
    c = synth.make_corr_problem("frontend_small", seed=0, device=cuda, dtype=torch.float32)
    pyr = levels_of(c["fmaps"])
    args = (pyr, p["poses"].to(cuda), p["disps"].to(cuda), p["intrinsics"].to(cuda))
    corr = backends.corr_reproject_lookup(*args, c["ii"], c["jj"], 3, return_coords=False)
    assert corr.shape == (c["ii"].numel(), 4 * 49, 48, 64)
    # an edge outside the frame buffers is reported, like the other ops
    bad = c["jj"].clone()
    bad[0] = 99
    corr_bad, _ = backends.corr_reproject_lookup(*args, c["ii"], bad, 3)
    torch.cuda.synchronize()
    assert float(corr_bad[0].abs().max()) == 0.0


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16], ids=["f16", "bf16"])
def test_fused_packed_path_matches_direct_kernel(cuda, dtype):
    """16-bit features with 128 channels take the channel-last tensor-core path (8x8-pixel
    blocks, reprojection in the kernel); it matches the per-tap kernel (only the summation
    order differs before the output is rounded) and reports an out-of-range edge the same way."""
    p = synth.make_ba_problem("frontend", seed=2)
    c = synth.make_corr_problem("frontend", seed=2, device=cuda, dtype=dtype)
    pyr = levels_of(c["fmaps"])
    args = (pyr, p["poses"].to(cuda), p["disps"].to(cuda), p["intrinsics"].to(cuda))
    ii, jj = c["ii"][:40], c["jj"][:40].clone()
    fast, cf = backends.corr_reproject_lookup(*args, ii, jj, 3)
    slow, cs = backends.corr_reproject_lookup(*args, ii, jj, 3, path="direct")
    assert float((cf - cs).abs().max()) < 1e-4
    tol = 2 ** -10 if dtype == torch.float16 else 2 ** -7
    assert rel(fast, slow) < tol
    jj[5] = 1000
    bad, _ = backends.corr_reproject_lookup(*args, ii, jj, 3)
    torch.cuda.synchronize()
    assert float(bad[5].float().abs().max()) == 0.0
    assert rel(bad[:5], fast[:5]) < tol
