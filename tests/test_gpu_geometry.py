"""iproj / covis_distance / depth_filter kernels against the float64 oracle (the kernels work
in float32, so counts may differ where a pixel sits on a comparison boundary)."""

import numpy as np
import pytest
import torch

import droid_backends
import oracle
from hislam2_b200 import synth

pytestmark = pytest.mark.gpu


def _buffer(cuda, K=12, seed=0, motion=1.0):
    p = synth.make_ba_problem("frontend", seed=seed)
    poses = p["poses"][:K].clone()
    poses[:, :3] *= motion
    disps = p["disps"][:K].clone()
    return poses.to(cuda), disps.to(cuda), p["intrinsics"].to(cuda)


def test_iproj_matches_oracle(cuda):
    poses, disps, intr = _buffer(cuda)
    got = droid_backends.iproj(poses, disps, intr)
    ref = oracle.geometry.iproj(poses.cpu().numpy(), disps.cpu().numpy(), intr.cpu().numpy())
    assert got.shape == (12,) + disps.shape[1:] + (3,)
    np.testing.assert_allclose(got.cpu().numpy(), ref, rtol=2e-5, atol=2e-5)


@pytest.mark.parametrize("motion", [1.0, 30.0])
def test_covis_distance_matches_oracle(cuda, motion):
    poses, disps, intr = _buffer(cuda, motion=motion)
    ii = torch.arange(1, 11, device=cuda)
    got = droid_backends.covis_distance(poses, disps, intr, ii).cpu().numpy()
    ref = oracle.geometry.covis_distance(poses.cpu().numpy(), disps.cpu().numpy(), intr.cpu().numpy(),
                                         ii.cpu().numpy())
    HW = disps.shape[1] * disps.shape[2]
    assert np.abs(got - ref).max() <= 3.0 / HW
    if motion > 1:
        assert ref.max() > 0


def test_covis_distance_rejects_edge_frames(cuda):
    poses, disps, intr = _buffer(cuda)
    for bad in (0, 11):
        with pytest.raises(RuntimeError, match="neighbours"):
            droid_backends.covis_distance(poses, disps, intr, torch.tensor([bad], device=cuda))


def test_depth_filter_matches_oracle(cuda):
    poses, disps, intr = _buffer(cuda)
    disps[:] = disps[0:1].clone()
    ix = torch.tensor([0, 2, 5, 9, 11], device=cuda)        # neighbours clipped at both ends
    thresh = torch.full((5,), 0.05, device=cuda)
    got = droid_backends.depth_filter(poses, disps, intr, ix, thresh).cpu().numpy()
    ref = oracle.geometry.depth_filter(poses.cpu().numpy(), disps.cpu().numpy(), intr.cpu().numpy(),
                                       ix.cpu().numpy(), thresh.cpu().numpy())
    assert got.shape == ref.shape
    assert (got == np.round(got)).all() and got.max() <= 6
    assert np.mean(got != ref) < 2e-3, np.mean(got != ref)
    assert ref.max() >= 2


def test_depth_filter_rejects_bad_index(cuda):
    poses, disps, intr = _buffer(cuda)
    with pytest.raises(RuntimeError, match="ix outside"):
        droid_backends.depth_filter(poses, disps, intr, torch.tensor([12], device=cuda),
                                    torch.ones(1, device=cuda))


def test_proj_trans_matches_oracle(cuda):
    p = synth.make_ba_problem("frontend", seed=3)
    q = {k: (v.to(cuda) if torch.is_tensor(v) else v) for k, v in p.items()}
    intr2 = q["intrinsics"][None].contiguous()
    C, w = droid_backends.proj_trans(q["poses"], q["disps"], intr2, q["targets"], q["weights"], q["ii"], q["jj"])
    Co, wo = oracle.geometry.proj_trans(p["poses"].numpy(), p["disps"].numpy(), p["intrinsics"].numpy(),
                                        p["targets"].numpy(), p["weights"].numpy(), p["ii"].numpy(), p["jj"].numpy())
    assert C.shape == Co.shape
    for got, ref in ((C, Co), (w, wo)):
        got = got.double().cpu().numpy()
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 1e-5, err


def test_bi_inter_matches_oracle(cuda):
    g = torch.Generator().manual_seed(5)
    M, ht, wd, hs, ws = 3, 43, 77, 6, 8
    scales = (0.5 + torch.rand(M, hs, ws, generator=g)).to(cuda)
    mx, my = torch.meshgrid(torch.linspace(0, hs - 1 - 1e-6, ht), torch.linspace(0, ws - 1 - 1e-6, wd), indexing="ij")
    grids = torch.stack((my, mx), -1)[None].expand(M, -1, -1, -1).contiguous().to(cuda)
    out, jac = droid_backends.bi_inter(scales, grids)
    ro, rj = oracle.geometry.bi_inter(scales.cpu().numpy(), grids.cpu().numpy())
    np.testing.assert_allclose(out.cpu().numpy(), ro, rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(jac.cpu().numpy(), rj, rtol=2e-6, atol=2e-6)
    bad = grids.clone()
    bad[0, 0, 0, 0] = ws - 1.0                     # cell would leave the grid
    with pytest.raises(RuntimeError, match="leaves the scale grid"):
        droid_backends.bi_inter(scales, bad)
