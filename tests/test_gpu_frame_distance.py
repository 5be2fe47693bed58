"""frame_distance on the B200 kernel against the float64 oracle."""

import numpy as np
import pytest
import torch

import droid_backends
from hislam2_b200 import synth
from oracle import frame_distance as ofd

pytestmark = pytest.mark.gpu


def test_frame_distance_matrix_vs_oracle(cuda):
    p = synth.make_ba_problem("frontend", seed=4)
    K = p["poses"].shape[0]
    ii, jj = torch.meshgrid(torch.arange(K), torch.arange(K), indexing="ij")
    ii, jj = ii.reshape(-1), jj.reshape(-1)
    d = droid_backends.frame_distance(p["poses"].to(cuda), p["disps"].to(cuda), p["intrinsics"].to(cuda),
                                      ii.to(cuda), jj.to(cuda), 0.3)
    ref = ofd.frame_distance(p["poses"].double().numpy(), p["disps"].double().numpy(),
                             p["intrinsics"].double().numpy(), ii.numpy(), jj.numpy(), 0.3)
    got = d.cpu().double().numpy()
    far = ref >= 1000
    assert np.array_equal(got >= 1000, far)
    np.testing.assert_allclose(got[~far], ref[~far], rtol=1e-4, atol=1e-5)


def test_frame_distance_invalid_fraction_and_bad_index(cuda):
    p = synth.make_ba_problem("frontend_small", seed=0)
    poses = p["poses"].clone()
    poses[1, 2] = -10.0
    ii = torch.tensor([0, 2], device=cuda)
    jj = torch.tensor([1, 3], device=cuda)
    d = droid_backends.frame_distance(poses.to(cuda), p["disps"].to(cuda), p["intrinsics"].to(cuda), ii, jj, 0.3)
    assert d[0].item() == 1000.0 and d[1].item() < 1000.0
    with pytest.raises(RuntimeError, match="out of range"):
        droid_backends.frame_distance(poses.to(cuda), p["disps"].to(cuda), p["intrinsics"].to(cuda),
                                      torch.tensor([0, 99], device=cuda), jj, 0.3)
    empty = torch.zeros(0, dtype=torch.long, device=cuda)
    assert droid_backends.frame_distance(poses.to(cuda), p["disps"].to(cuda), p["intrinsics"].to(cuda),
                                         empty, empty, 0.3).numel() == 0
