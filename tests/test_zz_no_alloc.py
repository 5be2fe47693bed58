"""The allocation-free BA entry point (hs2_ba_noalloc) against the regular one.

hs2_ba_noalloc serves callers that cannot allocate device memory when they run a
BA step -- a process whose GPU memory budget is fixed at start-up, or a host in
another language without a caching allocator, for which cudaMalloc / cudaFree in
its loop would stall the device.  It takes its scratch from a 64 MiB static device array inside the
library instead of a caller workspace.  This test calls it through the C ABI on
two problems in a row (so the second call runs on the scratch the first one left
behind) and compares poses, disparities, dx and dz with droid_backends.ba, within
the 1e-4 relative tolerance of the other BA tests; a problem that needs more than
64 MiB of scratch must be refused with a clear error.
"""

import ctypes

import numpy as np
import pytest
import torch

import droid_backends
from hislam2_b200 import _lib, synth

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def rel(a, b):
    a = a.detach().double().cpu().numpy()
    b = b.detach().double().cpu().numpy()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else ctypes.c_void_p(0)


def call_noalloc(q, poses, disps, iters):
    ht, wd = disps.shape[1:]
    P = q["t1"] - q["t0"]
    S = max(1, min(poses.shape[0], P + q["ii"].numel()))
    dx = torch.zeros(P, 6, device=poses.device)
    dz = torch.zeros(S, ht * wd, device=poses.device)
    info = torch.zeros(4, dtype=torch.int32, device=poses.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(poses.device).cuda_stream)
    rc = _lib.load().hs2_ba_noalloc(ptr(poses), poses.shape[0], ptr(disps), disps.shape[0], ht, wd,
                                    ptr(q["intrinsics"]), ptr(q["targets"]), ptr(q["weights"]), ptr(q["eta"]),
                                    q["eta"].shape[0], ptr(q["ii"]), ptr(q["jj"]), q["ii"].numel(), q["t0"],
                                    q["t1"], iters, q["lm"], q["ep"], 0, ptr(dx), ptr(dz), S, ptr(info), stream)
    return rc, dx, dz, info


def test_noalloc_matches_regular_entry_point(cuda):
    for name, seed in (("frontend", 5), ("frontend_small", 6)):
        p = synth.make_ba_problem(name, seed=seed)
        q = {k: (v.to(cuda) if torch.is_tensor(v) else v) for k, v in p.items()}
        poses_a, disps_a = q["poses"].clone(), q["disps"].clone()
        rc, dx_a, dz_a, info = call_noalloc(q, poses_a, disps_a, q["iters"])
        torch.cuda.synchronize()
        assert rc == _lib.HS2_OK, _lib.load().hs2_last_error()
        h = info.cpu()
        assert int(h[0]) == 0 and int(h[2]) == 0
        M = int(h[1])
        poses_b, disps_b = q["poses"].clone(), q["disps"].clone()
        dx_b, dz_b, _ = droid_backends.ba(poses_b, disps_b, q["intrinsics"], q["targets"], q["weights"], q["eta"],
                                          q["ii"], q["jj"], q["t0"], q["t1"], q["iters"], q["lm"], q["ep"], False)
        torch.cuda.synchronize()
        assert M == dz_b.shape[0]
        assert rel(poses_a, poses_b) < RTOL
        assert rel(disps_a, disps_b) < RTOL
        assert rel(dx_a, dx_b) < RTOL
        assert rel(dz_a[:M], dz_b) < RTOL


def test_noalloc_rejects_problems_beyond_its_scratch(cuda):
    p = synth.make_ba_problem("backend300", seed=0)
    q = {k: (v.to(cuda) if torch.is_tensor(v) else v) for k, v in p.items()}
    poses, disps = q["poses"].clone(), q["disps"].clone()
    rc, _, _, _ = call_noalloc(q, poses, disps, 1)
    assert rc == _lib.HS2_ERR_WORKSPACE
    assert b"allocation-free" in _lib.load().hs2_last_error()
    torch.cuda.synchronize()
    assert torch.equal(poses, q["poses"]) and torch.equal(disps, q["disps"])
