"""The B200 kernels against the reference's own operators.

Two sources of reference outputs:
  * the golden fixtures tests/golden/{ba,pgba,geo}_*.npz, made by
    tests/golden/make_golden_ba.py from HI-SLAM2's ``src/droid_kernels.cu`` run
    unmodified (oracle/_ref, Eigen replaced by the dense stand-in);
  * where oracle/_ref is built, the live reference operators on the same
    seeded inputs at the frontend window size (25 keyframes, 43x77, 258 edges,
    4 iterations), a 40-keyframe backend window, and the frontend window's
    4-level radius-4 correlation lookup (258 edges) in float32 and float16.
Tolerances: 1e-4 relative to the largest magnitude for poses, disparities, dx,
dz and the geometry outputs (the bar for the FP32 form); integer-valued counts
on all but boundary pixels; correlation lookups 1e-5 in float32 and 2e-3 in
float16 (the reference adds each bilinear term into a half-precision output in
place; ours accumulates the four terms in float32 and rounds once).
"""

import glob
import os

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import droid_backends
from hislam2_b200 import synth

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-4


def rel(a, b):
    a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.detach().double().cpu().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ba_*.npz"))),
                         ids=lambda f: os.path.basename(f)[:-4])
def test_ba_matches_reference_fixture(cuda, path):
    d = np.load(path)
    poses, disps = T(d["poses"], cuda), T(d["disps"], cuda)
    dx, dz, _ = droid_backends.ba(poses, disps, T(d["intrinsics"], cuda), T(d["targets"], cuda),
                                  T(d["weights"], cuda), T(d["eta"], cuda), T(d["ii"], cuda), T(d["jj"], cuda),
                                  int(d["t0"]), int(d["t1"]), int(d["iterations"]), float(d["lm"]),
                                  float(d["ep"]), bool(d["motion_only"]))
    assert rel(poses, d["out_poses"]) < RTOL
    assert rel(disps, d["out_disps"]) < RTOL
    assert rel(dx, d["dx"]) < 1e-3            # the last of three iterations: a converged update
    if bool(d["motion_only"]):
        assert dz is None
    else:
        assert rel(dz.reshape(d["dz"].shape), d["dz"]) < 1e-3


def test_pgba_matches_reference_fixture(cuda):
    d = np.load(os.path.join(GOLDEN, "pgba_tiny6.npz"))
    names = ("poses", "disps", "intrinsics", "targets", "weights", "eta", "Hsp", "vsp", "ii", "jj", "iip", "jjp")
    t = {k: T(d[k], cuda) for k in names}
    dx, dz = droid_backends.pgba(*(t[k] for k in names), int(d["t0"]), int(d["t1"]), float(d["lm"]),
                                 float(d["ep"]))
    assert rel(dx, d["dx"]) < RTOL
    assert rel(dz.reshape(d["dz"].shape), d["dz"]) < RTOL
    assert rel(t["disps"], d["out_disps"]) < RTOL


def test_geometry_matches_reference_fixtures(cuda):
    for name in ("geo_frame_distance_b03", "geo_frame_distance_b07"):
        d = np.load(os.path.join(GOLDEN, name + ".npz"))
        got = droid_backends.frame_distance(T(d["poses"], cuda), T(d["disps"], cuda), T(d["intrinsics"], cuda),
                                            T(d["ii"], cuda), T(d["jj"], cuda), float(d["beta"]))
        assert rel(got, d["dist"]) < RTOL
    d = np.load(os.path.join(GOLDEN, "geo_iproj.npz"))
    got = droid_backends.iproj(T(d["poses"], cuda), T(d["disps"], cuda), T(d["intrinsics"], cuda))
    assert rel(got, d["points"]) < RTOL
    d = np.load(os.path.join(GOLDEN, "geo_covis_distance.npz"))
    got = droid_backends.covis_distance(T(d["poses"], cuda), T(d["disps"], cuda), T(d["intrinsics"], cuda),
                                        T(d["ii"], cuda))
    HW = d["disps"].shape[1] * d["disps"].shape[2]
    assert np.abs(got.cpu().numpy() - d["dist"]).max() <= 1.0 / HW
    d = np.load(os.path.join(GOLDEN, "geo_depth_filter.npz"))
    got = droid_backends.depth_filter(T(d["poses"], cuda), T(d["disps"], cuda), T(d["intrinsics"], cuda),
                                      T(d["ix"], cuda), T(d["thresh"], cuda)).cpu().numpy()
    assert got.shape == d["counter"].shape and np.mean(got != d["counter"]) < 5e-3
    d = np.load(os.path.join(GOLDEN, "geo_proj_trans.npz"))
    C, w = droid_backends.proj_trans(T(d["poses"], cuda), T(d["disps"], cuda), T(d["intrinsics"][None], cuda),
                                     T(d["targets"], cuda), T(d["weights"], cuda), T(d["ii"], cuda),
                                     T(d["jj"], cuda))
    assert rel(C, d["C"]) < RTOL and rel(w, d["w"]) < RTOL
    d = np.load(os.path.join(GOLDEN, "geo_bi_inter.npz"))
    out, jac = droid_backends.bi_inter(T(d["scales"], cuda), T(d["grids"], cuda))
    assert rel(out, d["out"]) < 1e-5 and rel(jac, d["jac"]) < 1e-5


# ------------------------------------------------------------ live reference
def _need(ref_ops):
    if ref_ops is None:
        pytest.skip("oracle/_ref not built")


def _window(p, frames):
    m = (p["ii"] < frames) & (p["jj"] < frames)
    q = dict(p)
    for k in ("ii", "jj", "targets", "weights"):
        q[k] = p[k][m].contiguous()
    q["t1"] = frames
    q["eta"] = p["eta"][:frames].contiguous()
    return q


LIVE = {
    "frontend": lambda: synth.make_ba_problem("frontend", seed=1),
    "backend40": lambda: _window(synth.make_ba_problem("backend300", seed=2), 40),
}


def run_both(fn_ours, fn_ref, p, dev, iters, motion_only=False):
    q = {k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in p.items()}
    out = []
    for fn in (fn_ours, fn_ref):
        poses, disps = q["poses"].clone(), q["disps"].clone()
        dx, dz = fn(poses, disps, q["intrinsics"], q["targets"], q["weights"], q["eta"], q["ii"], q["jj"],
                    q["t0"], q["t1"], iters, q["lm"], q["ep"], motion_only)[:2]
        torch.cuda.synchronize()
        out.append((poses, disps, dx, dz))
    return out


@pytest.mark.parametrize("case", sorted(LIVE))
@pytest.mark.parametrize("motion_only", [False, True], ids=["full", "motion_only"])
def test_ba_matches_live_reference(cuda, ref_ops, case, motion_only):
    """Poses and disparities after the workload's iterations; dx and dz of a first
    iteration (those of a later, converged iteration are rounding noise)."""
    _need(ref_ops)
    p = LIVE[case]()
    (po, do, _, _), (pr, dr, _, _) = run_both(droid_backends.ba, ref_ops.ba, p, cuda, p["iters"], motion_only)
    assert rel(po, pr) < RTOL
    assert rel(do, dr) < RTOL
    (_, _, xo, zo), (_, _, xr, zr) = run_both(droid_backends.ba, ref_ops.ba, p, cuda, 1, motion_only)
    assert rel(xo, xr) < RTOL
    if not motion_only:
        assert rel(zo.reshape(zr.shape), zr) < RTOL


def test_frame_distance_matches_live_reference(cuda, ref_ops):
    _need(ref_ops)
    p = synth.make_ba_problem("frontend", seed=4)
    q = {k: (v.to(cuda) if torch.is_tensor(v) else v) for k, v in p.items()}
    args = (q["poses"], q["disps"], q["intrinsics"], q["ii"], q["jj"], 0.5)
    assert rel(droid_backends.frame_distance(*args), ref_ops.frame_distance(*args)) < RTOL


def frontend_pyramid(dev, dtype):
    """The frontend window's CorrBlock pyramid as the reference builds it
    (hislam2/modules/corr.py:29-38,63-71): matmul of the fmaps / 4, then avg_pool2d."""
    c = synth.make_corr_problem("frontend", seed=0, device=dev, dtype=dtype)
    f, ii, jj = c["fmaps"], c["ii"], c["jj"]
    E, (H, W) = ii.numel(), f.shape[2:]
    with torch.no_grad():
        vol = torch.matmul((f[ii].flatten(2) / 4.0).transpose(1, 2), f[jj].flatten(2) / 4.0)
        vol = vol.reshape(E * H * W, 1, H, W)
        pyr = []
        for lvl in range(4):
            pyr.append(vol.view(E, H, W, vol.shape[-2], vol.shape[-1]).contiguous())
            if lvl < 3:
                vol = F.avg_pool2d(vol, 2, stride=2)
    coords = c["coords"].permute(0, 3, 1, 2).contiguous()
    return pyr, coords, c["radius"]


def halves(n):
    return [(0, n // 2), (n // 2, n)]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16], ids=["f32", "f16"])
def test_corr_lookup_frontend_window_matches_live_reference(cuda, ref_ops, dtype):
    """258 edges, 43x77, radius 4, all four pyramid levels (coords / 2^level)."""
    _need(ref_ops)
    pyr, coords, r = frontend_pyramid(cuda, dtype)
    tol = 1e-5 if dtype == torch.float32 else 2e-3
    errs = []
    for lvl, vol in enumerate(pyr):
        crd = (coords / 2 ** lvl).contiguous()
        ours, = droid_backends.corr_index_forward(vol, crd, r)
        # the reference op indexes with 32-bit accessors: level 0 of 258 edges (2.8e9
        # elements) is fed to it in two halves
        ref = torch.cat([ref_ops.corr_index_forward(vol[a:b], crd[a:b], r)[0] for a, b in halves(vol.shape[0])])
        assert ours.shape == ref.shape == (vol.shape[0], 2 * r + 1, 2 * r + 1) + vol.shape[1:3]
        errs.append(rel(ours, ref))
        g = torch.randn(ours.shape, device=cuda, generator=torch.Generator(cuda).manual_seed(lvl)).to(dtype)
        vg_ours, = droid_backends.corr_index_backward(vol, crd, g, r)
        errs.append(max(rel(vg_ours[a:b], ref_ops.corr_index_backward(vol[a:b], crd[a:b], g[a:b], r)[0])
                        for a, b in halves(vol.shape[0])))
        del vg_ours
    print("corr lookup %s: max relative difference to the reference per level (fwd, bwd): %s"
          % (dtype, ["%.2e" % e for e in errs]))
    assert max(errs) < tol, errs
