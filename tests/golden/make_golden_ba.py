"""Generates tests/golden/{ba,pgba,geo}_*.npz: outputs of the reference's own BA-family
operators (HI-SLAM2 ``src/droid_kernels.cu`` through its binding ``src/droid.cpp``).

TEST INFRASTRUCTURE.  Needs a CUDA GPU and ``oracle/_ref`` (built by
``oracle/build_ref.py``: the reference sources compiled unmodified, with the
self-written dense stand-in for the Eigen facilities they include).  Inputs are
the seeded ``tiny6`` / ``tiny7`` problems of ``hislam2_b200.synth`` (a few
hundred kB) and are stored beside the reference's outputs, so
``tests/test_golden_ba.py`` checks the float64 oracle against the reference
without a GPU and without regenerating anything.

Usage: ``python tests/golden/make_golden_ba.py [outdir]``.
"""

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "hi-slam2_b200")]

from hislam2_b200 import synth  # noqa: E402
from oracle import build_ref  # noqa: E402

BA_KEYS = ("poses", "disps", "intrinsics", "targets", "weights", "eta", "ii", "jj")


def num_depth_frames(ii, t0, t1):
    return len(np.unique(np.concatenate([np.arange(t0, t1), ii.numpy()])))


def ba_case(ref, dev, name, t0=None, motion_only=False, eta_rows=None):
    p = synth.make_ba_problem(name, seed=0)
    t0 = p["t0"] if t0 is None else t0
    t1 = p["t1"]
    M = num_depth_frames(p["ii"], t0, t1)
    eta = p["eta"][: (M if eta_rows is None else eta_rows)].contiguous()
    inputs = {k: p[k] for k in BA_KEYS}
    inputs["eta"] = eta
    d = {k: v.to(dev) for k, v in inputs.items()}
    dx, dz, _ = ref.ba(d["poses"], d["disps"], d["intrinsics"], d["targets"], d["weights"], d["eta"], d["ii"],
                       d["jj"], t0, t1, p["iters"], p["lm"], p["ep"], motion_only)
    torch.cuda.synchronize()
    out = {k: v.numpy() for k, v in inputs.items()}
    out.update(t0=np.int64(t0), t1=np.int64(t1), iterations=np.int64(p["iters"]), lm=np.float64(p["lm"]),
               ep=np.float64(p["ep"]), motion_only=np.bool_(motion_only),
               out_poses=d["poses"].cpu().numpy(), out_disps=d["disps"].cpu().numpy(), dx=dx.cpu().numpy())
    if dz is not None:
        out["dz"] = dz.cpu().numpy()
    return out


def pgba_case(ref, dev, name):
    g = synth.make_pgba_problem(name, seed=0)
    M = num_depth_frames(g["ii"], g["t0"], g["t1"])
    g["eta"] = g["eta"][:M].contiguous()
    keys = ("poses", "disps", "intrinsics", "targets", "weights", "eta", "Hsp", "vsp", "ii", "jj", "iip", "jjp")
    d = {k: g[k].to(dev) for k in keys}
    dx, dz = ref.pgba(*(d[k] for k in keys), g["t0"], g["t1"], g["lm"], g["ep"])[:2]
    torch.cuda.synchronize()
    out = {k: g[k].numpy() for k in keys}
    out.update(t0=np.int64(g["t0"]), t1=np.int64(g["t1"]), lm=np.float64(g["lm"]), ep=np.float64(g["ep"]),
               out_poses=d["poses"].cpu().numpy(), out_disps=d["disps"].cpu().numpy(), dx=dx.cpu().numpy(),
               dz=dz.cpu().numpy())
    return out


def geometry_cases(ref, dev):
    p = synth.make_ba_problem("tiny6", seed=1)
    poses, disps, intr = p["poses"], p["disps"], p["intrinsics"]
    ii, jj = p["ii"], p["jj"]
    D = lambda t: t.to(dev)  # noqa: E731
    cases = {}
    for beta in (0.3, 0.7):
        dist = ref.frame_distance(D(poses), D(disps), D(intr), D(ii), D(jj), beta)
        cases["geo_frame_distance_b%02d" % int(beta * 10)] = dict(
            poses=poses.numpy(), disps=disps.numpy(), intrinsics=intr.numpy(), ii=ii.numpy(), jj=jj.numpy(),
            beta=np.float64(beta), dist=dist.cpu().numpy())
    pts = ref.iproj(D(poses), D(disps), D(intr))
    cases["geo_iproj"] = dict(poses=poses.numpy(), disps=disps.numpy(), intrinsics=intr.numpy(),
                              points=pts.cpu().numpy())
    ix = torch.arange(1, 5)
    cov = ref.covis_distance(D(poses), D(disps), D(intr), D(ix))
    cases["geo_covis_distance"] = dict(poses=poses.numpy(), disps=disps.numpy(), intrinsics=intr.numpy(),
                                       ii=ix.numpy(), dist=cov.cpu().numpy())
    same = disps[0:1].expand_as(disps).contiguous()
    ixf = torch.tensor([0, 2, 3, 5])
    thresh = torch.full((4,), 0.05)
    cnt = ref.depth_filter(D(poses), D(same), D(intr), D(ixf), D(thresh))
    cases["geo_depth_filter"] = dict(poses=poses.numpy(), disps=same.numpy(), intrinsics=intr.numpy(),
                                     ix=ixf.numpy(), thresh=thresh.numpy(), counter=cnt.cpu().numpy())
    intr2 = intr[None].contiguous()
    C, w = ref.proj_trans(D(poses), D(disps), D(intr2), D(p["targets"]), D(p["weights"]), D(ii), D(jj))
    cases["geo_proj_trans"] = dict(poses=poses.numpy(), disps=disps.numpy(), intrinsics=intr.numpy(),
                                   targets=p["targets"].numpy(), weights=p["weights"].numpy(), ii=ii.numpy(),
                                   jj=jj.numpy(), C=C.cpu().numpy(), w=w.cpu().numpy())
    g = torch.Generator().manual_seed(7)
    M, ht, wd, hs, ws = 2, 9, 11, 3, 4
    scales = 0.5 + torch.rand(M, hs, ws, generator=g)
    my, mx = torch.meshgrid(torch.linspace(0, hs - 1 - 1e-3, ht), torch.linspace(0, ws - 1 - 1e-3, wd),
                            indexing="ij")
    grids = torch.stack((mx, my), -1)[None].expand(M, -1, -1, -1).contiguous()
    out, jac = ref.bi_inter(D(scales), D(grids))
    cases["geo_bi_inter"] = dict(scales=scales.numpy(), grids=grids.numpy(), out=out.cpu().numpy(),
                                 jac=jac.cpu().numpy())
    return cases


def main(outdir=HERE):
    ref = build_ref.load()
    if ref is None:
        raise SystemExit("oracle/_ref is not built (python oracle/build_ref.py)")
    dev = torch.device("cuda:0")
    cases = {
        "ba_tiny6_t0_2": ba_case(ref, dev, "tiny6"),
        "ba_tiny6_t0_0": ba_case(ref, dev, "tiny6", t0=0),
        "ba_tiny6_motion_only": ba_case(ref, dev, "tiny6", motion_only=True),
        "ba_tiny6_eta_one_row": ba_case(ref, dev, "tiny6", eta_rows=1),
        "ba_tiny7_window": ba_case(ref, dev, "tiny7"),
        "pgba_tiny6": pgba_case(ref, dev, "tiny6"),
    }
    cases.update(geometry_cases(ref, dev))
    os.makedirs(outdir, exist_ok=True)
    for name, arrays in cases.items():
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **arrays)
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
