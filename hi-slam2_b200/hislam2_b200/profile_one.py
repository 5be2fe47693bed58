"""Runs one BA call and one correlation lookup of a workload, for profilers.

    python -m hislam2_b200.profile_one [--workload backend300] [--iters 1] [--edges 64]

Kernels launched, in order: ba_keys, then per iteration ba_edge_setup,
ba_linearize, ba_assemble, ba_schur_tc (+ the SIMT Gram for very large frames),
ba_cholesky, ba_backsub, ba_pose_retr; then one corr_index_fwd (fp16 volume,
radius 4) over the first --edges edges of the frontend window.  Small enough for
an ncu capture (about 1 GB on the device).
"""

import argparse
import sys

import torch

from . import synth
from .backends import ba, corr_index_forward


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="backend300")
    ap.add_argument("--iters", type=int, default=1)
    ap.add_argument("--edges", type=int, default=64)
    a = ap.parse_args(argv)
    dev = torch.device("cuda:0")
    p = synth.make_ba_problem(a.workload, seed=0, device=dev)
    poses, disps = p["poses"].clone(), p["disps"].clone()
    ba(poses, disps, p["intrinsics"], p["targets"], p["weights"], p["eta"], p["ii"], p["jj"], p["t0"], p["t1"],
       a.iters, p["lm"], p["ep"], False)
    c = synth.make_corr_problem("frontend", seed=0, device=dev, num_edges=a.edges, dtype=torch.float16)
    f = c["fmaps"]
    H, W = f.shape[2:]
    vol = torch.matmul((f[c["ii"]].flatten(2) / 4).transpose(1, 2), f[c["jj"]].flatten(2) / 4)
    vol = vol.view(-1, H, W, H, W).contiguous()
    corr_index_forward(vol, c["coords"].permute(0, 3, 1, 2).contiguous(), 4)
    torch.cuda.synchronize()
    print("profile_one: done")
    return 0


if __name__ == "__main__":
    sys.exit(main())
