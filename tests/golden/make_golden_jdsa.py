"""Generates tests/golden/jdsa_*.npz: outputs of the reference's own mono-prior alignment
step, HI-SLAM2 ``hislam2/geom/ba.py:JDSA`` (with ``geom/chol.py:schur_solve_mono_prior``).

TEST INFRASTRUCTURE.  Runs on the CPU, in float32 as the reference does, by importing the
reference's ``geom`` package unmodified from the checkout (``$HISLAM2_REFERENCE``, else
the default of ``oracle/build_ref.py``) with three modules it imports supplied here:

* ``droid_backends``: ``proj_trans`` and ``bi_inter`` from ``oracle.geometry`` (the float64
  restatement that ``tests/test_golden_ba.py`` pins to the reference's compiled kernels
  through ``geo_proj_trans.npz`` / ``geo_bi_inter.npz``), returned as float32 tensors;
* ``torch_scatter.scatter_sum``: its published semantics (sum of ``src`` slices into
  ``dim_size`` rows of ``dim`` by ``index``), written with ``index_add_``;
* ``lietorch``: a holder whose ``.data`` is the pose tensor -- JDSA reads nothing else.

``Tensor.cuda`` is made the identity while JDSA runs, so the reference's ``.cuda()``
calls stay on the CPU.  Inputs come from ``hislam2_b200.synth.make_jdsa_problem`` and
are stored beside the outputs, so ``tests/test_golden_jdsa.py`` checks the float64
oracle (``oracle/jdsa.py``) without regenerating anything.

Usage: ``python tests/golden/make_golden_jdsa.py [outdir]``.
"""

import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "hi-slam2_b200")]

from hislam2_b200 import synth  # noqa: E402
from oracle import build_ref, geometry  # noqa: E402

CASES = {
    # the HI-SLAM2 configuration: a 2x2 scale grid per frame, mono_depth_alpha 0.01
    "jdsa_tiny6_2x2": dict(name="tiny6", hs=2, ws=2, alpha=0.01),
    # a finer 3x4 grid (several interpolation cells), alpha 0.001 (the Replica config)
    "jdsa_tiny6_3x4": dict(name="tiny6", hs=3, ws=4, alpha=0.001),
    # a 4x4 grid: 16 scale unknowns per frame, the most the kernel takes
    "jdsa_tiny6_4x4": dict(name="tiny6", hs=4, ws=4, alpha=0.01),
    # source frames {0, 1, 3, 4, 5}: keys kx - kx[0] skip 2, so one block gets no prior
    # terms, key 5 is dropped by safe_scatter_add_mat, and blocks 3 and 4 pair the prior
    # terms of frames 3 and 4 with the rows (C, w, mask) of frames 4 and 5.  A prior on
    # every pixel keeps each block positive definite.
    "jdsa_tiny6_gap": dict(name="tiny6", hs=2, ws=2, alpha=0.01, keep=lambda i: i != 2, holes=0.0),
    # the same with 10% prior holes: a block pairs a prior pixel (J != 0) with a hole of
    # the other frame (Q = 1/(C + eta), large), its Schur complement is not positive
    # definite, and the reference raises (linalg.inv of the zero factor it returns)
    "jdsa_tiny6_gap_fails": dict(name="tiny6", hs=2, ws=2, alpha=0.01, keep=lambda i: i != 2),
    # source frames {1, 2, 4, 5} (kx[0] = 1) in tiny7's window, 5% outliers, disparities
    # above 10 in frame 3 (no source edges: only the where/clamp touch it)
    "jdsa_tiny7_offset": dict(name="tiny7", hs=2, ws=2, alpha=0.01, keep=lambda i: i not in (0, 3), hot=3,
                              holes=0.0),
}


def _stub_modules():
    def proj_trans(poses, disps, intrinsics, targets, weights, ii, jj):
        C, w = geometry.proj_trans(poses.numpy(), disps.numpy(), intrinsics.numpy(), targets.numpy(),
                                   weights.numpy(), ii.numpy(), jj.numpy())
        return [torch.from_numpy(C).float(), torch.from_numpy(w).float()]

    def bi_inter(scales, grids):
        out, jac = geometry.bi_inter(scales.numpy(), grids.numpy())
        return [torch.from_numpy(out).float(), torch.from_numpy(jac).float()]

    def scatter_sum(src, index, dim=-1, dim_size=None):
        dim = dim % src.dim()
        n = int(index.max()) + 1 if dim_size is None else dim_size
        shape = list(src.shape)
        shape[dim] = n
        return torch.zeros(shape, dtype=src.dtype).index_add_(dim, index, src)

    class _Group:
        def __init__(self, data):
            self.data = data

    db = types.ModuleType("droid_backends")
    db.proj_trans, db.bi_inter = proj_trans, bi_inter
    ts = types.ModuleType("torch_scatter")
    ts.scatter_sum = scatter_sum
    lt = types.ModuleType("lietorch")
    lt.SE3 = lt.Sim3 = _Group
    return {"droid_backends": db, "torch_scatter": ts, "lietorch": lt}


def load_reference_jdsa(reference=None):
    sys.modules.update(_stub_modules())
    sys.path.insert(0, os.path.join(build_ref.reference_path(reference), "hislam2"))
    from geom.ba import JDSA
    return JDSA, sys.modules["lietorch"].SE3


def run_case(JDSA, SE3, cfg):
    p = synth.make_jdsa_problem(cfg["name"], hs=cfg["hs"], ws=cfg["ws"], alpha=cfg["alpha"], keep=cfg.get("keep"),
                                prior_holes=cfg.get("holes", 0.1))
    if "hot" in cfg:
        p["disps"][cfg["hot"], :3] = 12.0
    disps_in = p["disps"].clone()
    dscales = p["dscales"].clone()
    cuda = torch.Tensor.cuda
    torch.Tensor.cuda = lambda self, *a, **k: self
    arrays = {k: (v.numpy() if isinstance(v, torch.Tensor) else np.asarray(v)) for k, v in p.items()}
    arrays["disps"] = disps_in.numpy()
    try:
        disps, dscales_out, dzcov = JDSA(p["targets"], p["weights"], p["eta"], SE3(p["poses"][None].clone()),
                                         disps_in[None].clone(), p["intrinsics"][None, None].clone(),
                                         p["disps_prior"], dscales, p["ii"], p["jj"], p["alpha"])
    except torch.linalg.LinAlgError:
        arrays.update(raised=np.array(True))
        return arrays
    finally:
        torch.Tensor.cuda = cuda
    arrays.update(raised=np.array(False), out_disps=disps[0].numpy(), out_dscales=dscales_out.numpy(),
                  out_dzcov=dzcov.numpy())
    return arrays


def main(outdir=HERE):
    JDSA, SE3 = load_reference_jdsa()
    os.makedirs(outdir, exist_ok=True)
    for name, cfg in CASES.items():
        arrays = run_case(JDSA, SE3, cfg)
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **arrays)
        print("wrote", name)


if __name__ == "__main__":
    main(*sys.argv[1:])
