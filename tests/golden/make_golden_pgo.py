"""Generates tests/golden/pgo_*.npz: outputs of the reference's own relative-pose factor
terms, HI-SLAM2 ``hislam2/pgo_buffer.py:15-63`` (``diff``, ``num_jacobi``,
``global_relative_posesim3_constraints``).

TEST INFRASTRUCTURE.  Runs on the CPU.  The three functions and ``eps`` are taken from the
checkout's ``pgo_buffer.py`` with ``ast`` (``$HISLAM2_REFERENCE``, else the default of
``oracle/build_ref.py``) and executed unmodified; importing the whole module would pull
in the networks and the multiprocessing buffer, which these functions do not use.  Their
free names are supplied here:

* ``Sim3`` / ``SE3``: a stand-in for lietorch's groups (a third-party submodule of
  HI-SLAM2, princeton-vl/lietorch, unpinned and not installed) with the members the
  functions use -- construction from data or from an SE3, ``.data``, ``.shape``,
  ``manifold_dim``, indexing, broadcast products, ``inv``, ``log`` and ``Sim3.exp`` --
  evaluated element by element with ``oracle/pgo.py``'s float64 Sim3 (the definitions
  lietorch's Sim3 follows, computed as scipy's expm / logm);
* ``torch``: the real module, except that ``zeros(..., device='cuda')`` stays on the CPU.

So the fixtures pin the reference's procedure -- step 1e-8 central differences, the float32
/ float64 casts, the block layout and the chi^2 sums -- while the Sim3 algebra itself stays
as pinned as ``oracle/pgo.py`` is (group identities).  Inputs are stored beside the outputs.

Usage: ``python tests/golden/make_golden_pgo.py [outdir]``.
"""

import ast
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "hi-slam2_b200")]

from hislam2_b200 import synth  # noqa: E402
from oracle import build_ref  # noqa: E402
from oracle import pgo as opgo  # noqa: E402


class SE3:
    def __init__(self, data):
        self.data = data


class Sim3:
    """Elements are kept as 4x4 matrices between operations: converting a product back to
    [t, q, s] (quaternion from a rotation matrix) would lose the 1e-8 perturbations."""
    manifold_dim = 7

    def __init__(self, data=None, mats=None):
        if isinstance(data, SE3):
            d = data.data
            data = torch.cat([d, torch.ones(d.shape[:-1] + (1,), dtype=d.dtype)], -1)
        self._data, self._M = data, mats

    @property
    def data(self):
        if self._data is None:
            M = self._M
            flat = np.stack([opgo.from_matrix(m) for m in M.reshape(-1, 4, 4)])
            self._data = torch.from_numpy(flat.reshape(M.shape[:-2] + (8,)))
        return self._data

    @property
    def shape(self):
        return self._M.shape[:-2] if self._data is None else self._data.shape[:-1]

    def __getitem__(self, idx):
        return Sim3(self.data[idx])

    def _mats(self):
        if self._M is None:
            d = self._data.double().numpy()
            self._M = np.stack([opgo.to_matrix(x) for x in d.reshape(-1, 8)]).reshape(d.shape[:-1] + (4, 4))
        return self._M

    def __mul__(self, other):
        return Sim3(mats=np.matmul(self._mats(), other._mats()))

    def inv(self):
        return Sim3(mats=np.linalg.inv(self._mats()))

    def log(self):
        M = self._mats()
        out = np.stack([opgo.log(m) for m in M.reshape(-1, 4, 4)])
        return torch.from_numpy(out.reshape(M.shape[:-2] + (7,)))

    @staticmethod
    def exp(xi):
        x = xi.double().numpy()
        return Sim3(mats=np.stack([opgo.exp(v) for v in x.reshape(-1, 7)]).reshape(x.shape[:-1] + (4, 4)))


class _TorchOnCpu:
    def __getattr__(self, name):
        return getattr(torch, name)

    @staticmethod
    def zeros(*size, device=None, **kw):
        return torch.zeros(*size, **kw)


def load_reference_constraints(reference=None):
    path = os.path.join(build_ref.reference_path(reference), "hislam2", "pgo_buffer.py")
    tree = ast.parse(open(path).read(), path)
    keep = [n for n in tree.body
            if (isinstance(n, ast.FunctionDef) and n.name in ("diff", "num_jacobi", "global_relative_posesim3_constraints"))
            or (isinstance(n, ast.Assign) and any(getattr(t, "id", None) == "eps" for t in n.targets))]
    ns = {"torch": _TorchOnCpu(), "Sim3": Sim3, "SE3": SE3}
    exec(compile(ast.Module(body=keep, type_ignores=[]), path, "exec"), ns)
    return ns["global_relative_posesim3_constraints"]


CASES = {
    # frontend_small's 16 factors (8 Sim3 poses), se3 noise 0.02 on the measurements
    "pgo_frontend_small": dict(name="frontend_small", seed=0, noise=0.02, pw=1e-3),
    # 25 poses, 40 factors, larger measurement noise and the reference's default pw
    "pgo_frontend40": dict(name="frontend", seed=1, noise=0.1, pw=1e-5, num_factors=40),
}


def run_case(fn, cfg):
    p = synth.make_pgba_problem(cfg["name"], cfg["seed"], num_factors=cfg.get("num_factors"))
    rel, infos = synth.make_pgo_factors(p["poses"], p["iip"], p["jjp"], seed=cfg["seed"], noise=cfg["noise"])
    Hsp, vsp, chi2, chi2s = fn(p["iip"], p["jjp"], Sim3(p["poses"][None].clone()), rel[None].clone(), infos,
                               pw=cfg["pw"])
    return dict(poses=p["poses"].numpy(), iip=p["iip"].numpy(), jjp=p["jjp"].numpy(), rel=rel.numpy(),
                infos=infos.numpy(), pw=np.array(cfg["pw"]), Hsp=Hsp.numpy(), vsp=vsp.numpy(),
                chi2=np.array(float(chi2)), chi2_scaled=np.array(float(chi2s)))


def main(outdir=HERE):
    fn = load_reference_constraints()
    os.makedirs(outdir, exist_ok=True)
    for name, cfg in CASES.items():
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **run_case(fn, cfg))
        print("wrote", name)


if __name__ == "__main__":
    main(*sys.argv[1:])
