"""The CPU oracle pinned against outputs of the reference's own correlation kernels.

The fixtures in tests/golden/ were produced by tests/golden/make_golden.py, which
runs HI-SLAM2's ``src/correlation_kernels.cu`` / ``src/altcorr_kernel.cu``
(compiled unmodified into oracle/_ref) on a GPU.  Tolerances: float32 inputs
1e-5 relative to the largest output; float16 inputs 2e-3, since the reference
accumulates each of the <=4 bilinear terms in half precision in place.
"""

import glob
import os

import numpy as np
import pytest

from oracle import corr as oc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def rel(a, b):
    b = np.asarray(b, np.float64)
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def test_fixtures_present():
    names = {os.path.basename(f)[:-4] for f in FILES}
    assert {"corr_index_f32_r3", "corr_index_f32_r4_int", "corr_index_f16_r2", "altcorr_f32_r2",
            "altcorr_f32_r3"} <= names


@pytest.mark.parametrize("path", [f for f in FILES if "corr_index" in os.path.basename(f)],
                         ids=lambda f: os.path.basename(f))
def test_corr_index_oracle_matches_reference(path):
    d = np.load(path)
    r = int(d["radius"])
    tol = 2e-3 if d["volume"].dtype == np.float16 else 1e-5
    out = oc.corr_index_forward(d["volume"], d["coords"], r)
    assert rel(out, d["corr"]) < tol
    vg = oc.corr_index_backward(d["volume"].shape, d["coords"], d["corr_grad"], r)
    assert rel(vg, d["volume_grad"]) < tol


@pytest.mark.parametrize("path", [f for f in FILES if "altcorr" in os.path.basename(f)],
                         ids=lambda f: os.path.basename(f))
def test_altcorr_oracle_matches_reference(path):
    d = np.load(path)
    r = int(d["radius"])
    out = oc.altcorr_forward(d["fmap1"], d["fmap2"], d["coords"], d["ii"], d["jj"], r)
    assert rel(out, d["corr"]) < 1e-5
    # the reference operator leaves out the forward's 1/16 (scale = 1)
    g1, g2 = oc.altcorr_backward(d["fmap1"], d["fmap2"], d["coords"], d["ii"], d["jj"], d["grad"], r)
    assert rel(g1, d["fmap1_grad"]) < 1e-5
    assert rel(g2, d["fmap2_grad"]) < 1e-5
