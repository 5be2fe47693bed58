"""Pins the float64 JDSA oracle (``oracle/jdsa.py``) to the reference's own ``JDSA``
(``hislam2/geom/ba.py:170-219`` run in float32 by ``tests/golden/make_golden_jdsa.py``)."""

import glob
import os

import numpy as np
import pytest

from oracle import jdsa

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "jdsa_*.npz")))


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def run_oracle(g):
    return jdsa.jdsa(g["targets"], g["weights"], g["eta"], g["poses"], g["disps"], g["intrinsics"],
                     g["disps_prior"], g["dscales"], g["ii"], g["jj"], float(g["alpha"]))


def rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def test_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in CASES}
    assert {"jdsa_tiny6_2x2", "jdsa_tiny6_3x4", "jdsa_tiny6_4x4", "jdsa_tiny6_gap", "jdsa_tiny6_gap_fails",
            "jdsa_tiny7_offset"} <= names


@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_jdsa(path):
    g = load(path)
    if bool(g["raised"]):
        with pytest.raises(np.linalg.LinAlgError):
            run_oracle(g)
        return
    r = run_oracle(g)
    # the reference runs in float32 (a dense [M*D, M*D] Cholesky and a float32 Schur
    # complement over all M*HW unknowns); disparities within 1e-5 of their range
    assert rel(r["disps"], g["out_disps"]) < 1e-5
    assert rel(r["dscales"] - g["dscales"], g["out_dscales"] - g["dscales"]) < 1e-3
    assert rel(r["dzcov"], g["out_dzcov"]) < 1e-4


def test_where_and_clamp_cover_frames_without_edges():
    g = load(os.path.join(GOLDEN, "jdsa_tiny7_offset.npz"))
    r = run_oracle(g)
    assert 3 not in set(r["kx"].tolist())
    assert np.all(r["disps"][3, :3] == 0.001)            # > 10 -> 0 -> clamp(min=0.001)
    np.testing.assert_array_equal(r["disps"][3, 3:], np.maximum(g["disps"][3, 3:], 0.001))
