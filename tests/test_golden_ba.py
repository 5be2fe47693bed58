"""The float64 oracle pinned against outputs of the reference's own BA-family operators.

The fixtures (tests/golden/{ba,pgba,geo}_*.npz) were produced by
tests/golden/make_golden_ba.py, which runs HI-SLAM2's ``src/droid_kernels.cu``
through its own binding ``src/droid.cpp`` (compiled unmodified into oracle/_ref,
the Eigen facilities replaced by the dense stand-in in oracle/eigen_standin) on a
GPU, on the seeded tiny6 / tiny7 problems.  The reference computes in float32 on
the GPU and solves the reduced system in float64; the oracle is float64
throughout.  Tolerances (relative to the largest magnitude of each output):
poses, disparities and the geometry outputs 1e-4 (the bar for the FP32 form); dx and
dz, which the fixtures record for the LAST of three iterations (converged updates
whose relative rounding is larger), 1e-3; counts (depth_filter) must agree on all
but boundary pixels.
"""

import glob
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BA = sorted(glob.glob(os.path.join(GOLDEN, "ba_*.npz")))


def rel(a, b):
    b = np.asarray(b, np.float64)
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def test_fixtures_present():
    names = {os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    assert {"ba_tiny6_t0_2", "ba_tiny6_t0_0", "ba_tiny6_motion_only", "ba_tiny6_eta_one_row", "ba_tiny7_window",
            "pgba_tiny6", "geo_frame_distance_b03", "geo_frame_distance_b07", "geo_iproj", "geo_covis_distance",
            "geo_depth_filter", "geo_proj_trans", "geo_bi_inter"} <= names


@pytest.mark.parametrize("path", BA, ids=lambda f: os.path.basename(f)[:-4])
def test_ba_oracle_matches_reference(path):
    d = np.load(path)
    motion_only = bool(d["motion_only"])
    r = oracle.ba.ba(d["poses"], d["disps"], d["intrinsics"], d["targets"], d["weights"], d["eta"], d["ii"],
                     d["jj"], int(d["t0"]), int(d["t1"]), int(d["iterations"]), float(d["lm"]), float(d["ep"]),
                     motion_only)
    assert rel(r.poses, d["out_poses"]) < 1e-4
    assert rel(r.disps, d["out_disps"]) < 1e-4
    assert rel(r.dx, d["dx"]) < 1e-3
    if motion_only:
        assert "dz" not in d.files
        np.testing.assert_array_equal(r.disps, d["disps"])
    else:
        assert rel(r.dz.reshape(d["dz"].shape), d["dz"]) < 1e-3


def test_ba_reference_leaves_frames_outside_the_window_and_graph_alone():
    d = np.load(os.path.join(GOLDEN, "ba_tiny7_window.npz"))
    t0, t1 = int(d["t0"]), int(d["t1"])
    np.testing.assert_array_equal(d["out_poses"][:t0], d["poses"][:t0])
    np.testing.assert_array_equal(d["out_poses"][t1:], d["poses"][t1:])
    np.testing.assert_array_equal(d["out_disps"][t1:], d["disps"][t1:])   # frame 6 is in no edge


def test_pgba_oracle_matches_reference():
    d = np.load(os.path.join(GOLDEN, "pgba_tiny6.npz"))
    names = ("poses", "disps", "intrinsics", "targets", "weights", "eta", "Hsp", "vsp", "ii", "jj", "iip", "jjp")
    r = oracle.pgba.pgba(*(d[k] for k in names), int(d["t0"]), int(d["t1"]), float(d["lm"]), float(d["ep"]))
    assert rel(r.dx, d["dx"]) < 1e-4
    assert rel(r.dz.reshape(d["dz"].shape), d["dz"]) < 1e-4
    assert rel(r.disps, d["out_disps"]) < 1e-4
    np.testing.assert_array_equal(d["out_poses"], d["poses"])              # pgba leaves the poses to its caller


@pytest.mark.parametrize("name", ["geo_frame_distance_b03", "geo_frame_distance_b07"])
def test_frame_distance_oracle_matches_reference(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    got = oracle.frame_distance.frame_distance(d["poses"], d["disps"], d["intrinsics"], d["ii"], d["jj"],
                                               float(d["beta"]))
    assert rel(got, d["dist"]) < 1e-4


def test_geometry_oracle_matches_reference():
    g = oracle.geometry
    d = np.load(os.path.join(GOLDEN, "geo_iproj.npz"))
    assert rel(g.iproj(d["poses"], d["disps"], d["intrinsics"]), d["points"]) < 1e-4
    d = np.load(os.path.join(GOLDEN, "geo_covis_distance.npz"))
    got = g.covis_distance(d["poses"], d["disps"], d["intrinsics"], d["ii"])
    HW = d["disps"].shape[1] * d["disps"].shape[2]
    assert np.abs(got - d["dist"]).max() <= 1.0 / HW                     # at most one boundary pixel
    d = np.load(os.path.join(GOLDEN, "geo_depth_filter.npz"))
    got = g.depth_filter(d["poses"], d["disps"], d["intrinsics"], d["ix"], d["thresh"])
    assert got.shape == d["counter"].shape
    assert np.mean(got != d["counter"]) < 5e-3
    d = np.load(os.path.join(GOLDEN, "geo_proj_trans.npz"))
    C, w = g.proj_trans(d["poses"], d["disps"], d["intrinsics"], d["targets"], d["weights"], d["ii"], d["jj"])
    assert rel(C, d["C"]) < 1e-4 and rel(w, d["w"]) < 1e-4
    d = np.load(os.path.join(GOLDEN, "geo_bi_inter.npz"))
    out, jac = g.bi_inter(d["scales"], d["grids"])
    assert rel(out, d["out"]) < 1e-5 and rel(jac, d["jac"]) < 1e-5
