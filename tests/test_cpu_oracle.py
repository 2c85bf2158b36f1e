"""The oracle against the golden vectors and closed-form cases (no GPU)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_morton3d_matches_reference_golden():
    g = np.load(os.path.join(GOLDEN, "morton_ref.npz"))
    codes = O.morton(g["points"], bbox_mode=0, scene_min=(0, 0, 0), scene_max=(1, 1, 1))
    assert np.array_equal(codes, g["codes3"])


def test_morton6d_matches_reference_golden():
    g = np.load(os.path.join(GOLDEN, "morton_ref.npz"))
    pts, n01 = g["points"], g["normals01"]
    # the oracle normalises normals over their own box (min..max); feed values whose box is [0,1]
    nrm = np.concatenate([np.zeros((1, 3), np.float32), np.ones((1, 3), np.float32), n01])
    p = np.concatenate([np.zeros((2, 3), np.float32), pts])
    codes = O.morton(p, nrm, consider_normals=True, bbox_mode=0)
    ref6 = O.ref_morton6d(p, nrm)
    if ref6 is not None:
        assert np.array_equal(codes, ref6)
    assert np.array_equal(codes[2:], g["codes6"])


def test_morton_reference_live_when_available():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(1)
    pts = rng.random((50000, 3), dtype=np.float32) * 1.2 - 0.1
    assert np.array_equal(O.morton(pts), O.ref_morton3d(pts))


def test_morton_avpl_box_mode_uses_flt_min_seed():
    # all-negative coordinates on x: the reference's max reduction keeps FLT_MIN (bvh.cu:349-350)
    pts = np.array([[-0.5, 0.2, 0.3], [-0.25, 0.8, 0.9], [-0.75, 0.5, 0.1]], np.float32)
    codes = O.morton(pts, bbox_mode=1)
    mn = pts.min(0)
    mx = np.maximum(pts.max(0), np.float32(np.finfo(np.float32).tiny))
    q = np.clip(((pts - mn) / (mx - mn)).astype(np.float32) * np.float32(1024), 0, 1023).astype(np.uint32)
    exp = O.ref_morton3d(((pts - mn) / (mx - mn)).astype(np.float32))
    if exp is not None:
        assert np.array_equal(codes, exp)
    assert q.shape == (3, 3)


def test_stable_sort_matches_numpy():
    rng = np.random.default_rng(2)
    keys = rng.integers(0, 64, size=10000).astype(np.uint32)
    assert np.array_equal(O.stable_sort(keys), np.argsort(keys, kind="stable"))


@pytest.mark.parametrize("n,dup", [(2, False), (3, False), (17, True), (1000, False), (4096, True), (65536, True)])
def test_karras_equals_topdown_and_is_consistent(n, dup):
    rng = np.random.default_rng(n)
    hi = 64 if dup else 1 << 30
    codes = np.sort(rng.integers(0, hi, size=n).astype(np.uint32))
    left, right, parents = O.karras(codes)
    l2, r2 = O.topdown(codes)
    assert np.array_equal(left, l2) and np.array_equal(right, r2)
    rc, _ = O.check_tree(left, right, parents)
    assert rc == 0


def test_karras_all_equal_codes():
    codes = np.zeros(1000, np.uint32)
    left, right, parents = O.karras(codes)
    assert O.check_tree(left, right, parents)[0] == 0
    l2, r2 = O.topdown(codes)
    assert np.array_equal(left, l2) and np.array_equal(right, r2)


def test_check_tree_detects_corruption():
    codes = np.arange(64, dtype=np.uint32)
    left, right, parents = O.karras(codes)
    bad = left.copy()
    bad[5] = bad[6]
    assert O.check_tree(bad, right, parents)[0] != 0


def _kat_inputs(c):
    pos = np.array([[c["pixel_pos"] + [1.0]]], np.float32)
    nrm = np.array([[c["pixel_nrm"] + [float(c["pixel_mat"])]]], np.float32)
    from antiradiancecuts_b200.scene import AVPL_DTYPE

    a = np.zeros(1, AVPL_DTYPE)
    a["position"], a["normal"], a["incDirection"] = c["avpl_pos"], c["avpl_nrm"], c["avpl_w"]
    a["incRadiance"], a["antiradiance"] = c["L"], c["A"]
    a["materialIndex"], a["bounce"] = c["avpl_mat"], 2
    return pos, nrm, a


def test_oracle_known_answer_cases():
    with open(os.path.join(GOLDEN, "gather_kat.json")) as f:
        cases = json.load(f)
    for c in cases:
        pos, nrm, a = _kat_inputs(c)
        prm = O.params(c["ar_kind"], c["half_angle_deg"], c["clamp"], c.get("disk_radius", 0.0))
        rad, ar, res = O.gather_fp64(pos, nrm, [0], a, c["materials"], c["specular"], c["exponent"], c["cam"], prm)
        np.testing.assert_allclose(rad[0], c["rad"], rtol=2e-6, atol=1e-12, err_msg=c["name"])
        np.testing.assert_allclose(ar[0], c["ar"], rtol=2e-6, atol=1e-12, err_msg=c["name"])
        np.testing.assert_allclose(res[0], np.array(c["rad"]) - np.array(c["ar"]), rtol=2e-6, atol=1e-9)
        r32 = O.gather_fp32(pos, nrm, [0], a, c["materials"], c["specular"], c["exponent"], c["cam"], prm)
        np.testing.assert_allclose(r32[0], res[0], rtol=1e-4, atol=1e-6, err_msg=c["name"])


def test_fp32_oracle_close_to_fp64_on_room(room_small):
    d = room_small
    px = np.arange(0, d["pos"].shape[0] * d["pos"].shape[1], 7)
    prm = O.params(2, 30.0, 0.01)
    _, _, ref = O.gather_fp64(d["pos"], d["nrm"], px, d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"], prm)
    r32 = O.gather_fp32(d["pos"], d["nrm"], px, d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"], prm, threads=4)
    err = np.sqrt(np.mean((r32 - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
    assert err < 1e-5


def test_bottom_up_invariants(room_small):
    d = room_small
    tree = O.build_tree(d["avpls"], d["dif"])
    n = len(d["avpls"])
    assert tree["size"][n] == n
    # root box contains every AVPL; summed L equals the float64 sum within rounding
    b = tree["bounds"][0]
    p = d["avpls"]["position"]
    assert (p >= b[0:3]).all() and (p <= b[4:7]).all()
    np.testing.assert_allclose(tree["incRadiance"][n], d["avpls"]["incRadiance"].astype(np.float64).sum(0), rtol=1e-4)
    # representative of every inner node is one of its leaves
    assert math.isfinite(float(tree["records"][n][0]))


def test_scene_generator_is_frozen():
    """The synthetic-scene generator (shared by the CPU and GPU versions) still produces the inputs
    the benchmark and the shipped network were made with (tests/golden/scene_gen.json)."""
    import json
    import os
    import sys

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    import make_golden

    with open(os.path.join(here, "scene_gen.json")) as f:
        want = json.load(f)
    assert make_golden.scene_digests() == want


@pytest.mark.parametrize("w,h,z_near,theta_deg", [(48, 32, 0.1, None), (37, 21, 0.1, 20.0), (32, 32, 1e-6, 0.5)])
def test_clustered_disk_antiradiance_equals_bruteforce_in_the_oracle(w, h, z_near, theta_deg):
    """The cluster light lists keep every AVPL whose disk antiradiance reaches a pixel of the
    cluster: in the FP64 oracle the clustered sum equals the full sum bit for bit (the AVPLs left
    out contribute exact zeros, and the order is the AVPLs' order).  Also on partial tiles and with
    slices so thin that most pixels of a tile are clusters of their own."""
    import helpers as H
    from antiradiancecuts_b200 import scene
    from oracle import oracle as O

    d = H.workload("boxes2_720p_64k", w, h, 2048)
    r = 2.0 * scene.scene_extent(d["desc"]) / 100.0
    prm = O.params(1, 30.0, 0.0, r)
    theta = math.radians(0.5 * d["desc"].camera_fov_deg if theta_deg is None else theta_deg)
    ar, nclusters, entries = O.clustered_disk_ar(d["pos"], d["nrm"], d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"],
                                                 z_near, theta, prm)
    px = np.arange(w * h)
    _, full, _ = O.gather_fp64(d["pos"], d["nrm"], px, d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"], prm)
    assert np.abs(full).max() > 0 and nclusters > 6
    if z_near < 1e-3:
        assert nclusters > 4 * 64  # four 16x16 tiles, most of their pixels in clusters of their own
    assert 0 < entries < nclusters * len(d["avpls"])  # the lists do cull
    assert np.array_equal(ar, full)
