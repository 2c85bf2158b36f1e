"""Clustered deferred antiradiance (arc_antiradiance_clustered): the screen clusters, the cluster
light lists against a NumPy restatement of intersectBB (cudaGather.cu:663-684), and the image
against the brute-force disk antiradiance."""
import ctypes as C
import math

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api, scene

pytestmark = pytest.mark.gpu

W, HGT, N = 96, 64, 8192


@pytest.fixture(scope="module")
def case(ctx):
    d = H.workload("boxes2_720p_64k", W, HGT, N)
    ctx.upload_materials(d["mats"])
    dv = api.DeviceAvpls(d["avpls"])
    gb = api.GBuffer(d["pos"], d["nrm"])
    r = 2.0 * scene.scene_extent(d["desc"]) / 100.0  # photonRadiusScale * sceneExtent / 100
    prm = api.gather_params(L.ARC_AR_DISK, 30.0, 0.0, disk_radius=r)
    cp = L.ArcClusterParams(0.1, math.radians(0.5 * d["desc"].camera_fov_deg))
    out = api.Outputs(W, HGT)
    info = L.ArcClusterInfo()
    L.check(ctx.lib.arc_antiradiance_clustered(ctx.handle, C.byref(dv.param), C.byref(gb.view()), L.f3(d["cam"]),
                                               C.byref(cp), C.byref(prm), C.byref(out.view()), C.byref(info)),
            "arc_antiradiance_clustered")
    assert ctx.synchronize() == 0
    host = {
        "pixel": ctx.d2h(info.pixel_cluster, np.int32, W * HGT).reshape(HGT, W),
        "tile_count": ctx.d2h(info.tile_count, np.int32, info.num_tiles),
        "box": ctx.d2h(info.box, np.float32, info.num_tiles * info.slots_per_tile * 8).reshape(-1, 8),
        "counts": ctx.d2h(info.counts, np.int32, info.num_tiles * info.slots_per_tile),
        "lists": ctx.d2h(info.lists, np.int32, max(1, info.list_entries))[: info.list_entries],
    }
    return d, dv, gb, prm, r, out, info, host


def test_clusters_partition_the_surface_pixels(case):
    d, _, _, _, _, _, info, h = case
    surface = d["nrm"][..., 3] > 0
    pix = h["pixel"]
    assert np.all(pix[~surface] == -1) and np.all(pix[surface] >= 0)
    tiles_x = (W + 15) // 16
    ys, xs = np.nonzero(surface)
    tile = (ys // 16) * tiles_x + xs // 16
    slot = pix[ys, xs]
    assert np.all(slot // info.slots_per_tile == tile)
    assert np.all(slot % info.slots_per_tile < h["tile_count"][tile])
    # every cluster's box is the box of its pixels
    pos = d["pos"][ys, xs, :3]
    for s in np.unique(slot):
        p = pos[slot == s]
        assert np.array_equal(h["box"][s, :3], p.min(0)) and np.array_equal(h["box"][s, 4:7], p.max(0))
    # within a tile, clusters are depth slices in increasing distance from the camera
    dist = np.linalg.norm(pos - np.array(d["cam"], np.float32), axis=1)
    for t in np.unique(tile):
        sl = slot[tile == t]
        dd = dist[tile == t]
        order = [dd[sl == s] for s in np.unique(sl)]
        assert all(a.max() <= b.min() * (1 + 1e-5) for a, b in zip(order, order[1:]))


def test_cluster_lists_match_the_ray_box_test(case):
    d, _, _, _, r, _, info, h = case
    av = d["avpls"]
    o = av["position"].astype(np.float32)
    dirs = av["incDirection"].astype(np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        f = np.float32(1.0) / dirs
    grow = np.float32(2.0 * np.float32(r))
    offs = np.concatenate([[0], np.cumsum(h["counts"])])
    used = np.nonzero(h["counts"])[0]
    assert len(used) > 0
    for s in used[:: max(1, len(used) // 40)]:
        lo = (h["box"][s, :3] - grow).astype(np.float32)
        hi = (h["box"][s, 4:7] + grow).astype(np.float32)
        with np.errstate(invalid="ignore"):
            t1 = (lo - o) * f
            t2 = (hi - o) * f
        tmin = np.fmax(np.fmax(np.fmin(t1[:, 0], t2[:, 0]), np.fmin(t1[:, 1], t2[:, 1])), np.fmin(t1[:, 2], t2[:, 2]))
        tmax = np.fmin(np.fmin(np.fmax(t1[:, 0], t2[:, 0]), np.fmax(t1[:, 1], t2[:, 1])), np.fmax(t1[:, 2], t2[:, 2]))
        want = np.nonzero(~((tmax < 0) | (tmin > tmax)))[0]
        got = h["lists"][offs[s]:offs[s + 1]]
        assert np.array_equal(got, want), s


def test_clustered_antiradiance_equals_bruteforce(ctx, case):
    d, dv, gb, prm, _, out, _, _ = case
    ref = api.Outputs(W, HGT)
    api.gather_bruteforce(ctx, dv.param, gb, d["cam"], prm, ref)
    assert ctx.synchronize() == 0
    a = out.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3)
    b = ref.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3)
    assert np.abs(b).max() > 0  # the case has disk antiradiance
    assert H.rel_rmse(a, b) < 1e-5
    assert np.array_equal(np.all(a == 0, axis=1), np.all(b == 0, axis=1))  # the same pixels receive some


def test_clustered_needs_the_disk_variant(ctx, case):
    d, dv, gb, _, _, out, _, _ = case
    cone = api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    cp = L.ArcClusterParams(0.1, 0.35)
    st = ctx.lib.arc_antiradiance_clustered(ctx.handle, C.byref(dv.param), C.byref(gb.view()), L.f3(d["cam"]),
                                            C.byref(cp), C.byref(cone), C.byref(out.view()), None)
    assert st == L.ARC_ERR_INVALID_ARG


@pytest.mark.parametrize("w,h,z_near,theta", [(37, 21, 0.1, 0.35), (64, 48, 1e-6, 0.01)])
def test_clustered_edge_cases(ctx, w, h, z_near, theta):
    """Partial tiles (an image that is not a multiple of 16), and slices so thin that nearly every
    pixel of a tile is its own cluster (up to 256 per tile): still the brute-force antiradiance."""
    d = H.workload("boxes2_720p_64k", w, h, 4096)
    ctx.upload_materials(d["mats"])
    dv = api.DeviceAvpls(d["avpls"])
    gb = api.GBuffer(d["pos"], d["nrm"])
    r = 2.0 * scene.scene_extent(d["desc"]) / 100.0
    prm = api.gather_params(L.ARC_AR_DISK, 30.0, 0.0, disk_radius=r)
    out, ref = api.Outputs(w, h), api.Outputs(w, h)
    info = L.ArcClusterInfo()
    L.check(ctx.lib.arc_antiradiance_clustered(ctx.handle, C.byref(dv.param), C.byref(gb.view()), L.f3(d["cam"]),
                                               C.byref(L.ArcClusterParams(z_near, theta)), C.byref(prm),
                                               C.byref(out.view()), C.byref(info)), "arc_antiradiance_clustered")
    api.gather_bruteforce(ctx, dv.param, gb, d["cam"], prm, ref)
    assert ctx.synchronize() == 0
    tc = ctx.d2h(info.tile_count, np.int32, info.num_tiles)
    a = out.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3)
    b = ref.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3)
    assert H.rel_rmse(a, b) < 1e-5
    if z_near < 1e-3:
        assert tc.max() > 64  # many clusters in a tile


def test_clustered_antiradiance_matches_the_oracle(case):
    """Against the oracle's restatement of the whole path (oracle_clustered_disk_ar: the same
    screen clusters, light lists by the slab test, FP64 disk terms over each list): the number of
    clusters and list entries to 1% (a pixel on a depth-slice boundary may fall on the other side
    of it in FP64), the image to 1e-5 relative RMSE (FP32 terms on the GPU)."""
    from oracle import oracle as O

    d, _, _, _, r, out, info, h = case
    op = O.params(1, 30.0, 0.0, disk_radius=r)
    ref, nclusters, entries = O.clustered_disk_ar(d["pos"], d["nrm"], d["avpls"], d["dif"], d["spe"], d["ex"],
                                                  d["cam"], 0.1, math.radians(0.5 * d["desc"].camera_fov_deg), op)
    assert abs(int(h["tile_count"].sum()) - nclusters) <= 0.01 * nclusters
    assert abs(int(info.list_entries) - entries) <= 0.01 * entries
    a = out.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3)
    assert np.abs(ref).max() > 0
    assert H.rel_rmse(a, ref) < 1e-5
