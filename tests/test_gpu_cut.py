"""Cut gathers on the GPU against the oracle: the solid-angle lightcut (kernel_bvh semantics) and
the error-bound tile cut (cut lists identical, evaluation within FP tolerance)."""
import math

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api
from oracle import oracle as O

pytestmark = pytest.mark.gpu

W, HGT, N = 320, 180, 65536


@pytest.fixture(scope="module")
def boxes(ctx):
    d = H.workload("boxes2_720p_64k", W, HGT, N)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    bvh = api.AvplBvh(ctx)
    bvh.build(dv)
    assert ctx.synchronize() == 0
    tree = bvh.host_arrays()
    gb = api.GBuffer(d["pos"], d["nrm"])
    return d, dv, bvh, tree, gb


def test_solid_angle_cut_matches_oracle(ctx, boxes):
    d, dv, bvh, tree, gb = boxes
    w = d["w"]
    prm = api.gather_params(L.ARC_AR_CONE, w.cone_half_angle_deg, w.dist_clamp)
    cut = api.cut_params(L.ARC_CUT_SOLID_ANGLE, solid_angle_threshold=math.pi / 10)
    out = api.Outputs(W, HGT)
    api.gather_cut(ctx, bvh, dv, gb, d["cam"], prm, cut, out)
    assert ctx.synchronize() == 0
    px = np.arange(W * HGT)
    rad, err = O.cut_solid_angle(d["pos"], d["nrm"], px, tree, d["dif"], d["spe"], d["ex"], d["cam"], math.pi / 10,
                                 w.dist_clamp)
    assert err.sum() == 0
    got = out.radiance.cpu().numpy()[..., :3].reshape(-1, 3)
    assert H.rel_rmse(got, rad) < 1e-5
    _, ar, _ = O.gather_fp64(d["pos"], d["nrm"], px, d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"],
                             O.params(2, w.cone_half_angle_deg, w.dist_clamp))
    res = out.result64.cpu().numpy().reshape(-1, 3)
    assert H.rel_rmse(res, rad - ar) < 1e-5


def test_solid_angle_probe_marks_used_nodes(ctx, boxes):
    import torch

    d, dv, bvh, tree, gb = boxes
    used = torch.zeros(2 * N - 1, dtype=torch.int32, device="cuda")
    cut = api.cut_params(L.ARC_CUT_SOLID_ANGLE, debug_pixel=(160, 90), used_nodes=used.data_ptr())
    out = api.Outputs(W, HGT)
    api.gather_cut(ctx, bvh, dv, gb, d["cam"], api.gather_params(L.ARC_AR_NONE, dist_clamp=0.01), cut, out)
    assert ctx.synchronize() == 0
    u = used.cpu().numpy()
    assert u.sum() > 0
    # the used nodes form a cut: every leaf is covered by exactly one used node or is unreachable
    # because its cluster was culled; at least no used node is an ancestor of another used node
    n = N
    parents = tree["parents"]
    for idx in np.nonzero(u)[0][:2000]:
        p = parents[idx]
        while p != -1:
            assert u[n + p] == 0
            p = parents[n + p]


@pytest.mark.parametrize("eps", [0.03, 0.01])
def test_error_bound_cut_lists_identical(ctx, boxes, eps):
    d, dv, bvh, tree, gb = boxes
    w = d["w"]
    prm = api.gather_params(L.ARC_AR_CONE, w.cone_half_angle_deg, w.dist_clamp)
    cut = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=eps)
    out = api.Outputs(W, HGT)
    api.gather_cut(ctx, bvh, None, gb, d["cam"], prm, cut, out)
    assert ctx.synchronize() == 0
    gcuts = api.last_cut(ctx)
    ocuts, tau, ov = O.tile_cut(d["pos"], d["nrm"], tree, d["dif"], eps, w.dist_clamp, 2, w.cone_half_angle_deg,
                                max_cut=65536)
    assert ov == 0
    assert len(gcuts) == len(ocuts)
    bad = [t for t in range(len(gcuts)) if not np.array_equal(gcuts[t], ocuts[t])]
    assert not bad, f"{len(bad)} tiles differ, first {bad[:5]}"
    # the evaluation of the GPU's cuts against the FP64 evaluation of the same cuts
    rad, ar, res = O.eval_cut(d["pos"], d["nrm"], tree, gcuts, d["dif"], 2, w.cone_half_angle_deg, w.dist_clamp)
    got = out.result64.cpu().numpy().reshape(-1, 3)
    assert H.rel_rmse(got, res) < 2e-5
    # and the approximation error against the exact FP64 gather (reported; bound loosely)
    px = np.arange(W * HGT)
    _, _, exact = O.gather_fp64(d["pos"], d["nrm"], px, d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"],
                                O.params(2, w.cone_half_angle_deg, w.dist_clamp))
    assert H.rel_rmse(got, exact) < 0.05


def test_cut_overflow_is_reported(ctx, boxes):
    d, dv, bvh, tree, gb = boxes
    prm = api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    out = api.Outputs(W, HGT)
    # per-tile capacity
    cut = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.001, max_cut_nodes=2048)
    api.gather_cut(ctx, bvh, None, gb, d["cam"], prm, cut, out)
    assert ctx.synchronize() & L.ARC_DEVERR_CUT_OVERFLOW
    counts = api.cut_counts(ctx)
    assert counts.max() <= 2048
    # pool capacity
    cut = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.001, cut_pool_entries=100 * 1024)
    api.gather_cut(ctx, bvh, None, gb, d["cam"], prm, cut, out)
    assert ctx.synchronize() & L.ARC_DEVERR_CUT_OVERFLOW
    cl = api.last_cut(ctx)
    assert sum(len(c) for c in cl) <= 100 * 1024


def test_error_bound_cut_lists_identical_at_configuration_size(ctx):
    """The LBVH + error-bound cut configuration at its stated size: room + 2 boxes, 1280x720, 65,536
    AVPLs, relative error bound 1%.  Every tile's cut list equals the oracle's (the oracle runs
    strip by strip: a tile's cut depends only on its own pixels), and one strip's image equals the
    FP64 evaluation of the GPU's lists."""
    d = H.workload("boxes2_720p_64k")
    w = d["w"]
    Wf, Hf = w.width, w.height
    assert (Wf, Hf, len(d["avpls"])) == (1280, 720, 65536)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    bvh = api.AvplBvh(ctx)
    bvh.build(dv)
    gb = api.GBuffer(d["pos"], d["nrm"])
    prm = api.gather_params(L.ARC_AR_CONE, w.cone_half_angle_deg, w.dist_clamp)
    out = api.Outputs(Wf, Hf)
    api.gather_cut(ctx, bvh, None, gb, d["cam"], prm, api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.01), out)
    assert ctx.synchronize() == 0
    gcuts = api.last_cut(ctx)
    tree = bvh.host_arrays()
    tx = Wf // 8
    rows = 64  # strips of 8 tile rows
    total = 0
    for y0 in range(0, Hf, rows):
        ocuts, _, ov = O.tile_cut(d["pos"][y0:y0 + rows], d["nrm"][y0:y0 + rows], tree, d["dif"], 0.01, w.dist_clamp,
                                  2, w.cone_half_angle_deg, max_cut=65536)
        assert ov == 0
        first = (y0 // 8) * tx
        bad = [t for t in range(len(ocuts)) if not np.array_equal(gcuts[first + t], ocuts[t])]
        assert not bad, f"strip at row {y0}: {len(bad)} tiles differ, first {bad[:5]}"
        total += sum(len(c) for c in ocuts)
        if y0 == 320:
            _, _, res = O.eval_cut(d["pos"][y0:y0 + rows], d["nrm"][y0:y0 + rows], tree,
                                   gcuts[first:first + len(ocuts)], d["dif"], 2, w.cone_half_angle_deg, w.dist_clamp)
            got = out.result64.cpu().numpy()[y0:y0 + rows].reshape(-1, 3)
            assert H.rel_rmse(got, res) < 2e-5
    assert total == sum(len(c) for c in gcuts)
    bvh.close()
