"""Multi-view batches (arc_batch_*) and the brute-force launch-shape autotuner."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api, scene

pytestmark = pytest.mark.gpu

NUM_VIEWS = 5


@pytest.fixture(scope="module")
def views(ctx):
    """Views of the room + 2 boxes scene (seed 4 draws), at 1/8 resolution and at most 16,384 AVPLs
    each so that the test stays small; device inputs and outputs per view."""
    desc = scene.scene_desc(L.ARC_SCENE_ROOM_2BOXES, 2, 2)
    mats, _, _, _ = scene.materials(desc)
    ctx.upload_materials(mats)
    out = []
    for v in scene.batch_views(desc, 4, NUM_VIEWS):
        v.num_avpls = min(v.num_avpls, 16384)
        avpls, pos, nrm = scene.view_inputs(desc, v, scale=0.125)
        dv = api.DeviceAvpls(avpls)  # each view keeps its own device AVPL arrays
        h, w = pos.shape[:2]
        cam = (v.camera_position.x, v.camera_position.y, v.camera_position.z)
        out.append({"avpls": dv.param, "keep": dv, "gb": api.GBuffer(pos, nrm), "cam": cam, "w": w, "h": h})
    return out


def _params():
    return (api.lbvh_params(), api.gather_params(L.ARC_AR_CONE, 30.0, 0.01),
            api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.01))


def _individual(ctx, views):
    lp, gp, cp = _params()
    imgs = []
    for v in views:
        bvh = api.AvplBvh(ctx)
        L.check(ctx.lib.arc_lbvh_build(bvh.handle, C.byref(v["avpls"]), C.byref(lp)), "build")
        out = api.Outputs(v["w"], v["h"])
        api.gather_cut(ctx, bvh, v["avpls"], v["gb"], v["cam"], gp, cp, out)
        assert ctx.synchronize() == 0
        imgs.append(out.result64.cpu().numpy().copy())
        bvh.close()
    return imgs


def test_generator_draws_the_configured_distribution():
    desc = scene.scene_desc(L.ARC_SCENE_ROOM_2BOXES, 2, 2)
    vs = scene.batch_views(desc, 4, 256)
    assert {(v.width, v.height) for v in vs} == {(256, 256), (512, 512), (1280, 720), (1920, 1080)}
    n = np.array([v.num_avpls for v in vs])
    assert n.min() >= 8192 and n.max() <= 262144 and np.median(n) < 70000  # log-uniform
    assert [v.avpl_seed for v in scene.batch_views(desc, 4, 8)] == [v.avpl_seed for v in vs[:8]]


def test_batch_equals_individual_views_and_graph_replays_it(ctx, views):
    ref = _individual(ctx, views)
    lp, gp, cp = _params()
    outs = [api.Outputs(v["w"], v["h"]) for v in views]
    arr = api.Batch.views([(v["avpls"], v["gb"], v["cam"], o) for v, o in zip(views, outs)])
    batch = api.Batch(ctx)
    batch.render(arr, lp, gp, cp)
    assert ctx.synchronize() == 0
    for o, r in zip(outs, ref):
        assert np.array_equal(o.result64.cpu().numpy(), r)
    # recorded once, replayed twice with one launch each
    batch.capture(arr, lp, gp, cp)
    assert ctx.synchronize() == 0
    for _ in range(2):
        for o in outs:
            o.result64.zero_()
        batch.launch()
        assert ctx.synchronize() == 0
        for o, r in zip(outs, ref):
            assert np.array_equal(o.result64.cpu().numpy(), r)
    batch.close()


def test_learned_cuts_record_and_replay(ctx, views):
    """The learned selection reads nothing back on the host, so a batch of learned cuts records into
    one graph; its images equal each view rendered on its own (up to the order in which a tile's
    accepted nodes are summed, which the selection's atomics leave open)."""
    from antiradiancecuts_b200 import learned

    model = learned.load_default_model(ctx)
    lp, gp, _ = _params()
    cp = learned.cut_params(model)
    ref = []
    for v in views:
        bvh = api.AvplBvh(ctx)
        L.check(ctx.lib.arc_lbvh_build(bvh.handle, C.byref(v["avpls"]), C.byref(lp)), "build")
        out = api.Outputs(v["w"], v["h"])
        api.gather_cut(ctx, bvh, v["avpls"], v["gb"], v["cam"], gp, cp, out)
        assert ctx.synchronize() == 0
        ref.append(out.result64.cpu().numpy().copy())
        bvh.close()
    outs = [api.Outputs(v["w"], v["h"]) for v in views]
    arr = api.Batch.views([(v["avpls"], v["gb"], v["cam"], o) for v, o in zip(views, outs)])
    batch = api.Batch(ctx)
    batch.capture(arr, lp, gp, cp)
    assert ctx.synchronize() == 0
    for _ in range(2):
        for o in outs:
            o.result64.zero_()
        batch.launch()
        assert ctx.synchronize() == 0
        for o, r in zip(outs, ref):
            assert H.rel_rmse(o.result64.cpu().numpy(), r) < 1e-6
    batch.close()
    model.close()


def test_device_errors_of_a_lane_reach_the_batch(ctx, views):
    """A view whose G-buffer names a material past the table: the lane that renders it reports
    ARC_DEVERR_BAD_MATERIAL into the owner context's error word."""
    lp, gp, cp = _params()
    v = views[1]
    nrm = v["gb"].nrm.clone()
    nrm[0, 0, 3] = 60.0
    gb = api.GBuffer(None, None, size=(v["w"], v["h"]))
    gb.pos.copy_(v["gb"].pos)
    gb.nrm.copy_(nrm)
    out = api.Outputs(v["w"], v["h"])
    arr = api.Batch.views([(v["avpls"], gb, v["cam"], out)])
    batch = api.Batch(ctx)
    batch.render(arr, lp, gp, cp)
    assert ctx.synchronize() & L.ARC_DEVERR_BAD_MATERIAL
    batch.render(api.Batch.views([(v["avpls"], v["gb"], v["cam"], out)]), lp, gp, cp)
    assert ctx.synchronize() == 0  # the lane's word was cleared when it was folded in
    batch.close()


def test_autotuner_picks_a_shape_and_makes_it_the_default(ctx, views):
    v = max(views, key=lambda x: x["w"] * x["h"])
    gp = api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    out = api.Outputs(v["w"], v["h"])
    best, times = api.autotune_bruteforce(ctx, v["avpls"], v["gb"], v["cam"], gp, out)
    assert ctx.synchronize() == 0
    assert 0 <= best < len(times) and (times > 0).all() and times[best] == times.min()
    imgs = {}
    for cfg in (-1, best, 0):
        o = api.Outputs(v["w"], v["h"])
        api.gather_bruteforce(ctx, v["avpls"], v["gb"], v["cam"], api.gather_params(L.ARC_AR_CONE, 30.0, 0.01,
                                                                                       tile_config=cfg), o)
        assert ctx.synchronize() == 0
        imgs[cfg] = o.result64.cpu().numpy()
    L.check(ctx.lib.arc_context_set_tile_config(ctx.handle, -1), "set_tile_config")  # back to the built-in one
    assert np.array_equal(imgs[-1], imgs[best])  # the tuned shape was the default
    assert H.rel_rmse(imgs[0], imgs[best]) < 2e-5


def test_autotuner_cache_applies_a_stored_shape_without_timing(ctx, views, tmp_path):
    v = views[0]
    gp = api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    out = api.Outputs(v["w"], v["h"])
    cache = api.TuningCache(str(tmp_path / "autotune.json"))
    best, times = api.autotune_bruteforce(ctx, v["avpls"], v["gb"], v["cam"], gp, out, cache=cache)
    assert ctx.synchronize() == 0
    cache.save()
    L.check(ctx.lib.arc_context_set_tile_config(ctx.handle, -1), "set_tile_config")
    again = api.TuningCache(cache.path)
    best2, times2 = api.autotune_bruteforce(ctx, v["avpls"], v["gb"], v["cam"], gp, out, cache=again)
    assert best2 == best and len(times2) == len(times)
    o1, o2 = api.Outputs(v["w"], v["h"]), api.Outputs(v["w"], v["h"])
    api.gather_bruteforce(ctx, v["avpls"], v["gb"], v["cam"], gp, o1)  # the cached shape is the default
    api.gather_bruteforce(ctx, v["avpls"], v["gb"], v["cam"], api.gather_params(L.ARC_AR_CONE, 30.0, 0.01,
                                                                               tile_config=best), o2)
    assert ctx.synchronize() == 0
    assert np.array_equal(o1.result64.cpu().numpy(), o2.result64.cpu().numpy())
    L.check(ctx.lib.arc_context_set_tile_config(ctx.handle, -1), "set_tile_config")
