"""Learned cut: the level-synchronous selection, its training samples, and the trained model."""
import ctypes as C
import os

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api, learned, scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu

W, HGT, N = 160, 96, 16384


@pytest.fixture(scope="module")
def scene_(ctx):
    d = H.workload("boxes2_720p_64k", W, HGT, N)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    bvh = api.AvplBvh(ctx)
    bvh.build(dv)
    assert ctx.synchronize() == 0
    return d, dv, bvh, bvh.host_arrays(), api.GBuffer(d["pos"], d["nrm"])


def _gather(ctx, d, bvh, gb, cut):
    prm = api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    h, w = d["pos"].shape[:2]
    out = api.Outputs(w, h)
    api.gather_cut(ctx, bvh, None, gb, d["cam"], prm, cut, out)
    assert ctx.synchronize() == 0
    return out.result64.cpu().numpy().reshape(-1, 3), api.last_cut(ctx)


def test_always_refine_equals_error_bound_cut(ctx, scene_):
    d, dv, bvh, tree, gb = scene_
    model = learned.Model(ctx, seed=3)
    img_b, cuts_b = _gather(ctx, d, bvh, gb, api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.01))
    img_l, cuts_l = _gather(ctx, d, bvh, gb, api.cut_params(L.ARC_CUT_LEARNED, error_bound=0.01,
                                                            model=model.handle.value, mlp_threshold=0.0))
    assert all(np.array_equal(a, b) for a, b in zip(cuts_b, cuts_l))
    assert H.rel_rmse(img_l, img_b) < 1e-6
    model.close()


@pytest.mark.parametrize("band", [4.0, 64.0])
def test_band_only_cut_equals_scaled_error_bound_cut(ctx, scene_, band):
    """With threshold 1 the network never refines, so the learned cut refines exactly the nodes whose
    bound exceeds band * tau: the error-bound cut at band * eps (powers of two scale exactly)."""
    d, dv, bvh, tree, gb = scene_
    model = learned.Model(ctx, seed=5, loss=L.ARC_MLP_LOSS_BCE)  # probability threshold 1: never refines
    eps = float(np.float32(0.01))
    img_b, cuts_b = _gather(ctx, d, bvh, gb, api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=eps * band))
    img_l, cuts_l = _gather(ctx, d, bvh, gb, api.cut_params(L.ARC_CUT_LEARNED, error_bound=eps, mlp_band=band,
                                                            model=model.handle.value, mlp_threshold=1.0))
    assert all(np.array_equal(a, b) for a, b in zip(cuts_b, cuts_l))
    assert H.rel_rmse(img_l, img_b) < 1e-6
    model.close()


def test_learned_cut_overflow_is_reported(ctx, scene_):
    """A cut pool too small for the cut: the selection keeps what fits, reports
    ARC_DEVERR_CUT_OVERFLOW in the device error word, and the frame still completes."""
    d, dv, bvh, tree, gb = scene_
    model = learned.Model(ctx, seed=6, loss=L.ARC_MLP_LOSS_BCE)
    cut = api.cut_params(L.ARC_CUT_LEARNED, error_bound=0.01, model=model.handle.value, mlp_threshold=0.0,
                         cut_pool_entries=2048)
    prm = api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    h, w = d["pos"].shape[:2]
    out = api.Outputs(w, h)
    api.gather_cut(ctx, bvh, None, gb, d["cam"], prm, cut, out)
    assert ctx.synchronize() & L.ARC_DEVERR_CUT_OVERFLOW
    # the next frame with room is unaffected
    img, _ = _gather(ctx, d, bvh, gb, api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.01))
    assert np.isfinite(img).all()
    model.close()


def test_learned_cut_evaluation_matches_oracle(ctx, scene_):
    d, dv, bvh, tree, gb = scene_
    model = learned.Model(ctx, seed=4)
    img, cuts = _gather(ctx, d, bvh, gb, api.cut_params(L.ARC_CUT_LEARNED, error_bound=0.01,
                                                        model=model.handle.value, mlp_threshold=0.5))
    _, _, ref = O.eval_cut(d["pos"], d["nrm"], tree, cuts, d["dif"], 2, 30.0, 0.01)
    assert H.rel_rmse(img, ref) < 2e-5
    # every tile's accepted nodes form a cut: no accepted node is an ancestor of another
    par = tree["parents"]
    n = len(tree["morton"])
    for c in cuts[:: max(1, len(cuts) // 40)]:
        s = set(int(x) for x in c)
        for x in c:
            p = par[x]
            while p != -1:
                assert (n + p) not in s
                p = par[n + p]
    model.close()


def test_training_samples(ctx):
    f, l, e = learned.scene_samples(ctx, 101, capacity=400000, width=96, height=64, num_avpls=8192, delta=5e-4)
    assert f.shape[0] > 100
    fl = f.float()
    assert bool(torch_isfinite(fl)) and set(np.unique(l.cpu().numpy())) <= {0.0, 1.0}
    f2, l2, _ = learned.scene_samples(ctx, 101, capacity=400000, width=96, height=64, num_avpls=8192, delta=5e-2)
    assert l2.mean().item() < l.mean().item()  # a looser bound refines less


def torch_isfinite(t):
    import torch

    return torch.isfinite(t).all().item()


@pytest.mark.skipif(not os.path.exists(learned.DEFAULT_MODEL), reason="no trained model")
@pytest.mark.parametrize("seed", [500, 501, 502])
def test_trained_model_beats_analytic_cut_on_held_out_scenes(ctx, seed):
    """Ablation at the evaluation scale (room variants 1920x1080 with 1,048,576 AVPLs, seeds that
    neither trained the network (100-163) nor chose its operating point (164-171)): the shipped
    network's cut against the analytic error-bound cut without it, both scored against the scene's
    all-FP64 GPU image (itself checked against the CPU oracle in test_gpu_bruteforce).  At the bound
    where the analytic cut stays within 1% relative RMSE on the validation scenes, the learned cut
    (its threshold also chosen there) must stay within 1% here, with at most 60% of the analytic
    cut's nodes."""
    import json

    eps = 0.002
    cal = os.path.join(os.path.dirname(learned.DEFAULT_MODEL), "cutnet_calibration.json")
    if os.path.exists(cal):
        eps = json.load(open(cal))["analytic"]["chosen"] or eps
    sc = learned.EvalScene(ctx, seed)
    pool = sc.tiles * 65536
    model = learned.load_default_model(ctx)
    an = sc.cut(api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=eps, ar_uncertain_factor=learned.PREACCEPT_K,
                               cut_pool_entries=pool), reps=1)
    lc = sc.cut(learned.cut_params(model, cut_pool_entries=pool), reps=1)
    print(f"seed {seed}: analytic {an}, learned {lc}")
    assert lc["rel_rmse"] <= 0.01
    assert lc["nodes_per_tile"] <= 0.6 * an["nodes_per_tile"]
    model.close()
    sc.close()
