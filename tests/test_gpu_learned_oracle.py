"""The learned cut's inputs against the CPU oracle: the 16 features and the refine/accept labels of
every training sample (arc_cut_training_samples against oracle_training_samples, whose exact node
contributions are FP64 sums over each node's leaves), and the learned selection itself against the
oracle's level-by-level walk with the network restated at the kernels' BF16 rounding points.

Tolerances: the GPU computes the features with the hardware's approximate log2, square root,
reciprocal square root and division and stores them as BF16, so a feature may differ from the
oracle's correctly rounded FP32 value by one BF16 step (2^-7 relative) plus 2e-3; features 12 and
13 are logs of |rad - rad_l - rad_r| (a difference that can cancel to rounding noise) and are
compared where the difference is at least 1e-3 of the sum of the magnitudes.  Labels agree except
where the node's error lies within 1% of the threshold delta; errors agree to 1% + 2e-6 of the tile
value.  A learned-cut tile may differ from the oracle's only if one of its scored nodes has a logit
within 0.1 of the threshold, the lists differ in at most 2% of their nodes, and the two cuts'
images agree to 1e-3 relative RMSE (the hardware tanh and the features' approximate operations
are restated only up to their rounding, so a near-threshold decision may flip)."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api, learned
from oracle import oracle as O

pytestmark = pytest.mark.gpu

W, HGT, N = 160, 96, 16384
EPS, K, BAND, DELTA = learned.PREACCEPT_EPS, learned.PREACCEPT_K, learned.PREACCEPT_BAND, learned.LABEL_DELTA
CONE, CLAMP = 30.0, 0.01


@pytest.fixture(scope="module")
def scene_(ctx):
    d = H.workload("boxes2_720p_64k", W, HGT, N)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    bvh = api.AvplBvh(ctx)
    bvh.build(dv)
    assert ctx.synchronize() == 0
    tree = O.build_tree(d["avpls"], d["dif"])
    gtree = bvh.host_arrays()
    for k in ("left", "right", "records", "bounds", "dirstat"):
        assert np.array_equal(tree[k].view(np.uint8), gtree[k].view(np.uint8)), k
    return d, bvh, tree, api.GBuffer(d["pos"], d["nrm"])


def _gpu_samples(ctx, bvh, gb, d, capacity=2_000_000):
    import torch

    prm = api.gather_params(L.ARC_AR_CONE, CONE, CLAMP)
    cut = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=EPS, ar_uncertain_factor=K, mlp_band=BAND)
    feats = torch.empty((capacity, 16), dtype=torch.bfloat16, device="cuda")
    labels = torch.empty(capacity, dtype=torch.float32, device="cuda")
    errs = torch.empty(capacity, dtype=torch.float32, device="cuda")
    keys = torch.empty((capacity, 2), dtype=torch.int32, device="cuda")
    count = C.c_int32()
    gv = gb.view()
    L.check(ctx.lib.arc_cut_training_samples(ctx.handle, bvh.handle, C.byref(gv), L.f3(d["cam"]), C.byref(prm),
                                             C.byref(cut), DELTA, C.c_void_p(feats.data_ptr()),
                                             C.c_void_p(labels.data_ptr()), C.c_void_p(errs.data_ptr()),
                                             C.c_void_p(keys.data_ptr()), capacity, C.byref(count)),
            "arc_cut_training_samples")
    assert ctx.synchronize() == 0
    k = count.value
    assert 0 < k < capacity
    return (keys[:k].cpu().numpy(), feats[:k].float().cpu().numpy(), labels[:k].cpu().numpy(),
            errs[:k].cpu().numpy())


def _index(keys):
    return {(int(t), int(n)): i for i, (t, n) in enumerate(keys)}


def test_training_features_and_labels_match_oracle(ctx, scene_):
    d, bvh, tree, gb = scene_
    gk, gf, gl, ge = _gpu_samples(ctx, bvh, gb, d)
    ok, of, ol, oe = O.training_samples(d["pos"], d["nrm"], tree, d["dif"], EPS, CLAMP, 2, CONE, BAND, DELTA,
                                        ar_uncertain=K, capacity=1 << 22)
    assert len(ok) < 1 << 22
    gi, oi = _index(gk), _index(ok)
    assert len(gi) == len(gk) and len(oi) == len(ok), "a (tile, node) pair was sampled twice"
    common = sorted(set(gi) & set(oi))
    # a label decided the other way changes which children are walked: the sets differ only there
    assert len(common) >= 0.99 * max(len(gi), len(oi)), (len(gi), len(oi), len(common))
    g = np.array([gi[c] for c in common])
    o = np.array([oi[c] for c in common])
    F, R = gf[g], of[o]
    # labels and errors
    near = np.abs(oe[o] / DELTA - 1.0) < 1e-2
    lab_bad = (gl[g] != ol[o]) & ~near
    assert not lab_bad.any(), f"{lab_bad.sum()} labels differ away from the threshold"
    np.testing.assert_allclose(ge[g], oe[o], rtol=1e-2, atol=2e-6)
    # flags and depth exactly
    for j in (8, 9, 14):
        np.testing.assert_array_equal(F[:, j], R[:, j], err_msg=f"feature {j}")
    # features with a correctly rounded counterpart: one BF16 step + 2e-3
    tol = np.abs(R) * 2.0 ** -7 + 2e-3
    for j in (0, 1, 2, 3, 4, 5, 6, 7, 10, 11, 15):
        bad = np.abs(F[:, j] - R[:, j]) > tol[:, j]
        assert not bad.any(), (j, F[bad, j][:5], R[bad, j][:5])
    # the lookahead features where the difference they take the log of is well conditioned
    depth = np.rint(R[:, 14] * 32).astype(np.int32)
    trec = O.tile_records(d["pos"], d["nrm"], tree, d["dif"], EPS, CLAMP)
    keys = np.array(common, np.int32)
    _, RF, aux = O.pair_features(trec, keys[:, 0], keys[:, 1], depth, tree, CLAMP, 2, CONE, ar_uncertain=K)
    np.testing.assert_array_equal(RF, R)  # the walk's features are the pair features
    for j, (a, b) in ((12, (0, 1)), (13, (2, 3))):
        cond = aux[:, a] >= 1e-3 * aux[:, b]
        bad = cond & (np.abs(F[:, j] - R[:, j]) > tol[:, j] + 2e-3)
        assert not bad.any(), (j, F[bad, j][:5], R[bad, j][:5])
        assert cond.mean() > 0.5
    print(f"{len(common)} common samples ({len(gi)} GPU, {len(oi)} oracle), "
          f"{(gl[g] != ol[o]).sum()} labels at the threshold")


def test_learned_selection_matches_oracle(ctx, scene_):
    d, bvh, tree, gb = scene_
    model = learned.load_default_model(ctx)
    params = model.params()
    thr = float(np.log(model.threshold / (1.0 - model.threshold)))
    prm = api.gather_params(L.ARC_AR_CONE, CONE, CLAMP)
    out = api.Outputs(W, HGT)
    api.gather_cut(ctx, bvh, None, gb, d["cam"], prm, learned.cut_params(model), out)
    assert ctx.synchronize() == 0
    gcuts = api.last_cut(ctx)
    ocuts, scored = O.learned_cut(d["pos"], d["nrm"], tree, d["dif"], params, model.eps, K, model.band, thr, CLAMP,
                                  2, CONE, act=model.act)
    assert len(scored) > 1000
    differ = [t for t in range(len(gcuts)) if not np.array_equal(gcuts[t], ocuts[t])]
    close = {int(t) for t, _, y in scored if abs(y - thr) < 0.1}
    assert set(differ) <= close, sorted(set(differ) - close)[:10]
    # a decision taken the other way swaps a node for its subtree's cut: the lists differ in few nodes
    total = sum(len(g) for g in gcuts)
    swapped = sum(len(np.setxor1d(g, o)) for g, o in zip(gcuts, ocuts))
    assert swapped <= 0.02 * total, (swapped, total)
    # the image is the oracle's evaluation of the GPU's own lists
    _, _, ref = O.eval_cut(d["pos"], d["nrm"], tree, gcuts, d["dif"], 2, CONE, CLAMP)
    img = out.result64.cpu().numpy().reshape(-1, 3)
    assert H.rel_rmse(img, ref) < 2e-5
    # and the oracle's own cut renders the same image up to those swaps
    _, _, oimg = O.eval_cut(d["pos"], d["nrm"], tree, ocuts, d["dif"], 2, CONE, CLAMP)
    assert H.rel_rmse(img, oimg) < 1e-3
    print(f"{len(scored)} scored rows, {len(differ)} of {len(gcuts)} tiles differ (all near the threshold), "
          f"{swapped} of {total} nodes swapped")
    model.close()
