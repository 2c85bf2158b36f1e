"""CPU checks of the oracle's restatement of the learned cut (features, labelling walk, selection):
its selection reduces to the analytic error-bound cut at both ends of the network's range, its
labelling walk samples exactly the nodes the selection would score, and its labels follow delta."""
import math

import numpy as np
import pytest

import helpers as H
from oracle import mlp_oracle as M
from oracle import oracle as O

EPS, K, BAND, CONE, CLAMP = 0.01, 16.0, 8.0, 30.0, 0.01


@pytest.fixture(scope="module")
def small():
    d = H.workload("boxes2_720p_64k", 64, 48, 4096)
    tree = O.build_tree(d["avpls"], d["dif"])
    return d, tree


def test_selection_ends_equal_error_bound_cuts(small):
    d, tree = small
    p = np.random.default_rng(0).standard_normal(M.NUM_PARAMS) * 0.1
    base, _, _ = O.tile_cut(d["pos"], d["nrm"], tree, d["dif"], EPS, CLAMP, 2, CONE, ar_uncertain=K)
    wide, _, _ = O.tile_cut(d["pos"], d["nrm"], tree, d["dif"], EPS * BAND, CLAMP, 2, CONE, ar_uncertain=K)
    always, s1 = O.learned_cut(d["pos"], d["nrm"], tree, d["dif"], p, EPS, K, BAND, -math.inf, CLAMP, 2, CONE)
    never, s2 = O.learned_cut(d["pos"], d["nrm"], tree, d["dif"], p, EPS, K, BAND, math.inf, CLAMP, 2, CONE)
    assert len(s1) > 0 and len(s2) > 0
    assert all(np.array_equal(a, b) for a, b in zip(base, always))
    assert all(np.array_equal(a, b) for a, b in zip(wide, never))


def test_labelling_walk_samples_what_the_selection_scores(small):
    """With every label "refine" (delta < 0) the walk visits what the always-refine selection scores;
    the pair features of those nodes are the walk's features."""
    d, tree = small
    keys, F, lab, err = O.training_samples(d["pos"], d["nrm"], tree, d["dif"], EPS, CLAMP, 2, CONE, BAND, -1.0,
                                           ar_uncertain=K)
    assert len(keys) > 100 and lab.min() == 1.0 and np.isfinite(F).all() and (err >= 0).all()
    p = np.zeros(M.NUM_PARAMS)
    _, scored = O.learned_cut(d["pos"], d["nrm"], tree, d["dif"], p, EPS, K, BAND, -math.inf, CLAMP, 2, CONE)
    assert {(int(t), int(n)) for t, n, _ in scored} == {(int(t), int(n)) for t, n in keys}
    trec = O.tile_records(d["pos"], d["nrm"], tree, d["dif"], EPS, CLAMP)
    depth = np.rint(F[:, 14] * 32).astype(np.int32)
    _, F2, _ = O.pair_features(trec, keys[:, 0], keys[:, 1], depth, tree, CLAMP, 2, CONE, ar_uncertain=K)
    np.testing.assert_array_equal(F, F2)


def test_labels_follow_delta(small):
    d, tree = small
    _, _, l1, e1 = O.training_samples(d["pos"], d["nrm"], tree, d["dif"], EPS, CLAMP, 2, CONE, BAND, 1e-4,
                                      ar_uncertain=K)
    _, _, l2, _ = O.training_samples(d["pos"], d["nrm"], tree, d["dif"], EPS, CLAMP, 2, CONE, BAND, 1e-1,
                                     ar_uncertain=K)
    assert l2.mean() < l1.mean()
    np.testing.assert_array_equal(l1 > 0.5, e1 > 1e-4)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0e-5, 65504.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0078125
    assert abs(r[3] / -3.0e-5 - 1) < 2 ** -8
    assert r[4] == 65536.0
