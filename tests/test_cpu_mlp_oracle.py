"""The FP64 MLP oracle's gradient against central finite differences (no GPU)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def test_num_params():
    assert M.NUM_PARAMS == 9473


@pytest.mark.parametrize("act", ["gelu", "relu"])
@pytest.mark.parametrize("loss", ["bce", "squared"])
def test_gradient_matches_finite_differences(loss, act):
    """(ReLU's kink: a step of 1e-6 crosses it only where a pre-activation lies within 1e-6 of 0,
    which these seeded inputs do not hit.)"""
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, M.NUM_PARAMS)
    x = rng.normal(0, 1, (40, 16))
    lab = (rng.random(40) > 0.5).astype(np.float64) if loss == "bce" else rng.normal(-8, 3, 40)
    w = rng.random(40) + 0.5
    _, g = M.loss_and_grad(p, x, lab, w, loss=loss, act=act)
    idx = rng.choice(M.NUM_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, x, lab, w, loss=loss, act=act)[0]
              - M.loss_and_grad(pm, x, lab, w, loss=loss, act=act)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


@pytest.mark.parametrize("act", ["gelu", "relu", 0, 1])
def test_bf16_forward_follows_fp64_forward(act):
    """The BF16-rounding restatement (the folded form for GELU) is the same network as the FP64
    one up to BF16 rounding of inputs, weights and hidden activations."""
    rng = np.random.default_rng(9)
    p = rng.normal(0, 0.3, M.NUM_PARAMS).astype(np.float32).astype(np.float64)
    x = rng.normal(0, 1, (300, 16))
    y64, _ = M.forward(p, x, act)
    yb = M.forward_bf16(p, x, act)
    assert np.max(np.abs(yb - y64)) <= 3e-2 * max(1.0, np.abs(y64).max())
    with pytest.raises(ValueError):
        M.forward(p, x, "tanh")


def test_shipped_model_archive():
    """The shipped cut network: the archive fields a C / C++ host reads, the parameter count the
    library expects, finite weights, finite logits through the FP64 network, and the operating
    point it ships with is the one its calibration report chose on the validation scenes."""
    import json
    import os

    from antiradiancecuts_b200 import _lib as L
    from antiradiancecuts_b200 import learned

    z = np.load(learned.DEFAULT_MODEL)
    assert set(z.files) >= {"params", "loss", "threshold", "band", "eps"}
    act = int(z["act"]) if "act" in z.files else L.ARC_MLP_ACT_GELU
    assert act in (L.ARC_MLP_ACT_GELU, L.ARC_MLP_ACT_RELU)
    p = z["params"]
    assert p.dtype == np.float32 and p.shape == (M.NUM_PARAMS,)
    assert L.load().arc_mlp_num_params() == M.NUM_PARAMS == learned.NUM_PARAMS
    assert np.all(np.isfinite(p)) and np.abs(p).max() > 0
    assert int(z["loss"]) == L.ARC_MLP_LOSS_BCE
    rep = json.load(open(os.path.join(os.path.dirname(learned.DEFAULT_MODEL), "cutnet_calibration.json")))
    chosen = rep["chosen"]
    assert float(z["threshold"]) == pytest.approx(chosen["threshold"])
    assert float(z["band"]) == chosen["band"] and float(z["eps"]) == pytest.approx(chosen["eps"])
    assert max(chosen["worst_rel_rmse"][chosen["thresholds"].index(chosen["threshold"])], 0) <= rep["target_rel_rmse"]
    assert rep["seeds"] == list(learned.VALIDATION_SEEDS)
    x = np.random.default_rng(0).normal(0, 1, (256, 16))
    logits, _ = M.forward(p.astype(np.float64), x, act)
    assert np.all(np.isfinite(logits)) and np.std(logits) > 0
