"""The FP64 MLP oracle's gradient against central finite differences (no GPU)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def test_num_params():
    assert M.NUM_PARAMS == 9473


@pytest.mark.parametrize("loss", ["bce", "squared"])
def test_gradient_matches_finite_differences(loss):
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, M.NUM_PARAMS)
    x = rng.normal(0, 1, (40, 16))
    lab = (rng.random(40) > 0.5).astype(np.float64) if loss == "bce" else rng.normal(-8, 3, 40)
    w = rng.random(40) + 0.5
    _, g = M.loss_and_grad(p, x, lab, w, loss=loss)
    idx = rng.choice(M.NUM_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, x, lab, w, loss=loss)[0] - M.loss_and_grad(pm, x, lab, w, loss=loss)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
