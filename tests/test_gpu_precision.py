"""Precision modes of the brute-force gather on the high-cancellation workload (16 random boxes,
cone 60 deg, clamp 0.005) on a small frame with the full 262,144 AVPLs per pixel, where summation
error shows, against the all-FP64 GPU image and the CPU FP64 oracle (precision_report.py makes the
full-size report)."""
import numpy as np
import pytest

import precision_report as P


@pytest.fixture(scope="module")
def results():
    return P.measure(width=128, height=72, num_avpls=262144, sample=256)


@pytest.mark.gpu
def test_fp64_gpu_matches_oracle(results):
    # FP64 throughout; the cone threshold itself is an FP32 cosf, so pairs on the cone boundary may
    # classify differently from the oracle's (measured: 4.7e-8 relative RMSE, 4.5e-6 max)
    rel, mx = results["vs_oracle"]["FP64"]
    assert rel.max() < 1e-6 and mx.max() < 1e-4, (rel, mx)


@pytest.mark.gpu
def test_compensated_sums_beat_naive(results):
    # measured: naive 2.6e-5 .. 7.6e-5, Kahan 5.4e-6 .. 8.6e-6 relative RMSE per channel
    naive = results["vs_fp64_gpu"]["NAIVE"][0]
    kahan = results["vs_fp64_gpu"]["KAHAN"][0]
    strict = results["vs_fp64_gpu"]["KAHAN_STRICT"][0]
    assert kahan.max() < 2e-5 and strict.max() < 2e-5, (kahan, strict)
    assert kahan.max() < 0.5 * naive.max() and strict.max() < 0.5 * naive.max(), (kahan, strict, naive)


def test_channel_errors_definition():
    ref = np.array([[1.0, 2.0, 0.0], [3.0, -4.0, 1.0]])
    x = ref + np.array([[0.1, 0.0, 0.0], [0.0, 0.0, 0.001]])
    rel, mx = P.channel_errors(x, ref)
    assert np.isclose(rel[0], np.sqrt(0.01 / 2) / np.sqrt(5.0))
    assert rel[1] == 0.0 and np.isclose(mx[0], 0.1) and np.isclose(mx[2], 0.001)
