"""Accumulation over frames, normalisation by the path count and the image error on the device
(arc_accumulate, arc_accum_normalize, arc_image_error) against NumPy restatements."""
import numpy as np
import pytest

import image_io as IO
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api

pytestmark = pytest.mark.gpu


def test_accumulate_and_normalize(ctx):
    import torch

    h, w = 37, 53
    rng = np.random.default_rng(1)
    acc = api.Accumulator(ctx, w, h)
    ref = np.zeros((h, w, 9))
    frames = []
    for k in range(3):
        out = api.Outputs(w, h)
        for j, plane in enumerate((out.result, out.radiance, out.antiradiance)):
            v = rng.normal(0.0, 1.0 + k, (h, w, 4)).astype(np.float32)
            plane.copy_(torch.from_numpy(v))
            ref[..., 3 * j:3 * j + 3] += v[..., :3].astype(np.float64)
        frames.append(out)
        acc.add(out, paths=1000)
    norm = acc.normalize(api.Outputs(w, h))
    assert ctx.synchronize() == 0
    assert np.array_equal(acc.sum.cpu().numpy(), ref)  # FP64 sums of FP32 values: exact here
    inv = 1.0 / 3000.0
    for j, plane in enumerate((norm.result, norm.radiance, norm.antiradiance)):
        got = plane.cpu().numpy()
        assert np.array_equal(got[..., :3], (ref[..., 3 * j:3 * j + 3] * inv).astype(np.float32))
        assert np.all(got[..., 3] == 1.0)
    assert np.array_equal(norm.result64.cpu().numpy(), ref[..., :3] * inv)
    # no paths: zeros, as Normalize with a zero factor
    z = acc.normalize(api.Outputs(w, h), paths=0)
    acc.clear()
    assert ctx.synchronize() == 0
    assert not z.result[..., :3].any() and not acc.sum.any()


@pytest.mark.parametrize("metric", [L.ARC_ERROR_REFERENCE, L.ARC_ERROR_RMSE])
def test_image_error_matches_reference_formula(ctx, metric):
    import torch

    h, w = 61, 89
    rng = np.random.default_rng(metric + 5)
    a = rng.normal(0.0, 3.0, (h, w, 4)).astype(np.float32)
    b = a + rng.normal(0.0, 0.5, (h, w, 4)).astype(np.float32)
    b[3, 4, 1] += 50.0  # a difference the clamp at 100 cuts
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    err, ch = api.image_error(ctx, ta, tb, metric)
    assert ctx.synchronize() == 0
    ref_err, ref_ch = IO.reference_error(a, b, as_written=metric == L.ARC_ERROR_REFERENCE)
    assert np.allclose(ch, ref_ch, rtol=1e-12) and err == pytest.approx(ref_err, rel=1e-12)
