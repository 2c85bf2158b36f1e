"""PFM and Radiance HDR export (host functions of the library) read back by independent readers,
and the reference's image-error formula on a hand-computed case."""
import numpy as np
import pytest

import image_io as IO
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api


def _plane(h, w, seed):
    rng = np.random.default_rng(seed)
    a = np.zeros((h, w, 4), np.float32)
    a[..., :3] = rng.lognormal(-1.0, 2.0, (h, w, 3)).astype(np.float32)
    a[0, 0, :3] = 0.0  # black
    a[-1, -1, :3] = (1e-6, 2e3, 0.5)  # wide dynamic range in one pixel
    a[..., 3] = 1.0
    return a


@pytest.mark.parametrize("shape", [(5, 3), (17, 40), (64, 300)])
def test_pfm_round_trip(tmp_path, shape):
    a = _plane(*shape, seed=shape[1])
    p = tmp_path / "x.pfm"
    api.export_pfm(p, a)
    assert np.array_equal(IO.read_pfm(str(p)), a[..., :3])
    head = p.read_bytes()[:32]
    assert head.startswith(f"PF\n{shape[1]} {shape[0]}\n-1.0\n".encode())


@pytest.mark.parametrize("shape", [(5, 3), (17, 40), (64, 300)])  # flat and run-length scanlines
def test_hdr_round_trip(tmp_path, shape):
    a = _plane(*shape, seed=shape[0])
    p = tmp_path / "x.hdr"
    api.export_hdr(p, a)
    got = IO.read_hdr(str(p))
    ref = a[..., :3]
    # RGBE keeps 8 bits of mantissa relative to the pixel's largest channel
    tol = np.max(ref, axis=2, keepdims=True) / 128.0
    assert np.all(np.abs(got - ref) <= tol)
    assert np.all(got[0, 0] == 0.0)


def test_export_reports_unwritable_path(tmp_path):
    a = _plane(4, 4, 0)
    lib = L.load()
    for fn in (lib.arc_export_pfm, lib.arc_export_hdr):
        bad = str(tmp_path / "missing" / "x.out")
        st = fn(bad.encode(), a.ctypes.data, 4, 4, 4)
        assert st == L.ARC_ERR_IO
        msg = lib.arc_last_error().decode()
        assert "cannot open" in msg and bad in msg and "No such file" in msg


def test_reference_error_formula():
    # one pixel, d = (1, 2, 20): squared (1, 4, 400 -> clamped 100), e = (1, 2, 10)
    ref = np.array([[[1.0, 2.0, 20.0, 1.0]]], np.float32)
    img = np.zeros_like(ref)
    err, e = IO.reference_error(ref, img)
    assert np.allclose(e, [1.0, 2.0, 10.0]) and err == pytest.approx((1.0 * 2.0 + 10.0) / 3.0)
    err2, _ = IO.reference_error(ref, img, as_written=False)
    assert err2 == pytest.approx(13.0 / 3.0)
