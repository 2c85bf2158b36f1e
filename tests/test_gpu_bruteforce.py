"""Brute-force gather on the GPU against the FP64 oracle (parity)."""
import json
import os

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu

# Tolerances (FP32 terms, compensated sums, FP64 combine vs the FP64 oracle):
#   relative RMSE per channel <= 2e-5, and per pixel |err| <= 1e-4 * (|rad| + |antirad|) for all
#   but 0.1% of pixels.  With cone antiradiance the FP32 test d^.w > cos(h) and the oracle's FP64
#   acos(d^.w) < h classify a few pairs that lie within rounding of the cone boundary
#   differently; each such pair moves one pixel by a whole A * G_A term, so the cone mode's image
#   tolerance is relative RMSE <= 2e-4 (antiradiance alone <= 1e-3), with the same per-pixel bound.
REL_RMSE = 2e-5
CONE_REL_RMSE = 2e-4
PIX_TOL = 1e-4
NAIVE_REL_RMSE = 1e-4

_ORACLE_CACHE = {}


def _oracle(d, ar, clamp, half, disk_r):
    key = (id(d), ar, clamp, half, disk_r)
    if key not in _ORACLE_CACHE:
        px = np.arange(d["pos"].shape[0] * d["pos"].shape[1])
        _ORACLE_CACHE[key] = O.gather_fp64(d["pos"], d["nrm"], px, d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"],
                                           O.params(ar, half, clamp, disk_r))
    return _ORACLE_CACHE[key]


def _run(ctx, d, prm):
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    gb = api.GBuffer(d["pos"], d["nrm"])
    H_, W_ = d["pos"].shape[:2]
    out = api.Outputs(W_, H_)
    api.gather_bruteforce(ctx, dv, gb, d["cam"], prm, out)
    assert ctx.synchronize() == 0
    return out


@pytest.mark.parametrize("ar", [L.ARC_AR_NONE, L.ARC_AR_DISK, L.ARC_AR_CONE])
@pytest.mark.parametrize("prec", [L.ARC_PREC_KAHAN, L.ARC_PREC_KAHAN_STRICT, L.ARC_PREC_NAIVE, L.ARC_PREC_FP64])
def test_bruteforce_room_256_4k(ctx, ar, prec):
    d = H.workload("room_256_4k")
    w = d["w"]
    disk_r = H.disk_radius(d["desc"])
    prm = api.gather_params(ar, w.cone_half_angle_deg, w.dist_clamp, disk_r, precision=prec)
    out = _run(ctx, d, prm)
    rad, arr, res = _oracle(d, ar, w.dist_clamp, w.cone_half_angle_deg, disk_r)
    got = out.result64.cpu().numpy().reshape(-1, 3)
    err = H.rel_rmse(got, res)
    tol = NAIVE_REL_RMSE if prec == L.ARC_PREC_NAIVE else REL_RMSE
    if ar == L.ARC_AR_CONE and prec != L.ARC_PREC_FP64:
        tol = CONE_REL_RMSE
    assert err < tol, f"relative RMSE {err}"
    pe = H.pixel_rel_err(got, res, np.abs(rad) + np.abs(arr))
    assert np.mean(pe > PIX_TOL) <= 1e-3, f"max pixel error {pe.max()}"
    # float4 planes agree with the FP64 plane and carry w = 1
    r4 = out.result.cpu().numpy()
    assert np.allclose(r4[..., :3].reshape(-1, 3), got, rtol=1e-6, atol=1e-6 * np.abs(got).max())
    assert np.all(r4[..., 3] == 1.0)
    if ar != L.ARC_AR_NONE:
        gar = out.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3)
        assert H.rel_rmse(gar, arr) < (1e-3 if ar == L.ARC_AR_CONE else 1e-4)


@pytest.mark.parametrize("tile_config", list(range(8)))
def test_tile_shapes_agree(ctx, tile_config):
    d = H.workload("room_256_4k", 100, 77, 1500)  # ragged image and AVPL count
    w = d["w"]
    ref = _run(ctx, d, api.gather_params(L.ARC_AR_CONE, 30.0, w.dist_clamp, tile_config=2)).result64.cpu().numpy()
    got = _run(ctx, d, api.gather_params(L.ARC_AR_CONE, 30.0, w.dist_clamp, tile_config=tile_config)).result64
    got = got.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
    _, _, res = _oracle(d, L.ARC_AR_CONE, w.dist_clamp, 30.0, 0.0)
    assert H.rel_rmse(got.reshape(-1, 3), res) < CONE_REL_RMSE


def _kat_case_inputs(c):
    from antiradiancecuts_b200.scene import AVPL_DTYPE

    pos = np.array([[c["pixel_pos"] + [1.0]]], np.float32)
    nrm = np.array([[c["pixel_nrm"] + [float(c["pixel_mat"])]]], np.float32)
    a = np.zeros(1, AVPL_DTYPE)
    a["position"], a["normal"], a["incDirection"] = c["avpl_pos"], c["avpl_nrm"], c["avpl_w"]
    a["incRadiance"], a["antiradiance"] = c["L"], c["A"]
    a["materialIndex"], a["bounce"] = c["avpl_mat"], 2
    mats = (L.ArcMaterial * 3)()
    for i in range(3):
        mats[i].diffuse = L.f3(c["materials"][i])
        mats[i].specular = L.f3(c["specular"][i])
        mats[i].exponent = c["exponent"][i]
    return pos, nrm, a, mats


@pytest.mark.parametrize("prec", [L.ARC_PREC_KAHAN, L.ARC_PREC_FP64])
def test_known_answer_cases(ctx, prec):
    with open(os.path.join(GOLDEN, "gather_kat.json")) as f:
        cases = json.load(f)
    for c in cases:
        pos, nrm, a, mats = _kat_case_inputs(c)
        ctx.upload_materials(mats)
        dv = ctx.upload_avpls(a)
        gb = api.GBuffer(pos, nrm)
        out = api.Outputs(1, 1)
        prm = api.gather_params(c["ar_kind"], c["half_angle_deg"], c["clamp"], c.get("disk_radius", 0.0),
                                precision=prec)
        api.gather_bruteforce(ctx, dv, gb, c["cam"], prm, out)
        assert ctx.synchronize() == 0
        got_rad = out.radiance.cpu().numpy()[0, 0, :3]
        got_ar = out.antiradiance.cpu().numpy()[0, 0, :3]
        np.testing.assert_allclose(got_rad, c["rad"], rtol=2e-5, atol=1e-7, err_msg=c["name"])
        np.testing.assert_allclose(got_ar, c["ar"], rtol=2e-5, atol=1e-7, err_msg=c["name"])


def test_zero_avpls_gives_zero(ctx):
    d = H.workload("room_256_4k", 32, 32, 16)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"][:0])
    out = api.Outputs(32, 32)
    api.gather_bruteforce(ctx, dv, api.GBuffer(d["pos"], d["nrm"]), d["cam"], api.gather_params(), out)
    assert ctx.synchronize() == 0
    assert np.all(out.result64.cpu().numpy() == 0)


def test_bad_material_index_sets_error_bit(ctx):
    d = H.workload("room_256_4k", 16, 16, 64)
    nrm = d["nrm"].copy()
    nrm[3, 3, 3] = 60.0  # beyond the uploaded materials
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    out = api.Outputs(16, 16)
    api.gather_bruteforce(ctx, dv, api.GBuffer(d["pos"], nrm), d["cam"], api.gather_params(), out)
    word = ctx.synchronize()
    assert word & L.ARC_DEVERR_BAD_MATERIAL
    assert np.all(out.result64.cpu().numpy()[3, 3] == 0)


def test_invalid_arguments(ctx):
    d = H.workload("room_256_4k", 16, 16, 64)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    out = api.Outputs(16, 16)
    prm = api.gather_params(L.ARC_AR_DISK, disk_radius=0.0)
    with pytest.raises(L.ArcError) as e:
        api.gather_bruteforce(ctx, dv, api.GBuffer(d["pos"], d["nrm"]), d["cam"], prm, out)
    assert e.value.status == L.ARC_ERR_INVALID_ARG
