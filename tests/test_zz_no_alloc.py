"""arc_gather_bruteforce_noalloc: the brute-force gather for callers that may not allocate device
memory through the library (hosts with a fixed, pre-allocated device budget, where a cudaMalloc
mid-frame could synchronise the device and stall the frame).  Its result must equal the regular
arc_gather_bruteforce on the same inputs, call after call, while the process's free device memory
stays unchanged.  Collected last on purpose (file name), so a failure here leaves every other
test already run."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api

pytestmark = pytest.mark.gpu

REL_RMSE = 2e-5  # the brute-force tests' tolerance
W, HT = 96, 64


def _call(ctx, mats, dv, gb, cam, prm, out):
    gv, ov = gb.view(), out.view()
    word = C.c_uint32(0xFFFFFFFF)
    st = ctx.lib.arc_gather_bruteforce_noalloc(C.c_void_p(ctx.stream.cuda_stream), mats, len(mats), C.byref(dv),
                                               C.byref(gv), L.f3(cam), C.byref(prm), C.byref(ov), C.byref(word))
    return st, word.value


def _own_copy(ctx, av):
    """Device SoA arrays of `av` that outlive the context's next upload (which reuses its buffers)."""
    import torch

    dv = ctx.upload_avpls(av)
    keep = {}
    for name in ("position", "normal", "incDirection", "incRadiance", "antiradiance"):
        t = torch.from_numpy(np.ascontiguousarray(av[name], np.float32)).cuda()
        keep[name] = t
        setattr(dv, name, t.data_ptr())
    for name in ("materialIndex", "bounce"):
        t = torch.from_numpy(np.ascontiguousarray(av[name], np.int32)).cuda()
        keep[name] = t
        setattr(dv, name, t.data_ptr())
    return dv, keep


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    ctx = api.Context(0)
    d = H.workload("room_256_4k", W, HT, 3000)
    gb = api.GBuffer(d["pos"], d["nrm"])
    prm = api.gather_params(L.ARC_AR_CONE, d["w"].cone_half_angle_deg, d["w"].dist_clamp)
    ctx.upload_materials(d["mats"])
    cases = [d["avpls"], d["avpls"][:1234]]  # second call: fewer AVPLs, so stale records would show
    refs, outs, dvs = [], [], []
    for av in cases:
        dvs.append(_own_copy(ctx, av))
        ref = api.Outputs(W, HT)
        api.gather_bruteforce(ctx, dvs[-1][0], gb, d["cam"], prm, ref)  # also loads the gather kernels
        assert ctx.synchronize() == 0
        refs.append(ref.result64.cpu().numpy().copy())
        outs.append(api.Outputs(W, HT))
    torch.cuda.synchronize()
    free = [torch.cuda.mem_get_info()[0]]  # before the first allocation-free call
    for i, (dv, _) in enumerate(dvs):
        st, word = _call(ctx, d["mats"], dv, gb, d["cam"], prm, outs[i])
        assert st == L.ARC_OK, L.load().arc_last_error()
        assert word == 0
        torch.cuda.synchronize()
        got = outs[i].result64.cpu().numpy()
        assert H.rel_rmse(got, refs[i]) < REL_RMSE
        np.testing.assert_allclose(got, refs[i], rtol=1e-6, atol=1e-9 * np.abs(refs[i]).max())
        free.append(torch.cuda.mem_get_info()[0])
    assert free[0] == free[1] == free[2], f"device memory changed across allocation-free calls: {free}"
    ctx.close()


# (ar_kind, precision, specular material, bad material index)
CASES = [
    (L.ARC_AR_NONE, L.ARC_PREC_KAHAN, False, False),
    (L.ARC_AR_DISK, L.ARC_PREC_KAHAN, False, False),
    (L.ARC_AR_CONE, L.ARC_PREC_NAIVE, False, False),
    (L.ARC_AR_CONE, L.ARC_PREC_FP64, False, False),
    (L.ARC_AR_CONE, L.ARC_PREC_KAHAN, True, False),   # Phong material: the general kernel
    (L.ARC_AR_CONE, L.ARC_PREC_KAHAN, False, True),   # a pixel names a material past the table
]


@pytest.mark.parametrize("ar_kind,precision,specular,bad_material", CASES)
def test_noalloc_variants_match_regular_entry_point(ar_kind, precision, specular, bad_material):
    ctx = api.Context(0)
    d = H.workload("room_256_4k", W, HT, 2000)
    mats = (L.ArcMaterial * len(d["mats"]))(*d["mats"])
    if specular:
        mats[2].specular = L.ArcFloat3(0.3, 0.3, 0.3)
        mats[2].exponent = 20.0
    nrm = d["nrm"].copy()
    if bad_material:
        nrm[5, 7, 3] = 60.0
    gb = api.GBuffer(d["pos"], nrm)
    prm = api.gather_params(ar_kind, d["w"].cone_half_angle_deg, d["w"].dist_clamp,
                            disk_radius=H.disk_radius(d["desc"]), precision=precision)
    ctx.upload_materials(mats)
    dv, _keep = _own_copy(ctx, d["avpls"])
    ref = api.Outputs(W, HT)
    api.gather_bruteforce(ctx, dv, gb, d["cam"], prm, ref)
    ref_word = ctx.synchronize()
    want = ref.result64.cpu().numpy().copy()
    for _ in range(2):
        out = api.Outputs(W, HT)
        st, word = _call(ctx, mats, dv, gb, d["cam"], prm, out)
        assert st == L.ARC_OK, L.load().arc_last_error()
        assert word == ref_word
        assert bool(word & L.ARC_DEVERR_BAD_MATERIAL) == bad_material
        got = out.result64.cpu().numpy()
        assert H.rel_rmse(got, want) < REL_RMSE
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-9 * np.abs(want).max())
    ctx.close()


def test_noalloc_rejects_more_avpls_than_its_scratch_holds():
    ctx = api.Context(0)
    d = H.workload("room_256_4k", 16, 16, 64)
    gb = api.GBuffer(d["pos"], d["nrm"])
    dv = ctx.upload_avpls(d["avpls"])
    dv.numAvpls = 65537  # no GPU work happens: the size check comes first
    st, _ = _call(ctx, d["mats"], dv, gb, d["cam"], api.gather_params(), api.Outputs(16, 16))
    assert st == L.ARC_ERR_INVALID_ARG
    assert b"65536" in L.load().arc_last_error()
    ctx.close()
