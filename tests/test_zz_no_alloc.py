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


def _call(ctx, mats, dv, gb, cam, prm, out):
    gv, ov = gb.view(), out.view()
    word = C.c_uint32(0xFFFFFFFF)
    st = ctx.lib.arc_gather_bruteforce_noalloc(C.c_void_p(ctx.stream.cuda_stream), mats, len(mats), C.byref(dv),
                                               C.byref(gv), L.f3(cam), C.byref(prm), C.byref(ov), C.byref(word))
    return st, word.value


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    ctx = api.Context(0)
    d = H.workload("room_256_4k", 96, 64, 3000)
    gb = api.GBuffer(d["pos"], d["nrm"])
    prm = api.gather_params(L.ARC_AR_CONE, d["w"].cone_half_angle_deg, d["w"].dist_clamp)
    ctx.upload_materials(d["mats"])
    cases = [d["avpls"], d["avpls"][:1234]]  # second call: fewer AVPLs, so stale records would show
    refs, outs, dvs = [], [], []
    for av in cases:
        dv = ctx.upload_avpls(av)
        # keep each upload alive: the context reuses its AVPL buffer, so copy into tensors
        keep = {}
        for name in ("position", "normal", "incDirection", "incRadiance", "antiradiance"):
            t = torch.from_numpy(np.ascontiguousarray(av[name], np.float32)).cuda()
            keep[name] = t
            setattr(dv, name, t.data_ptr())
        for name in ("materialIndex", "bounce"):
            t = torch.from_numpy(np.ascontiguousarray(av[name], np.int32)).cuda()
            keep[name] = t
            setattr(dv, name, t.data_ptr())
        dvs.append((dv, keep))
        ref = api.Outputs(96, 64)
        api.gather_bruteforce(ctx, dv, gb, d["cam"], prm, ref)
        assert ctx.synchronize() == 0
        refs.append(ref.result64.cpu().numpy().copy())
        outs.append(api.Outputs(96, 64))
    torch.cuda.synchronize()
    free = []
    for i, (dv, _) in enumerate(dvs):
        st, word = _call(ctx, d["mats"], dv, gb, d["cam"], prm, outs[i])
        assert st == L.ARC_OK, L.load().arc_last_error()
        assert word == 0
        torch.cuda.synchronize()
        got = outs[i].result64.cpu().numpy()
        assert H.rel_rmse(got, refs[i]) < REL_RMSE
        np.testing.assert_allclose(got, refs[i], rtol=1e-6, atol=1e-9 * np.abs(refs[i]).max())
        free.append(torch.cuda.mem_get_info()[0])
    assert free[0] == free[1], "device memory changed between allocation-free calls"
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
