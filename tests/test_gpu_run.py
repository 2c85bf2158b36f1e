"""CudaGather::run through the C ABI (arc_run): upload, optional LBVH + cut, antiradiance, combine."""
import math

import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api, scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("use_cuts", [0, 1])
def test_run_matches_oracle(ctx, use_cuts):
    d = H.workload("room_256_4k", 128, 128, 4096)
    gb = api.GBuffer(d["pos"], d["nrm"])
    g = api.CudaGather(ctx, gb, d["mats"])
    ext = scene.scene_extent(d["desc"])
    cfg = api.run_config(useLightCuts=use_cuts, ar_kind=L.ARC_AR_DISK, dist_clamp=0.01)
    out = g.run(d["avpls"], d["cam"], ext, cfg)
    got = out.result64.cpu().numpy().reshape(-1, 3)
    px = np.arange(128 * 128)
    r = 2.0 * ext / 100.0  # photonRadiusScale * sceneExtent / 100
    rad, ar, res = O.gather_fp64(d["pos"], d["nrm"], px, d["avpls"], d["dif"], d["spe"], d["ex"], d["cam"],
                                 O.params(1, 30.0, 0.01, r))
    if use_cuts == 0:
        assert H.rel_rmse(got, res) < 2e-5
    else:
        # radiance through the solid-angle lightcut (threshold pi/10), antiradiance brute force
        ctx.upload_materials(d["mats"])
        dv = ctx.upload_avpls(d["avpls"])
        bvh = api.AvplBvh(ctx)
        bvh.build(dv)
        tree = bvh.host_arrays()
        crad, err = O.cut_solid_angle(d["pos"], d["nrm"], px, tree, d["dif"], d["spe"], d["ex"], d["cam"],
                                      math.pi / 10, 0.01)
        assert H.rel_rmse(got, crad - ar) < 1e-5


def test_back_to_back_runs_keep_their_uploads(ctx):
    """arc_run's upload converts into two pinned staging buffers in turn without waiting for the
    previous frame: three runs queued back to back (AVPL sets A, B, A) give each set's own image."""
    import torch

    da = H.workload("room_256_4k", 64, 64, 4096)
    avpls_b = da["avpls"].copy()
    avpls_b["incRadiance"] *= 0.5  # a second AVPL set: half the radiance
    gb = api.GBuffer(da["pos"], da["nrm"])
    g = api.CudaGather(ctx, gb, da["mats"])
    ext = scene.scene_extent(da["desc"])
    cfg = api.run_config(useLightCuts=0, ar_kind=L.ARC_AR_DISK, dist_clamp=0.01)
    ref = {}
    for name, av in (("a", da["avpls"]), ("b", avpls_b)):
        ref[name] = g.run(av, da["cam"], ext, cfg).result64.clone()
        assert ctx.synchronize() == 0
    got = []
    for av in (da["avpls"], avpls_b, da["avpls"]):  # no synchronisation in between
        got.append(g.run(av, da["cam"], ext, cfg).result64.clone())
    torch.cuda.synchronize()
    assert ctx.synchronize() == 0
    assert torch.equal(got[0], ref["a"]) and torch.equal(got[1], ref["b"]) and torch.equal(got[2], ref["a"])
    assert not torch.equal(ref["a"], ref["b"])


@pytest.mark.parametrize("use_cuts", [0, 1])
def test_run_clustered_deferred_antiradiance(ctx, use_cuts):
    """useClusteredDeferred (cudaGather.cu:948-1031): the disk antiradiance through screen
    clusters gives the brute-force antiradiance's image up to summation order."""
    d = H.workload("boxes2_720p_64k", 96, 64, 8192)
    gb = api.GBuffer(d["pos"], d["nrm"])
    g = api.CudaGather(ctx, gb, d["mats"])
    ext = scene.scene_extent(d["desc"])
    imgs = []
    for clustered in (0, 1):
        cfg = api.run_config(useLightCuts=use_cuts, ar_kind=L.ARC_AR_DISK, useClusteredDeferred=clustered,
                             cluster_theta=math.radians(0.5 * d["desc"].camera_fov_deg))
        out = g.run(d["avpls"], d["cam"], ext, cfg)
        assert ctx.synchronize() == 0
        imgs.append((out.result64.cpu().numpy().reshape(-1, 3).copy(), out.antiradiance.cpu().numpy().copy()))
    assert np.abs(imgs[0][1]).max() > 0
    assert H.rel_rmse(imgs[1][0], imgs[0][0]) < 1e-6
    assert H.rel_rmse(imgs[1][1][..., :3].reshape(-1, 3), imgs[0][1][..., :3].reshape(-1, 3)) < 1e-5


def test_run_profile_prints_stage_times_and_keeps_the_image(ctx, capfd):
    """ArcRunConfig.profile: the three stage lines of the reference's run() timers
    (cudaGather.cu:845-1049) are printed, the image is unchanged, and a profiled call that fails
    midway (one AVPL: too few for the tree) returns its status and leaves the context usable."""
    import ctypes as C

    d = H.workload("room_256_4k", 64, 64, 4096)
    gb = api.GBuffer(d["pos"], d["nrm"])
    g = api.CudaGather(ctx, gb, d["mats"])
    ext = scene.scene_extent(d["desc"])
    ref = g.run(d["avpls"], d["cam"], ext, api.run_config(useLightCuts=1, ar_kind=L.ARC_AR_DISK)).result64.clone()
    assert ctx.synchronize() == 0
    got = g.run(d["avpls"], d["cam"], ext, api.run_config(useLightCuts=1, ar_kind=L.ARC_AR_DISK, profile=1))
    assert ctx.synchronize() == 0
    C.CDLL(None).fflush(None)
    text = capfd.readouterr().out
    for line in ("transfer avpl data to gpu took:", "gather build bvh took:", "gather radiance and antiradiance took:"):
        assert line in text
    assert np.array_equal(got.result64.cpu().numpy(), ref.cpu().numpy())
    with pytest.raises(L.ArcError) as e:
        g.run(d["avpls"][:1], d["cam"], ext, api.run_config(useLightCuts=1, ar_kind=L.ARC_AR_DISK, profile=1))
    assert e.value.status == L.ARC_ERR_TOO_FEW_AVPLS
    again = g.run(d["avpls"], d["cam"], ext, api.run_config(useLightCuts=1, ar_kind=L.ARC_AR_DISK, profile=1))
    assert ctx.synchronize() == 0
    assert np.array_equal(again.result64.cpu().numpy(), ref.cpu().numpy())


def test_measure_fp32_peak_is_plausible(ctx):
    """arc_measure_fp32_peak: the FFMA microbenchmark that is the gather kernels' roofline
    denominator (B200: 148 SMs x 128 FP32 lanes x 2 FLOP x ~1.9 GHz = ~72 TFLOP/s)."""
    import ctypes as C

    sc, pk = C.c_double(), C.c_double()
    L.check(ctx.lib.arc_measure_fp32_peak(ctx.handle, C.byref(sc), C.byref(pk)), "arc_measure_fp32_peak")
    assert 20.0 < sc.value < 120.0 and 20.0 < pk.value < 120.0
