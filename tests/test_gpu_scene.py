"""The GPU scene generator (arc_scene_gbuffer_device, arc_scene_trace_avpls_device) against the
CPU one (arc_scene_gbuffer, arc_scene_trace_avpls) on Lambertian scenes: the G-buffer bit for
bit; the AVPLs in the same order from the same paths, with the same bounces and materials, and
floating-point fields equal up to the rounding of the azimuth's cos / sin, which the host and
device math libraries compute independently (both deterministic, so these cases are fixed)."""
import numpy as np
import pytest

from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import scene

pytestmark = pytest.mark.gpu

SCENES = [(L.ARC_SCENE_ROOM, 0, 0), (L.ARC_SCENE_ROOM_2BOXES, 2, 2), (L.ARC_SCENE_ROOM_RANDOM, 3, 16),
          (L.ARC_SCENE_TRAIN_VARIANT, 500, 0)]


@pytest.mark.parametrize("preset,seed,boxes", SCENES)
@pytest.mark.parametrize("size", [(160, 90), (97, 61)])
def test_gbuffer_device_equals_cpu(ctx, preset, seed, boxes, size):
    desc = scene.scene_desc(preset, seed, boxes)
    pos, nrm = scene.gbuffer(desc, *size)
    gb = scene.gbuffer_device(ctx, desc, *size)
    assert ctx.synchronize() == 0
    assert np.array_equal(gb.pos.cpu().numpy(), pos) and np.array_equal(gb.nrm.cpu().numpy(), nrm)


def _equal(a, b):
    """Same AVPLs: bounces, materials and (axis-aligned) normals equal, so every AVPL lies on the
    same surface of the same path; the other fields within 1e-4 of the CPU's, relative to
    max(1, |value|)."""
    if len(a) != len(b) or not all(np.array_equal(a[k], b[k]) for k in ("bounce", "materialIndex", "normal")):
        return False
    for k in ("position", "incRadiance", "antiradiance", "incDirection"):
        d = np.abs(a[k].astype(np.float64) - b[k]) / np.maximum(1.0, np.abs(b[k]))
        if not d.max() <= 1e-4:
            return False
    return True


@pytest.mark.parametrize("preset,seed,boxes", SCENES)
def test_tracer_device_equals_cpu(ctx, preset, seed, boxes):
    desc = scene.scene_desc(preset, seed, boxes)
    for avpl_seed, num, bounces, direct in ((7, 20000, 3, True), (11, 5000, 5, False)):
        ref, ref_paths = scene.trace_avpls(desc, avpl_seed, num, bounces, direct)
        dv, paths = scene.trace_avpls_device(ctx, desc, avpl_seed, num, bounces, direct)
        assert ctx.synchronize() == 0
        got = dv.to_host()
        assert paths == ref_paths
        assert _equal(got, ref), preset


def test_tracer_device_batches_and_edges(ctx):
    desc = scene.scene_desc(L.ARC_SCENE_ROOM, 0, 0)
    # one bounce per path and an open front: fewer AVPLs than paths, so several batches of paths
    ref, ref_paths = scene.trace_avpls(desc, 5, 30000, 1)
    dv, paths = scene.trace_avpls_device(ctx, desc, 5, 30000, 1)
    assert ctx.synchronize() == 0
    assert ref_paths > 30000 and paths == ref_paths and _equal(dv.to_host(), ref)
    # nothing asked: no paths
    dv0, p0 = scene.trace_avpls_device(ctx, desc, 5, 0, 3)
    assert p0 == 0 and dv0.n == 0
    # bounce limit out of range: refused before any work
    from antiradiancecuts_b200 import api
    import ctypes as C

    d = api.DeviceAvpls.empty(16)
    st = ctx.lib.arc_scene_trace_avpls_device(ctx.handle, C.byref(desc), 1, 0, 1, C.byref(d.param), None)
    assert st == L.ARC_ERR_INVALID_ARG
