"""The seeded synthetic workloads against the configurations they stand in for (no GPU): sizes,
seeds, bounce limits, antiradiance settings, and the scenes' walls, light, camera and boxes."""
import numpy as np
import pytest

from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import scene

RED, GREEN, GRAY = (0.63, 0.065, 0.05), (0.14, 0.45, 0.09), (0.7, 0.7, 0.7)


def _f3(v):
    return np.array([v.x, v.y, v.z], np.float64)


@pytest.mark.parametrize("name,preset,scene_seed,boxes,avpl_seed,size,avpls,bounces,cone,clamp", [
    ("room_256_4k", L.ARC_SCENE_ROOM, 1, 0, 1, (256, 256), 4096, 3, 30.0, 0.01),
    ("boxes2_720p_64k", L.ARC_SCENE_ROOM_2BOXES, 2, 2, 2, (1280, 720), 65536, 3, 30.0, 0.01),
    ("boxes16_1080p_256k", L.ARC_SCENE_ROOM_RANDOM, 3, 16, 3, (1920, 1080), 262144, 5, 60.0, 0.005),
    ("variant500_1080p_1m", L.ARC_SCENE_TRAIN_VARIANT, 500, 0, 500, (1920, 1080), 1 << 20, 3, 30.0, 0.01),
])
def test_workload_sizes(name, preset, scene_seed, boxes, avpl_seed, size, avpls, bounces, cone, clamp):
    w = scene.WORKLOADS[name]
    assert (w.preset, w.scene_seed, w.num_boxes, w.avpl_seed) == (preset, scene_seed, boxes, avpl_seed)
    assert (w.width, w.height, w.num_avpls, w.max_bounces) == (*size, avpls, bounces)
    assert w.ar_kind == L.ARC_AR_CONE and w.cone_half_angle_deg == cone and w.dist_clamp == clamp


@pytest.mark.parametrize("preset,seed,boxes", [(L.ARC_SCENE_ROOM, 1, 0), (L.ARC_SCENE_ROOM_2BOXES, 2, 2),
                                               (L.ARC_SCENE_ROOM_RANDOM, 3, 16)])
def test_room_light_and_camera(preset, seed, boxes):
    """Open-front room [0,1]^3: gray 0.7, red left wall, green right wall; a 0.25 x 0.25 light at
    y = 0.999 centred in x / z with radiance (17, 12, 4); a pinhole camera at (0.5, 0.5, -1.4)
    looking +z with a 40 degree field of view."""
    d = scene.scene_desc(preset, seed, boxes)
    assert np.array_equal(_f3(d.scene_min), [0, 0, 0]) and np.array_equal(_f3(d.scene_max), [1, 1, 1])
    for i, albedo in ((1, GRAY), (2, RED), (3, GREEN)):
        assert np.allclose(_f3(d.materials[i].diffuse), albedo, atol=1e-7)
    assert np.allclose(_f3(d.light_center), [0.5, 0.999, 0.5], atol=1e-7)
    assert d.light_half_size == pytest.approx(0.125)
    assert np.allclose(_f3(d.light_radiance), [17, 12, 4])
    assert np.allclose(_f3(d.camera_position), [0.5, 0.5, -1.4], atol=1e-7)
    look = _f3(d.camera_target) - _f3(d.camera_position)
    assert look[0] == 0 and look[1] == 0 and look[2] > 0
    assert d.camera_fov_deg == 40.0
    assert d.num_boxes == boxes


def test_two_boxes():
    """0.3^3 at (0.2, 0, 0.55) and 0.3 x 0.6 x 0.3 at (0.55, 0, 0.2), albedo 0.7."""
    d = scene.scene_desc(L.ARC_SCENE_ROOM_2BOXES, 2, 2)
    got = sorted((tuple(np.round(_f3(b.lo), 6)), tuple(np.round(_f3(b.hi) - _f3(b.lo), 6)), b.material)
                 for b in d.boxes[:2])
    assert got[0][:2] == ((0.2, 0.0, 0.55), (0.3, 0.3, 0.3))
    assert got[1][:2] == ((0.55, 0.0, 0.2), (0.3, 0.6, 0.3))
    for b in d.boxes[:2]:
        assert np.allclose(_f3(d.materials[b.material].diffuse), GRAY, atol=1e-7)


def test_random_boxes():
    """16 boxes (seed 3) with edge lengths in [0.05, 0.25] and per-channel albedo in [0.3, 0.8]."""
    d = scene.scene_desc(L.ARC_SCENE_ROOM_RANDOM, 3, 16)
    assert d.num_boxes == 16
    for b in d.boxes[:16]:
        e = _f3(b.hi) - _f3(b.lo)
        assert np.all(e >= 0.05 - 1e-6) and np.all(e <= 0.25 + 1e-6)
        a = _f3(d.materials[b.material].diffuse)
        assert np.all(a >= 0.3 - 1e-6) and np.all(a <= 0.8 + 1e-6)


def test_batch_views():
    """32 views (seed 4) of the room + 2 boxes scene: resolutions from {256^2, 512^2, 1280 x 720,
    1920 x 1080}, 8,192 - 262,144 AVPLs each, cameras inside the room and outside the boxes."""
    d = scene.scene_desc(L.ARC_SCENE_ROOM_2BOXES, 2, 2)
    views = scene.batch_views(d, 4, 32)
    assert len(views) == 32
    sizes = {(v.width, v.height) for v in views}
    assert sizes <= {(256, 256), (512, 512), (1280, 720), (1920, 1080)} and len(sizes) > 1
    for v in views:
        assert 8192 <= v.num_avpls <= 262144
        c = _f3(v.camera_position)
        assert np.all(c > 0) and np.all(c < 1)
        for b in d.boxes[:2]:
            assert not (np.all(c > _f3(b.lo)) and np.all(c < _f3(b.hi)))
    again = scene.batch_views(d, 4, 32)
    assert [(v.width, v.num_avpls, v.avpl_seed) for v in views] == [(v.width, v.num_avpls, v.avpl_seed) for v in again]
