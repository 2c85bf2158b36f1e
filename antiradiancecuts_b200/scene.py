"""Seeded synthetic inputs: scene descriptions, AVPL sets and G-buffers as numpy arrays, produced
by libarc's CPU scene generator (arc_scene_*), plus the named workloads the tests and the
benchmark run.  These are inputs of the gather, not part of it.  Every CPU generator function takes
an optional `lib`: another library that exports the arc_scene_* entry points (the generator's
source built without the GPU library, see _lib.load_scene_library); libarc by default."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

# ArcAvplHost as a numpy record (68 bytes, no padding)
AVPL_DTYPE = np.dtype([("position", "<f4", 3), ("normal", "<f4", 3), ("incRadiance", "<f4", 3),
                       ("antiradiance", "<f4", 3), ("incDirection", "<f4", 3), ("bounce", "<i4"),
                       ("materialIndex", "<i4")])
assert AVPL_DTYPE.itemsize == C.sizeof(L.ArcAvplHost)


def _check(lib, status: int, where: str) -> None:
    if status != L.ARC_OK:
        raise L.ArcError(status, where, lib.arc_last_error().decode())


def scene_desc(preset: int, seed: int = 0, num_boxes: int = 0, lib=None) -> L.ArcSceneDesc:
    lib = lib or L.load()
    d = L.ArcSceneDesc()
    _check(lib, lib.arc_scene_preset_desc(int(preset), int(seed), int(num_boxes), C.byref(d)), "arc_scene_preset_desc")
    return d


def trace_avpls(desc: L.ArcSceneDesc, seed: int, num: int, max_bounces: int = 3,
                explicit_direct: bool = True, lib=None) -> tuple[np.ndarray, int]:
    lib = lib or L.load()
    out = np.zeros(num, dtype=AVPL_DTYPE)
    paths = C.c_int64(0)
    _check(lib, lib.arc_scene_trace_avpls(C.byref(desc), int(seed), int(max_bounces), int(explicit_direct), int(num),
                                          out.ctypes.data_as(C.POINTER(L.ArcAvplHost)), C.byref(paths)),
           "arc_scene_trace_avpls")
    return out, int(paths.value)


def gbuffer(desc: L.ArcSceneDesc, width: int, height: int, lib=None) -> tuple[np.ndarray, np.ndarray]:
    lib = lib or L.load()
    pos = np.zeros((height, width, 4), dtype=np.float32)
    nrm = np.zeros((height, width, 4), dtype=np.float32)
    _check(lib, lib.arc_scene_gbuffer(C.byref(desc), int(width), int(height), pos.ctypes.data, nrm.ctypes.data),
           "arc_scene_gbuffer")
    return pos, nrm


def gbuffer_device(ctx, desc: L.ArcSceneDesc, width: int, height: int):
    """The G-buffer of `desc` rendered on the GPU (arc_scene_gbuffer_device) into a new
    api.GBuffer; the same bits as gbuffer()."""
    from . import api

    gb = api.GBuffer.empty(width, height)
    L.check(ctx.lib.arc_scene_gbuffer_device(ctx.handle, C.byref(desc), C.byref(gb.view())), "arc_scene_gbuffer_device")
    return gb


def trace_avpls_device(ctx, desc: L.ArcSceneDesc, seed: int, num: int, max_bounces: int = 3,
                       explicit_direct: bool = True):
    """`num` AVPLs traced on the GPU (arc_scene_trace_avpls_device) into a new api.DeviceAvpls,
    and the number of light paths; the AVPLs of trace_avpls(), in the same order, up to the
    rounding of the azimuth's cos / sin."""
    from . import api

    dv = api.DeviceAvpls.empty(num)
    paths = C.c_int64(0)
    L.check(ctx.lib.arc_scene_trace_avpls_device(ctx.handle, C.byref(desc), int(seed), int(max_bounces),
                                                 int(explicit_direct), C.byref(dv.param), C.byref(paths)),
            "arc_scene_trace_avpls_device")
    return dv, int(paths.value)


def materials(desc: L.ArcSceneDesc):
    """(ctypes array of ArcMaterial, diffuse[m,3], specular[m,3], exponent[m])"""
    n = desc.num_materials
    arr = (L.ArcMaterial * n)(*[desc.materials[i] for i in range(n)])
    dif = np.array([[m.diffuse.x, m.diffuse.y, m.diffuse.z] for m in arr], dtype=np.float32)
    spe = np.array([[m.specular.x, m.specular.y, m.specular.z] for m in arr], dtype=np.float32)
    exp = np.array([m.exponent for m in arr], dtype=np.float32)
    return arr, dif, spe, exp


def scene_extent(desc: L.ArcSceneDesc) -> float:
    """|bbMax - bbMin| of the scene (Scene::getSceneExtent, Scene.h:75)."""
    a, b = desc.scene_min, desc.scene_max
    return math.sqrt((b.x - a.x) ** 2 + (b.y - a.y) ** 2 + (b.z - a.z) ** 2)


@dataclass
class Workload:
    """One named input configuration."""
    name: str
    preset: int
    scene_seed: int
    num_boxes: int
    avpl_seed: int
    width: int
    height: int
    num_avpls: int
    max_bounces: int
    ar_kind: int = L.ARC_AR_CONE
    cone_half_angle_deg: float = 30.0
    dist_clamp: float = 0.01
    error_bound: float = 0.01
    extra: dict = field(default_factory=dict)

    def build(self, width: int | None = None, height: int | None = None, num_avpls: int | None = None, lib=None):
        """Scene description, AVPLs, G-buffer (optionally at a reduced size for tests)."""
        desc = scene_desc(self.preset, self.scene_seed, self.num_boxes, lib=lib)
        avpls, paths = trace_avpls(desc, self.avpl_seed, num_avpls or self.num_avpls, self.max_bounces, lib=lib)
        pos, nrm = gbuffer(desc, width or self.width, height or self.height, lib=lib)
        return desc, avpls, paths, pos, nrm


# The benchmark's configurations: shapes, sizes and value distributions of the reference's
# experiment set-up, as seeded synthetic inputs.
WORKLOADS = {
    # plain brute-force gather, 256^2, 4096 AVPLs (seed 1, <= 3 bounces), cone 30 deg, clamp 0.01
    "room_256_4k": Workload("room_256_4k", L.ARC_SCENE_ROOM, 1, 0, 1, 256, 256, 4096, 3),
    # LBVH + error-bound cut, room + 2 boxes, 1280x720, 65,536 AVPLs (seed 2)
    "boxes2_720p_64k": Workload("boxes2_720p_64k", L.ARC_SCENE_ROOM_2BOXES, 2, 2, 2, 1280, 720, 65536, 3),
    # precision stress: 16 random boxes (seed 3), 1080p, 262,144 AVPLs (<= 5 bounces), cone 60, clamp 0.005
    "boxes16_1080p_256k": Workload("boxes16_1080p_256k", L.ARC_SCENE_ROOM_RANDOM, 3, 16, 3, 1920, 1080, 262144, 5,
                                   cone_half_angle_deg=60.0, dist_clamp=0.005),
    # learned-cut evaluation: held-out variant seed 500, 1080p, 1,048,576 AVPLs
    "variant500_1080p_1m": Workload("variant500_1080p_1m", L.ARC_SCENE_TRAIN_VARIANT, 500, 0, 500, 1920, 1080,
                                    1 << 20, 3),
}


def batch_views(desc: L.ArcSceneDesc, seed: int, count: int) -> list[L.ArcBatchViewDesc]:
    """Views of a multi-view batch in `desc` (arc_scene_batch_views): resolution, AVPL count and
    seed, camera pose inside the room."""
    out = (L.ArcBatchViewDesc * count)()
    L.check(L.load().arc_scene_batch_views(C.byref(desc), int(seed), int(count), out), "arc_scene_batch_views")
    return list(out)


def view_inputs(desc: L.ArcSceneDesc, view: L.ArcBatchViewDesc, max_bounces: int = 3, scale: float = 1.0):
    """(AVPLs, position, normal) of one batch view: its own AVPL set and its camera's G-buffer
    (resolution scaled by `scale`, for reduced test sizes)."""
    d = L.ArcSceneDesc()
    C.memmove(C.byref(d), C.byref(desc), C.sizeof(d))
    d.camera_position = view.camera_position
    d.camera_target = view.camera_target
    avpls, _ = trace_avpls(d, view.avpl_seed, view.num_avpls, max_bounces)
    w, h = max(8, int(view.width * scale)), max(8, int(view.height * scale))
    pos, nrm = gbuffer(d, w, h)
    return avpls, pos, nrm
