"""ctypes binding of libarc.so (include/arc_api.h).

The shared library is the product; this module only declares its C ABI for Python callers
(tests, benchmark, smoke check).  Loading fails loudly when libarc.so has not been built: there
is no Python or CPU fallback for any GPU entry point.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libarc.so")

ARC_OK = 0
ARC_ERR_INVALID_ARG = 1
ARC_ERR_TOO_FEW_AVPLS = 2
ARC_ERR_STACK_OVERFLOW = 3
ARC_ERR_TIMEOUT = 4
ARC_ERR_CUDA = 5
ARC_ERR_OUT_OF_MEMORY = 6
ARC_ERR_DEVICE = 7
ARC_ERR_UNSUPPORTED = 8
ARC_ERR_IO = 9

ARC_DEVERR_STACK_OVERFLOW = 0x1
ARC_DEVERR_TIMEOUT = 0x2
ARC_DEVERR_BAD_MATERIAL = 0x4
ARC_DEVERR_BAD_NODE = 0x8
ARC_DEVERR_CUT_OVERFLOW = 0x10

ARC_MAX_MATERIALS = 64
ARC_SCENE_MAX_BOXES = 32

ARC_AR_NONE, ARC_AR_DISK, ARC_AR_CONE = 0, 1, 2
ARC_ERROR_REFERENCE, ARC_ERROR_RMSE = 0, 1
ARC_PREC_KAHAN, ARC_PREC_KAHAN_STRICT, ARC_PREC_NAIVE, ARC_PREC_FP64 = 0, 1, 2, 3
ARC_BBOX_SCENE, ARC_BBOX_AVPL_REFERENCE = 0, 1
ARC_CUT_SOLID_ANGLE, ARC_CUT_ERROR_BOUND, ARC_CUT_LEARNED = 0, 1, 2
ARC_MLP_LOSS_BCE, ARC_MLP_LOSS_SQUARED = 0, 1
ARC_MLP_ACT_GELU, ARC_MLP_ACT_RELU = 0, 1
ARC_SCENE_ROOM, ARC_SCENE_ROOM_2BOXES, ARC_SCENE_ROOM_RANDOM, ARC_SCENE_TRAIN_VARIANT = 0, 1, 2, 3


class ArcFloat3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class ArcAvplHost(C.Structure):
    _fields_ = [("position", ArcFloat3), ("normal", ArcFloat3), ("incRadiance", ArcFloat3),
                ("antiradiance", ArcFloat3), ("incDirection", ArcFloat3), ("bounce", C.c_int32),
                ("materialIndex", C.c_int32)]


class ArcAvplsGpuParam(C.Structure):
    _fields_ = [("position", C.c_void_p), ("normal", C.c_void_p), ("incDirection", C.c_void_p),
                ("incRadiance", C.c_void_p), ("antiradiance", C.c_void_p), ("materialIndex", C.c_void_p),
                ("bounce", C.c_void_p), ("numAvpls", C.c_int32)]


class ArcMaterial(C.Structure):
    _fields_ = [("emissive", ArcFloat3), ("diffuse", ArcFloat3), ("specular", ArcFloat3), ("exponent", C.c_float)]


class ArcGBufferView(C.Structure):
    _fields_ = [("position", C.c_void_p), ("normal", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32),
                ("pitch", C.c_int64)]


class ArcOutputView(C.Structure):
    _fields_ = [("result", C.c_void_p), ("radiance", C.c_void_p), ("antiradiance", C.c_void_p),
                ("result_fp64", C.c_void_p), ("pitch", C.c_int64)]


class ArcClusterParams(C.Structure):
    _fields_ = [("z_near", C.c_float), ("theta", C.c_float)]


class ArcClusterInfo(C.Structure):
    _fields_ = [("pixel_cluster", C.c_void_p), ("box", C.c_void_p), ("tile_count", C.c_void_p),
                ("counts", C.c_void_p), ("lists", C.c_void_p), ("num_tiles", C.c_int32),
                ("slots_per_tile", C.c_int32), ("list_entries", C.c_int64)]


class ArcAccumView(C.Structure):
    _fields_ = [("sum", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32), ("pitch", C.c_int64)]


class ArcGatherParams(C.Structure):
    _fields_ = [("ar_kind", C.c_int32), ("disk_radius", C.c_float), ("cone_half_angle", C.c_float),
                ("dist_clamp", C.c_float), ("geo_limit_radiance", C.c_float),
                ("geo_limit_antiradiance", C.c_float), ("precision", C.c_int32), ("tile_config", C.c_int32)]


class ArcLbvhParams(C.Structure):
    _fields_ = [("consider_normals", C.c_int32), ("bbox_mode", C.c_int32), ("scene_min", ArcFloat3),
                ("scene_max", ArcFloat3), ("repr_seed", C.c_uint32), ("wait_limit", C.c_uint32)]


class ArcBvhNode(C.Structure):
    _fields_ = [("left", C.c_int32), ("right", C.c_int32), ("bbMin", ArcFloat3), ("bbMax", ArcFloat3),
                ("visited", C.c_int32)]


class ArcBvhParam(C.Structure):
    _fields_ = [("numLeafs", C.c_int32), ("numNodes", C.c_int32), ("nodes", C.c_void_p),
                ("positions", C.c_void_p), ("normals", C.c_void_p)]


class ArcAvplBvhNodeDataParam(C.Structure):
    _fields_ = [("size", C.c_void_p), ("materialIndex", C.c_void_p), ("randomNumbers", C.c_void_p),
                ("position", C.c_void_p), ("normal", C.c_void_p), ("incRadiance", C.c_void_p),
                ("incDirection", C.c_void_p)]


class ArcLbvhView(C.Structure):
    _fields_ = [("num_leaves", C.c_int32), ("num_nodes", C.c_int32), ("morton", C.c_void_p),
                ("sorted_index", C.c_void_p), ("left", C.c_void_p), ("right", C.c_void_p),
                ("parents", C.c_void_p), ("range", C.c_void_p), ("bounds", C.c_void_p), ("records", C.c_void_p),
                ("node_data", ArcAvplBvhNodeDataParam), ("dirstat", C.c_void_p)]


class ArcCutParams(C.Structure):
    _fields_ = [("kind", C.c_int32), ("solid_angle_threshold", C.c_float), ("error_bound", C.c_float),
                ("ar_uncertain_factor", C.c_float), ("max_cut_nodes", C.c_int32), ("cut_pool_entries", C.c_int64),
                ("model", C.c_void_p), ("mlp_threshold", C.c_float), ("mlp_band", C.c_float),
                ("debug_pixel_x", C.c_int32), ("debug_pixel_y", C.c_int32), ("used_nodes", C.c_void_p)]


class ArcCutLists(C.Structure):
    _fields_ = [("num_tiles", C.c_int32), ("chunk_size", C.c_int32), ("max_chunks", C.c_int32),
                ("pool_chunks_used", C.c_int32), ("counts", C.c_void_p), ("tables", C.c_void_p), ("pool", C.c_void_p)]


class ArcRunConfig(C.Structure):
    _fields_ = [("useLightCuts", C.c_int32), ("cut_kind", C.c_int32), ("clusterRefinementThreshold", C.c_float),
                ("error_bound", C.c_float), ("photonRadiusScale", C.c_float), ("ar_kind", C.c_int32),
                ("cone_half_angle", C.c_float), ("dist_clamp", C.c_float), ("precision", C.c_int32),
                ("considerNormals", C.c_int32), ("model", C.c_void_p), ("profile", C.c_int32),
                ("ar_uncertain_factor", C.c_float), ("mlp_threshold", C.c_float), ("mlp_band", C.c_float),
                ("cut_pool_entries", C.c_int64), ("useClusteredDeferred", C.c_int32), ("cluster_z_near", C.c_float),
                ("cluster_theta", C.c_float)]


class ArcBox(C.Structure):
    _fields_ = [("lo", ArcFloat3), ("hi", ArcFloat3), ("material", C.c_int32)]


class ArcSceneDesc(C.Structure):
    _fields_ = [("num_boxes", C.c_int32), ("boxes", ArcBox * ARC_SCENE_MAX_BOXES), ("num_materials", C.c_int32),
                ("materials", ArcMaterial * ARC_MAX_MATERIALS), ("light_center", ArcFloat3),
                ("light_half_size", C.c_float), ("light_radiance", ArcFloat3), ("light_material", C.c_int32),
                ("camera_position", ArcFloat3), ("camera_target", ArcFloat3), ("camera_fov_deg", C.c_float),
                ("scene_min", ArcFloat3), ("scene_max", ArcFloat3)]


class ArcBatchView(C.Structure):
    _fields_ = [("avpls", ArcAvplsGpuParam), ("gbuffer", ArcGBufferView), ("camera_position", ArcFloat3),
                ("out", ArcOutputView)]


class ArcBatchViewDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("num_avpls", C.c_int32), ("avpl_seed", C.c_uint64),
                ("camera_position", ArcFloat3), ("camera_target", ArcFloat3)]


P = C.POINTER
_vp = C.c_void_p
_st = C.c_int32

# name -> (restype, argtypes); every entry is a symbol declared in include/arc_api.h
SIGNATURES = {
    "arc_api_version": (C.c_int32, []),
    "arc_status_string": (C.c_char_p, [C.c_int32]),
    "arc_last_error": (C.c_char_p, []),
    "arc_gather_params_default": (None, [P(ArcGatherParams)]),
    "arc_lbvh_params_default": (None, [P(ArcLbvhParams)]),
    "arc_cut_params_default": (None, [P(ArcCutParams)]),
    "arc_run_config_default": (None, [P(ArcRunConfig)]),
    "arc_context_create": (_st, [C.c_int32, _vp, P(_vp)]),
    "arc_context_destroy": (_st, [_vp]),
    "arc_context_synchronize": (_st, [_vp, P(C.c_uint32)]),
    "arc_context_stream": (_vp, [_vp]),
    "arc_context_profile": (_st, [_vp, C.c_int32]),
    "arc_context_stage_times": (_st, [_vp, C.c_char_p, C.c_size_t, P(C.c_float), C.c_int32, P(C.c_int32)]),
    "arc_context_launch_count": (C.c_uint64, [_vp]),
    "arc_context_learned_rows": (C.c_uint64, [_vp]),
    "arc_measure_fp32_peak": (_st, [_vp, P(C.c_double), P(C.c_double)]),
    "arc_device_alloc": (_st, [_vp, C.c_size_t, P(_vp)]),
    "arc_device_free": (_st, [_vp, _vp]),
    "arc_copy_h2d": (_st, [_vp, _vp, _vp, C.c_size_t]),
    "arc_copy_d2h": (_st, [_vp, _vp, _vp, C.c_size_t]),
    "arc_materials_upload": (_st, [_vp, P(ArcMaterial), C.c_int32]),
    "arc_avpls_upload": (_st, [_vp, P(ArcAvplHost), C.c_int32, P(ArcAvplsGpuParam)]),
    "arc_gather_bruteforce": (_st, [_vp, P(ArcAvplsGpuParam), P(ArcGBufferView), ArcFloat3, P(ArcGatherParams),
                                    P(ArcOutputView)]),
    "arc_gather_bruteforce_noalloc": (_st, [_vp, P(ArcMaterial), C.c_int32, P(ArcAvplsGpuParam), P(ArcGBufferView),
                                            ArcFloat3, P(ArcGatherParams), P(ArcOutputView), P(C.c_uint32)]),
    "arc_lbvh_create": (_st, [_vp, P(_vp)]),
    "arc_lbvh_destroy": (_st, [_vp]),
    "arc_lbvh_build": (_st, [_vp, P(ArcAvplsGpuParam), P(ArcLbvhParams)]),
    "arc_lbvh_get_view": (_st, [_vp, P(ArcLbvhView)]),
    "arc_lbvh_reference_views": (_st, [_vp, P(ArcBvhParam), P(ArcAvplBvhNodeDataParam)]),
    "arc_gather_cut": (_st, [_vp, _vp, P(ArcAvplsGpuParam), P(ArcGBufferView), ArcFloat3, P(ArcGatherParams),
                             P(ArcCutParams), P(ArcOutputView)]),
    "arc_last_cut": (_st, [_vp, P(ArcCutLists)]),
    "arc_mlp_num_params": (C.c_int32, []),
    "arc_mlp_create": (_st, [_vp, C.c_uint64, P(_vp)]),
    "arc_mlp_destroy": (_st, [_vp]),
    "arc_mlp_set_params": (_st, [_vp, P(C.c_float), C.c_int32]),
    "arc_mlp_get_params": (_st, [_vp, P(C.c_float), C.c_int32]),
    "arc_mlp_forward": (_st, [_vp, _vp, C.c_int64, _vp]),
    "arc_mlp_gradients": (_st, [_vp, _vp, _vp, _vp, C.c_int64, C.c_float, P(C.c_float), P(C.c_float)]),
    "arc_mlp_train_step": (_st, [_vp, _vp, _vp, _vp, C.c_int64, C.c_float, C.c_float, _vp]),
    "arc_mlp_set_loss": (_st, [_vp, C.c_int32]),
    "arc_mlp_get_loss": (C.c_int32, [_vp]),
    "arc_mlp_set_activation": (_st, [_vp, C.c_int32]),
    "arc_mlp_get_activation": (C.c_int32, [_vp]),
    "arc_cut_training_samples": (_st, [_vp, _vp, P(ArcGBufferView), ArcFloat3, P(ArcGatherParams), P(ArcCutParams),
                                       C.c_float, _vp, _vp, _vp, _vp, C.c_int32, P(C.c_int32)]),
    "arc_run": (_st, [_vp, P(ArcAvplHost), C.c_int32, ArcFloat3, C.c_float, P(ArcRunConfig), P(ArcGBufferView),
                      P(ArcOutputView)]),
    "arc_scene_preset_desc": (_st, [C.c_int32, C.c_uint64, C.c_int32, P(ArcSceneDesc)]),
    "arc_scene_trace_avpls": (_st, [P(ArcSceneDesc), C.c_uint64, C.c_int32, C.c_int32, C.c_int32, P(ArcAvplHost),
                                    P(C.c_int64)]),
    "arc_scene_gbuffer": (_st, [P(ArcSceneDesc), C.c_int32, C.c_int32, _vp, _vp]),
    "arc_scene_gbuffer_device": (_st, [_vp, P(ArcSceneDesc), P(ArcGBufferView)]),
    "arc_accumulate": (_st, [_vp, P(ArcOutputView), P(ArcAccumView)]),
    "arc_antiradiance_clustered": (_st, [_vp, P(ArcAvplsGpuParam), P(ArcGBufferView), ArcFloat3, P(ArcClusterParams),
                                         P(ArcGatherParams), P(ArcOutputView), P(ArcClusterInfo)]),
    "arc_accum_clear": (_st, [_vp, P(ArcAccumView)]),
    "arc_accum_normalize": (_st, [_vp, P(ArcAccumView), C.c_int64, P(ArcOutputView)]),
    "arc_image_error": (_st, [_vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int64, C.c_int32, P(C.c_double),
                              P(C.c_double)]),
    "arc_export_pfm": (_st, [C.c_char_p, _vp, C.c_int32, C.c_int32, C.c_int64]),
    "arc_export_hdr": (_st, [C.c_char_p, _vp, C.c_int32, C.c_int32, C.c_int64]),
    "arc_scene_trace_avpls_device": (_st, [_vp, P(ArcSceneDesc), C.c_uint64, C.c_int32, C.c_int32,
                                           P(ArcAvplsGpuParam), P(C.c_int64)]),
    "arc_scene_batch_views": (_st, [P(ArcSceneDesc), C.c_uint64, C.c_int32, P(ArcBatchViewDesc)]),
    "arc_batch_create": (_st, [_vp, P(_vp)]),
    "arc_batch_destroy": (_st, [_vp]),
    "arc_batch_render": (_st, [_vp, P(ArcBatchView), C.c_int32, P(ArcLbvhParams), P(ArcGatherParams),
                               P(ArcCutParams)]),
    "arc_batch_capture": (_st, [_vp, P(ArcBatchView), C.c_int32, P(ArcLbvhParams), P(ArcGatherParams),
                                P(ArcCutParams)]),
    "arc_batch_launch": (_st, [_vp]),
    "arc_bruteforce_num_tile_shapes": (C.c_int32, []),
    "arc_context_set_tile_config": (_st, [_vp, C.c_int32]),
    "arc_autotune_bruteforce": (_st, [_vp, P(ArcAvplsGpuParam), P(ArcGBufferView), ArcFloat3, P(ArcGatherParams),
                                      P(ArcOutputView), P(C.c_int32), P(C.c_float), C.c_int32]),
}

_lib = None


class ArcError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        super().__init__(f"{where}: status {status} ({status_string(status)}) {msg}")


def load() -> C.CDLL:
    """Load libarc.so (built by antiradiancecuts_b200.build); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m antiradiancecuts_b200.build` "
                           "(the library has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


SCENE_SYMBOLS = ("arc_scene_preset_desc", "arc_scene_trace_avpls", "arc_scene_gbuffer", "arc_scene_batch_views")


def load_scene_library(path: str) -> C.CDLL:
    """A library that exports only the CPU scene generator's entry points (arc_scene_* and
    arc_last_error), with their signatures declared: the generator's source compiled on its own,
    for a process that must make the synthetic inputs without loading libarc."""
    lib = C.CDLL(path)
    for name in SCENE_SYMBOLS + ("arc_last_error",):
        res, args = SIGNATURES[name]
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def status_string(s: int) -> str:
    return load().arc_status_string(int(s)).decode()


def check(status: int, where: str) -> None:
    if status != ARC_OK:
        raise ArcError(status, where, load().arc_last_error().decode())


def f3(x, y=None, z=None) -> ArcFloat3:
    if y is None:
        x, y, z = x
    return ArcFloat3(float(x), float(y), float(z))
