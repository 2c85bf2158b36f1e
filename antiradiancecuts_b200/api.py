"""Python host interface over libarc's C ABI, named after the reference's classes:

    CudaGather(ctx, gbuffer, materials).run(avpls, camera_position, scene_extent, config)
        -> CudaGather::run (cudaGather.cu:836-1051)
    AvplBvh(ctx, avpls, consider_normals)      -> AvplBvh (bvh.cu:746-774)
    gather_bruteforce / gather_cut             -> the gather kernels

Device buffers are torch CUDA tensors (torch is used for device memory and streams only); every
computation runs in libarc's sm_100a kernels on the context's stream, which is torch's current
stream so the two stay ordered.
"""
from __future__ import annotations

import ctypes as C
import math
import weakref

import numpy as np

from . import _lib as L
from .scene import AVPL_DTYPE


def _torch():
    import torch

    return torch


class Context:
    """arc_context on `device`.  It owns a torch CUDA stream and makes it torch's current stream,
    so tensor allocations, fills and copies are ordered with the library's kernels (the legacy
    default stream would not be: the library's streams are non-blocking)."""

    def __init__(self, device: int = 0):
        torch = _torch()
        self.lib = L.load()
        self.device = device
        torch.cuda.set_device(device)
        self.stream = torch.cuda.Stream(device)
        torch.cuda.set_stream(self.stream)
        h = C.c_void_p()
        L.check(self.lib.arc_context_create(device, C.c_void_p(self.stream.cuda_stream), C.byref(h)),
                "arc_context_create")
        self.handle = h
        self._avpl_keep = None
        self._children = weakref.WeakSet()  # objects whose handles live in this context

    def close(self):
        if self.handle:
            for ch in list(self._children):
                ch.close()
            self.lib.arc_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self) -> int:
        w = C.c_uint32(0)
        L.check(self.lib.arc_context_synchronize(self.handle, C.byref(w)), "arc_context_synchronize")
        return int(w.value)

    def upload_materials(self, mats) -> None:
        L.check(self.lib.arc_materials_upload(self.handle, mats, len(mats)), "arc_materials_upload")

    def upload_avpls(self, avpls: np.ndarray) -> L.ArcAvplsGpuParam:
        """AvplsGpu(avpls): host records -> context-owned device arrays."""
        avpls = np.ascontiguousarray(avpls, dtype=AVPL_DTYPE)
        out = L.ArcAvplsGpuParam()
        L.check(self.lib.arc_avpls_upload(self.handle, avpls.ctypes.data_as(C.POINTER(L.ArcAvplHost)), len(avpls),
                                          C.byref(out)), "arc_avpls_upload")
        self._avpl_keep = avpls
        return out

    def d2h(self, ptr, dtype, count) -> np.ndarray:
        out = np.empty(count, dtype=dtype)
        if count:
            L.check(self.lib.arc_copy_d2h(self.handle, out.ctypes.data, C.c_void_p(ptr), out.nbytes), "arc_copy_d2h")
        return out


class GBuffer:
    """Device G-buffer planes (float4 position, float4 normal with material in w), uploaded from
    host arrays or, with GBuffer.empty, left to be written on the device."""

    def __init__(self, pos: np.ndarray | None, nrm: np.ndarray | None, device: int = 0, size=None):
        torch = _torch()
        if pos is None:
            self.width, self.height = size
            self.pos = torch.zeros((self.height, self.width, 4), dtype=torch.float32, device=f"cuda:{device}")
            self.nrm = torch.zeros_like(self.pos)
            return
        self.height, self.width = pos.shape[:2]
        self.pos = torch.from_numpy(np.ascontiguousarray(pos)).to(f"cuda:{device}")
        self.nrm = torch.from_numpy(np.ascontiguousarray(nrm)).to(f"cuda:{device}")

    @classmethod
    def empty(cls, width: int, height: int, device: int = 0) -> "GBuffer":
        return cls(None, None, device, (width, height))

    def view(self) -> L.ArcGBufferView:
        return L.ArcGBufferView(self.pos.data_ptr(), self.nrm.data_ptr(), self.width, self.height, self.width)


class Outputs:
    """Result / radiance / antiradiance float4 planes and the FP64 result plane."""

    def __init__(self, width: int, height: int, device: int = 0, fp64: bool = True, parts: bool = True):
        torch = _torch()
        dev = f"cuda:{device}"
        self.width, self.height = width, height
        self.result = torch.zeros((height, width, 4), dtype=torch.float32, device=dev)
        self.radiance = torch.zeros_like(self.result) if parts else None
        self.antiradiance = torch.zeros_like(self.result) if parts else None
        self.result64 = torch.zeros((height, width, 3), dtype=torch.float64, device=dev) if fp64 else None

    def view(self) -> L.ArcOutputView:
        p = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
        return L.ArcOutputView(p(self.result), p(self.radiance), p(self.antiradiance), p(self.result64), self.width)


def gather_params(ar_kind=L.ARC_AR_CONE, cone_half_angle_deg=30.0, dist_clamp=0.0, disk_radius=0.0,
                  precision=L.ARC_PREC_KAHAN, tile_config=-1, geo_limit_radiance=0.0,
                  geo_limit_antiradiance=0.0) -> L.ArcGatherParams:
    p = L.ArcGatherParams()
    L.load().arc_gather_params_default(C.byref(p))
    p.ar_kind = ar_kind
    p.cone_half_angle = math.radians(cone_half_angle_deg)
    p.dist_clamp = dist_clamp
    p.disk_radius = disk_radius
    p.precision = precision
    p.tile_config = tile_config
    p.geo_limit_radiance = geo_limit_radiance
    p.geo_limit_antiradiance = geo_limit_antiradiance
    return p


def gather_bruteforce(ctx: Context, avpls: L.ArcAvplsGpuParam, gb: GBuffer, cam, params: L.ArcGatherParams,
                      out: Outputs) -> None:
    gv, ov = gb.view(), out.view()
    L.check(ctx.lib.arc_gather_bruteforce(ctx.handle, C.byref(avpls), C.byref(gv), L.f3(cam), C.byref(params),
                                          C.byref(ov)), "arc_gather_bruteforce")


class AvplBvh:
    """LBVH over uploaded AVPLs (AvplBvh(avpls, considerNormals), bvh.cu:746-774)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        L.check(ctx.lib.arc_lbvh_create(ctx.handle, C.byref(h)), "arc_lbvh_create")
        self.handle = h
        ctx._children.add(self)

    def build(self, avpls: L.ArcAvplsGpuParam, consider_normals=False, bbox_mode=L.ARC_BBOX_SCENE,
              scene_min=(0, 0, 0), scene_max=(1, 1, 1), repr_seed=None, wait_limit=0) -> None:
        p = L.ArcLbvhParams()
        self.ctx.lib.arc_lbvh_params_default(C.byref(p))
        p.consider_normals = int(consider_normals)
        p.bbox_mode = bbox_mode
        p.scene_min = L.f3(scene_min)
        p.scene_max = L.f3(scene_max)
        p.wait_limit = int(wait_limit)
        if repr_seed is not None:
            p.repr_seed = repr_seed
        L.check(self.ctx.lib.arc_lbvh_build(self.handle, C.byref(avpls), C.byref(p)), "arc_lbvh_build")

    def view(self) -> L.ArcLbvhView:
        v = L.ArcLbvhView()
        L.check(self.ctx.lib.arc_lbvh_get_view(self.handle, C.byref(v)), "arc_lbvh_get_view")
        return v

    def host_arrays(self) -> dict:
        """Copy every tree array to host numpy arrays."""
        v = self.view()
        n = v.num_leaves
        t = 2 * n - 1
        d = self.ctx.d2h
        nd = v.node_data
        return {
            "morton": d(v.morton, np.uint32, n),
            "sorted_index": d(v.sorted_index, np.int32, n),
            "left": d(v.left, np.int32, n - 1),
            "right": d(v.right, np.int32, n - 1),
            "parents": d(v.parents, np.int32, t),
            "range": d(v.range, np.int32, 2 * (n - 1)).reshape(-1, 2),
            "bounds": d(v.bounds, np.float32, 16 * (n - 1)).reshape(-1, 16),
            "records": d(v.records, np.float32, 16 * t).reshape(-1, 16),
            "dirstat": d(v.dirstat, np.float32, 4 * t).reshape(-1, 4),
            "size": d(nd.size, np.int32, t),
            "materialIndex": d(nd.materialIndex, np.int32, t),
            "randomNumbers": d(nd.randomNumbers, np.float32, t),
            "position": d(nd.position, np.float32, 3 * t).reshape(-1, 3),
            "normal": d(nd.normal, np.float32, 3 * t).reshape(-1, 3),
            "incRadiance": d(nd.incRadiance, np.float32, 3 * t).reshape(-1, 3),
            "incDirection": d(nd.incDirection, np.float32, 3 * t).reshape(-1, 3),
        }

    def reference_views(self):
        bp, nd = L.ArcBvhParam(), L.ArcAvplBvhNodeDataParam()
        L.check(self.ctx.lib.arc_lbvh_reference_views(self.handle, C.byref(bp), C.byref(nd)),
                "arc_lbvh_reference_views")
        return bp, nd

    def close(self):
        if self.handle and self.ctx.handle:
            self.ctx.lib.arc_lbvh_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cut_params(kind=L.ARC_CUT_ERROR_BOUND, error_bound=0.01, solid_angle_threshold=math.pi / 10,
               max_cut_nodes=1 << 20, model=None, mlp_threshold=0.5, debug_pixel=(-1, -1), used_nodes=None,
               ar_uncertain_factor=16.0, cut_pool_entries=0, mlp_band=None):
    p = L.ArcCutParams()
    L.load().arc_cut_params_default(C.byref(p))
    p.kind = kind
    p.error_bound = error_bound
    p.ar_uncertain_factor = ar_uncertain_factor
    p.solid_angle_threshold = solid_angle_threshold
    p.max_cut_nodes = max_cut_nodes
    p.cut_pool_entries = cut_pool_entries
    p.model = model
    p.mlp_threshold = mlp_threshold
    if mlp_band is not None:
        p.mlp_band = mlp_band
    p.debug_pixel_x, p.debug_pixel_y = debug_pixel
    p.used_nodes = used_nodes
    return p


def gather_cut(ctx: Context, bvh: AvplBvh, avpls: L.ArcAvplsGpuParam | None, gb: GBuffer, cam,
               params: L.ArcGatherParams, cut: L.ArcCutParams, out: Outputs) -> None:
    gv, ov = gb.view(), out.view()
    ap = C.byref(avpls) if avpls is not None else None
    L.check(ctx.lib.arc_gather_cut(ctx.handle, bvh.handle, ap, C.byref(gv), L.f3(cam), C.byref(params), C.byref(cut),
                                   C.byref(ov)), "arc_gather_cut")


def last_cut(ctx: Context) -> list[np.ndarray]:
    """Cut node lists of the last tile-cut gather, one sorted array per tile."""
    cl = L.ArcCutLists()
    L.check(ctx.lib.arc_last_cut(ctx.handle, C.byref(cl)), "arc_last_cut")
    counts = ctx.d2h(cl.counts, np.int32, cl.num_tiles)
    tables = ctx.d2h(cl.tables, np.int32, cl.num_tiles * cl.max_chunks).reshape(cl.num_tiles, cl.max_chunks)
    pool = ctx.d2h(cl.pool, np.int32, cl.pool_chunks_used * cl.chunk_size).reshape(-1, cl.chunk_size)
    out = []
    for t in range(cl.num_tiles):
        k = int(counts[t])
        nch = (k + cl.chunk_size - 1) // cl.chunk_size
        ent = pool[tables[t, :nch]].ravel()[:k] if nch else np.zeros(0, np.int32)
        out.append(np.sort(ent))
    return out


def cut_counts(ctx: Context) -> np.ndarray:
    cl = L.ArcCutLists()
    L.check(ctx.lib.arc_last_cut(ctx.handle, C.byref(cl)), "arc_last_cut")
    return ctx.d2h(cl.counts, np.int32, cl.num_tiles)


def run_config(**kw) -> L.ArcRunConfig:
    c = L.ArcRunConfig()
    L.load().arc_run_config_default(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class CudaGather:
    """CudaGather (cudaGather.h:25-70) over a device G-buffer and output planes instead of GL
    textures."""

    def __init__(self, ctx: Context, gbuffer: GBuffer, materials, outputs: Outputs | None = None):
        self.ctx = ctx
        self.gbuffer = gbuffer
        self.outputs = outputs or Outputs(gbuffer.width, gbuffer.height, ctx.device)
        ctx.upload_materials(materials)

    def run(self, avpls: np.ndarray, camera_position, scene_extent: float, config: L.ArcRunConfig | None = None):
        config = config or run_config()
        avpls = np.ascontiguousarray(avpls, dtype=AVPL_DTYPE)
        gv, ov = self.gbuffer.view(), self.outputs.view()
        L.check(self.ctx.lib.arc_run(self.ctx.handle, avpls.ctypes.data_as(C.POINTER(L.ArcAvplHost)), len(avpls),
                                     L.f3(camera_position), float(scene_extent), C.byref(config), C.byref(gv),
                                     C.byref(ov)), "arc_run")
        return self.outputs


class Batch:
    """Multi-view batch renderer (arc_batch_*): per view an LBVH build and a cut gather, eagerly
    (render) or recorded once into a CUDA graph (capture) and replayed with one launch (launch)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        L.check(ctx.lib.arc_batch_create(ctx.handle, C.byref(h)), "arc_batch_create")
        self.handle = h
        self._views = None
        ctx._children.add(self)

    @staticmethod
    def views(items) -> C.Array:
        """items: (ArcAvplsGpuParam, GBuffer, camera, Outputs) per view."""
        arr = (L.ArcBatchView * len(items))()
        for i, (av, gb, cam, out) in enumerate(items):
            arr[i].avpls = av
            arr[i].gbuffer = gb.view()
            arr[i].camera_position = L.f3(cam)
            arr[i].out = out.view()
        return arr

    def render(self, views, lbvh: L.ArcLbvhParams, gather: L.ArcGatherParams, cut: L.ArcCutParams) -> None:
        L.check(self.ctx.lib.arc_batch_render(self.handle, views, len(views), C.byref(lbvh), C.byref(gather),
                                              C.byref(cut)), "arc_batch_render")

    def capture(self, views, lbvh: L.ArcLbvhParams, gather: L.ArcGatherParams, cut: L.ArcCutParams) -> None:
        self._views = views  # the recorded graph refers to these views' buffers
        L.check(self.ctx.lib.arc_batch_capture(self.handle, views, len(views), C.byref(lbvh), C.byref(gather),
                                               C.byref(cut)), "arc_batch_capture")

    def launch(self) -> None:
        L.check(self.ctx.lib.arc_batch_launch(self.handle), "arc_batch_launch")

    def close(self):
        if self.handle and self.ctx.handle:
            self.ctx.lib.arc_batch_destroy(self.handle)
        self.handle = None


class Accumulator:
    """FP64 running sums of the output planes over frames (arc_accumulate), normalised by the
    number of light paths (arc_accum_normalize): Renderer::Add / Normalize (Render.cpp:298-316)."""

    def __init__(self, ctx: Context, width: int, height: int, device: int = 0):
        torch = _torch()
        self.ctx, self.width, self.height = ctx, width, height
        self.sum = torch.zeros((height, width, 9), dtype=torch.float64, device=f"cuda:{device}")
        self.paths = 0

    def view(self) -> L.ArcAccumView:
        return L.ArcAccumView(self.sum.data_ptr(), self.width, self.height, self.width)

    def add(self, frame: "Outputs", paths: int = 0) -> None:
        L.check(self.ctx.lib.arc_accumulate(self.ctx.handle, C.byref(frame.view()), C.byref(self.view())),
                "arc_accumulate")
        self.paths += int(paths)

    def clear(self) -> None:
        L.check(self.ctx.lib.arc_accum_clear(self.ctx.handle, C.byref(self.view())), "arc_accum_clear")
        self.paths = 0

    def normalize(self, out: "Outputs", paths: int | None = None) -> "Outputs":
        n = self.paths if paths is None else int(paths)
        L.check(self.ctx.lib.arc_accum_normalize(self.ctx.handle, C.byref(self.view()), n, C.byref(out.view())),
                "arc_accum_normalize")
        return out


def image_error(ctx: Context, reference, image, metric: int = L.ARC_ERROR_RMSE):
    """(error, per-channel RMSE) of a device RGBA plane against a reference plane
    (arc_image_error; CReferenceImage::GetError with metric ARC_ERROR_REFERENCE)."""
    h, w = image.shape[:2]
    err = C.c_double(0.0)
    ch = (C.c_double * 3)()
    L.check(ctx.lib.arc_image_error(ctx.handle, C.c_void_p(reference.data_ptr()), C.c_void_p(image.data_ptr()), w, h,
                                    w, int(metric), C.byref(err), ch), "arc_image_error")
    return err.value, np.array(list(ch))


def export_pfm(path: str, rgba: np.ndarray) -> None:
    """Host [H, W, 4] float32 plane (row 0 = top) to a PFM file (arc_export_pfm)."""
    a = np.ascontiguousarray(rgba, np.float32)
    L.check(L.load().arc_export_pfm(str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0], a.shape[1]),
            "arc_export_pfm")


def export_hdr(path: str, rgba: np.ndarray) -> None:
    """Host [H, W, 4] float32 plane (row 0 = top) to a Radiance RGBE file (arc_export_hdr)."""
    a = np.ascontiguousarray(rgba, np.float32)
    L.check(L.load().arc_export_hdr(str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0], a.shape[1]),
            "arc_export_hdr")


class DeviceAvpls:
    """AVPLs in caller-owned device memory (a torch buffer) in the AvplsGpuParam layout: every
    instance keeps its own arrays, unlike Context.upload_avpls, which reuses one context buffer.
    `param` is the ArcAvplsGpuParam view.  DeviceAvpls(avpls) uploads host AVPLs;
    DeviceAvpls.empty(n) leaves room for n (e.g. for the GPU light tracer)."""

    _F3 = ("position", "normal", "incDirection", "incRadiance", "antiradiance")
    _I = ("materialIndex", "bounce")

    def __init__(self, avpls: np.ndarray | None, device: int = 0, count: int | None = None):
        torch = _torch()
        if avpls is not None:
            a = np.ascontiguousarray(avpls, dtype=AVPL_DTYPE)
            n = len(a)
            f3 = [np.ascontiguousarray(a[k], np.float32).reshape(-1) for k in self._F3]
            i2 = [np.ascontiguousarray(a[k], np.int32) for k in self._I]
            host = np.concatenate([x.view(np.uint8) for x in f3 + i2]) if n else np.zeros(64, np.uint8)
            self.buf = torch.from_numpy(host).to(f"cuda:{device}")
        else:
            n = int(count)
            self.buf = torch.zeros(max(68 * n, 64), dtype=torch.uint8, device=f"cuda:{device}")
        self.n = n
        base = self.buf.data_ptr()
        p = L.ArcAvplsGpuParam()
        off = [0]
        def take(nbytes):  # noqa: E306
            ptr = base + off[0]
            off[0] += nbytes
            return ptr
        p.position = take(12 * n)
        p.normal = take(12 * n)
        p.incDirection = take(12 * n)
        p.incRadiance = take(12 * n)
        p.antiradiance = take(12 * n)
        p.materialIndex = take(4 * n)
        p.bounce = take(4 * n)
        p.numAvpls = n
        self.param = p

    @classmethod
    def empty(cls, count: int, device: int = 0) -> "DeviceAvpls":
        return cls(None, device, count)

    def to_host(self) -> np.ndarray:
        """The AVPLs as a host array of AVPL_DTYPE (synchronises with torch's current stream)."""
        raw = self.buf.cpu().numpy()
        n = self.n
        out = np.zeros(n, dtype=AVPL_DTYPE)
        off = 0
        for k in self._F3:
            out[k] = raw[off:off + 12 * n].view(np.float32).reshape(n, 3)
            off += 12 * n
        for k in self._I:
            out[k] = raw[off:off + 4 * n].view(np.int32)
            off += 4 * n
        return out


def lbvh_params(**kw) -> L.ArcLbvhParams:
    p = L.ArcLbvhParams()
    L.load().arc_lbvh_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class TuningCache:
    """Brute-force launch shapes chosen by the autotuner, keyed by the workload (width, height,
    AVPL count, antiradiance kind, precision), kept in a JSON file (shipped beside the cut network
    as models/autotune.json) so that a later process applies a shape without timing again."""

    def __init__(self, path: str | None = None):
        import json
        import os

        self.path = path
        self.entries: dict[str, dict] = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.entries = json.load(f).get("bruteforce", {})

    @staticmethod
    def key(width: int, height: int, num_avpls: int, ar_kind: int, precision: int) -> str:
        return f"{width}x{height}x{num_avpls}:ar{ar_kind}:prec{precision}"

    def get(self, key: str) -> int | None:
        e = self.entries.get(key)
        return int(e["tile_config"]) if e is not None else None

    def put(self, key: str, tile_config: int, times_ms) -> None:
        self.entries[key] = {"tile_config": int(tile_config), "times_ms": [round(float(t), 3) for t in times_ms]}

    def save(self, path: str | None = None) -> None:
        import json

        with open(path or self.path, "w") as f:
            json.dump({"bruteforce": self.entries}, f, indent=1, sort_keys=True)


def autotune_bruteforce(ctx: Context, avpls: L.ArcAvplsGpuParam, gb: GBuffer, cam, params: L.ArcGatherParams,
                        out: Outputs, cache: TuningCache | None = None) -> tuple[int, np.ndarray]:
    """arc_autotune_bruteforce: (chosen tile_config, time of every shape in ms).  With a cache that
    holds this workload's shape, the shape is applied as the context default without timing (times
    then come from the cache)."""
    if cache is not None:
        key = TuningCache.key(gb.width, gb.height, avpls.numAvpls, params.ar_kind, params.precision)
        hit = cache.get(key)
        if hit is not None and 0 <= hit < ctx.lib.arc_bruteforce_num_tile_shapes():
            L.check(ctx.lib.arc_context_set_tile_config(ctx.handle, hit), "arc_context_set_tile_config")
            return hit, np.asarray(cache.entries[key]["times_ms"], np.float32)
    best, times = _autotune(ctx, avpls, gb, cam, params, out)
    if cache is not None:
        cache.put(key, best, times)
    return best, times


def _autotune(ctx: Context, avpls: L.ArcAvplsGpuParam, gb: GBuffer, cam, params: L.ArcGatherParams,
              out: Outputs) -> tuple[int, np.ndarray]:
    n = ctx.lib.arc_bruteforce_num_tile_shapes()
    times = np.zeros(n, np.float32)
    best = C.c_int32()
    gv, ov = gb.view(), out.view()
    L.check(ctx.lib.arc_autotune_bruteforce(ctx.handle, C.byref(avpls), C.byref(gv), L.f3(cam), C.byref(params),
                                            C.byref(ov), C.byref(best), times.ctypes.data_as(C.POINTER(C.c_float)),
                                            n), "arc_autotune_bruteforce")
    return int(best.value), times
