#!/usr/bin/env python
"""ms/frame at 1920x1080 with 1,048,576 AVPLs: the cut gather (LBVH build + cut selection + cut
evaluation) against the exact brute-force gather, with the cut image's RMSE against an FP64 image.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--method learned|error_bound] [--small]
    python bench.py --impl reference      # the CPU gather (scalar FP32 restatement), same metric

One step = one frame rendered from device-resident inputs (AVPL arrays, G-buffer): LBVH build +
cut gather into HBM output planes.  Inputs (AVPLs 71 MB, G-buffer 66 MB) and the tree
(~0.9 GB) exceed the 126 MB L2, so no flush is needed between steps.  Under torchrun (N > 1)
every rank renders its own replica of the frame (the path does not shard across GPUs: replicas
only); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms/frame 1080p, 1M AVPLs: learned-cut vs exact gather at ≤1% RMSE (FP64)"
UNIT = "ms/frame"

# Algorithmic FLOPs of one (pixel, record) pair of the fast gather, Lambertian, counting FFMA = 2,
# FADD/FMUL/MUFU = 1, compares/selects = 0, per-pixel invariants hoisted:
#   radiance: d (3) + |d|^2 (5) + rsqrt (1) + n.d (5) + n_a.d (5) + 2 cosines (2) + r^2 (1)
#             + G (2) + 3 FFMA accumulate (6)                                        = 30
#   cone antiradiance: w.d (5) + cos (1) + G_A (1) + 3 FFMA accumulate (6)           = 13
#   disk antiradiance: w.n (5) + t (2) + hit (6) + |h - p|^2 (5) + 3 FFMA (6)         = 24
FLOP_PER_PAIR = {0: 30, 1: 54, 2: 43}
# MLP forward per scored row: 2 * (16*64 + 64*64 + 64*64 + 64) multiply-adds
FLOP_PER_ROW = 2 * (16 * 64 + 64 * 64 + 64 * 64 + 64)
# DRAM bytes (read + write) of all learned_level launches of a frame per scored row: one ncu capture
# of the 96 level launches of a 640x360 / 262,144-AVPL frame
# (profiles/learned_level_dram_640x360_262k.md), scaled to the frame by its scored rows
LEARNED_LEVEL_DRAM_BYTES_PER_ROW = 33.1


CALIBRATION = os.path.join(ROOT, "antiradiancecuts_b200", "models", "cutnet_calibration.json")
TUNING = os.path.join(ROOT, "antiradiancecuts_b200", "models", "autotune.json")


def calibrated_error_bound(default: float = 0.002) -> float:
    """The analytic cut's error bound chosen on the validation scenes (learned.calibrate)."""
    try:
        v = json.load(open(CALIBRATION))["analytic"]["chosen"]
        return float(v) if v is not None else default
    except (OSError, KeyError, ValueError):
        return default


def lbvh_bytes_per_avpl() -> dict:
    """Compulsory DRAM bytes per AVPL of each LBVH kernel (reads + writes of its inputs and
    outputs once, N leaves and N - 1 inner nodes)."""
    return {
        "lbvh_morton": 12 + 8,                     # positions in; key + index out
        "lbvh_sort": 4 * (8 + 8),                  # 4 passes: (key, index) in and out
        # codes, index, AVPL in; leaf records, cones, direction statistics, node data out
        "lbvh_karras": (4 + 4 + 64) + (16 + 4 + 64 + 32 + 16 + 24 + 60 + 24),
        "lbvh_bottom_up": 2 * (24 + 12 + 4 + 64 + 32 + 16) + (24 + 60 + 64 + 32 + 16 + 64),
    }


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(backend: str | None = None):
    """One process per GPU under torchrun: (world size, rank, local rank).  The process group is
    NCCL on GPUs; gloo (CPU) when asked for, as the multi-process tests do."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend or "nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _on_gpu() -> bool:
    import torch.distributed as dist

    return dist.get_backend() == "nccl"


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist

        if _on_gpu():
            dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            dist.barrier()


def max_over_ranks(world, x: float) -> float:
    """The maximum of x over the ranks (step times: the job takes as long as its slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if _on_gpu() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def host_threads() -> int:
    """The host cores this process may run on (its affinity mask, not the machine's count)."""
    try:
        return len(os.sched_getaffinity(0)) or 1
    except AttributeError:
        return os.cpu_count() or 1


def cgroup_cpu() -> dict:
    """This process's cgroup CPU bandwidth limit (quota / period in cores, None = unlimited) and the
    throttling counters so far (cgroup v2 cpu.max / cpu.stat, else v1 cpu.cfs_* / cpu.stat)."""
    out = {"quota_cores": None, "throttled_s": None, "nr_throttled": None}

    def read(path):
        try:
            with open(path) as f:
                return f.read().split()
        except OSError:
            return None

    v2 = read("/sys/fs/cgroup/cpu.max")
    if v2 and len(v2) == 2:
        if v2[0] != "max":
            out["quota_cores"] = int(v2[0]) / max(1, int(v2[1]))
        st = read("/sys/fs/cgroup/cpu.stat") or []
        kv = dict(zip(st[0::2], st[1::2]))
        if "throttled_usec" in kv:
            out["throttled_s"] = int(kv["throttled_usec"]) * 1e-6
            out["nr_throttled"] = int(kv.get("nr_throttled", 0))
        return out
    q, per = read("/sys/fs/cgroup/cpu/cpu.cfs_quota_us"), read("/sys/fs/cgroup/cpu/cpu.cfs_period_us")
    if q and per and int(q[0]) > 0:
        out["quota_cores"] = int(q[0]) / max(1, int(per[0]))
    st = read("/sys/fs/cgroup/cpu/cpu.stat") or []
    kv = dict(zip(st[0::2], st[1::2]))
    if "throttled_time" in kv:
        out["throttled_s"] = int(kv["throttled_time"]) * 1e-9
        out["nr_throttled"] = int(kv.get("nr_throttled", 0))
    return out


def host_cpu_times():
    """(busy, steal, total) jiffies over all CPUs of the host (/proc/stat), or None."""
    try:
        with open("/proc/stat") as f:
            v = [int(x) for x in f.readline().split()[1:]]
    except (OSError, ValueError):
        return None
    idle = v[3] + (v[4] if len(v) > 4 else 0)
    steal = v[7] if len(v) > 7 else 0
    total = sum(v[:8])
    return total - idle - steal, steal, total


def _cpu_gather_sample(O, pos, nrm, order, avpls, dif, spe, ex, cam, prm, target_s: float, threads: int):
    """Runs the scalar FP32 CPU gather over chunks of the pixel list `order` until target_s seconds
    of gather time are spent (or the list is done) -> (pixels gathered, seconds).  Every chunk is a
    multiple of `threads` pixels and the gather hands out one pixel at a time, so no thread idles
    while another still has pixels; after the first chunk each is sized to about a quarter of the
    remaining time at the rate measured so far."""
    k, dt, cpu, chunk = 0, 0.0, 0.0, threads
    while k < len(order) and dt < target_s:
        part = order[k:k + chunk]
        t0, c0 = time.perf_counter(), time.process_time()
        O.gather_fp32(pos, nrm, part, avpls, dif, spe, ex, cam, prm, threads=threads)
        dt += time.perf_counter() - t0
        cpu += time.process_time() - c0
        k += len(part)
        want = (k / max(dt, 1e-6)) * max(target_s - dt, 0.0) / 4
        chunk = max(threads, int(want // threads) * threads)
    return k, dt, cpu


def cpu_baseline(wl, desc, avpls, pos, nrm, dif, spe, ex, cam, target_s: float, threads: int, ref64=None,
                 single_s: float = 0.0) -> dict:
    """The scalar FP32 CPU gather (oracle restatement of the reference's formulas, -O3) on a seeded
    pixel sample over all AVPLs, with `threads` host threads, extrapolated to the full frame; with
    single_s > 0 also one thread for single_s seconds.  With ref64 (the all-FP64 GPU image,
    [pixels, 3]) it also checks that image against the CPU FP64 oracle on 64 sampled pixels."""
    from oracle import oracle as O

    prm = O.params(wl.ar_kind, wl.cone_half_angle_deg, wl.dist_clamp)
    valid = np.nonzero(nrm.reshape(-1, 4)[:, 3] > 0)[0]
    order = np.random.default_rng(7).permutation(valid)
    import resource

    cg0, hs0, ru0 = cgroup_cpu(), host_cpu_times(), resource.getrusage(resource.RUSAGE_SELF)
    k, dt, cpu = _cpu_gather_sample(O, pos, nrm, order, avpls, dif, spe, ex, cam, prm, target_s, threads)
    cg1, hs1, ru1 = cgroup_cpu(), host_cpu_times(), resource.getrusage(resource.RUSAGE_SELF)
    host = None
    if hs0 and hs1 and hs1[2] > hs0[2]:
        tot = hs1[2] - hs0[2]
        # busy and steal shares of every CPU of the host, this process's threads included
        host = {"busy": (hs1[0] - hs0[0]) / tot, "steal": (hs1[1] - hs0[1]) / tot, "cpus": os.cpu_count()}
    # every pixel costs the same (all AVPLs); background pixels cost nothing, so extrapolate over
    # the valid pixels
    ms_frame = dt * 1e3 * len(valid) / max(k, 1)
    single = None
    if single_s > 0:
        k1, dt1, _ = _cpu_gather_sample(O, pos, nrm, order, avpls, dif, spe, ex, cam, prm, single_s, 1)
        single = {"value": dt1 * 1e3 * len(valid) / max(k1, 1), "unit": UNIT, "cores": 1,
                  "sample": f"{k1} random surface pixels x {len(avpls)} AVPLs, {dt1:.1f} s"}
    sample = order[:k]
    check = None
    if ref64 is not None:
        px = sample[:64]
        _, _, o64 = O.gather_fp64(pos, nrm, px, avpls, dif, spe, ex, cam, prm, threads=threads)
        d = ref64[px] - o64
        check = float(np.max(np.sqrt(np.mean(d ** 2, 0)) / (np.sqrt(np.mean(o64 ** 2, 0)) + 1e-300)))
    out = {"value": ms_frame, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"{k} random surface pixels x {len(avpls)} AVPLs (scalar FP32 C, -O3, {threads} threads, "
                     f"one pixel per work item), {dt:.1f} s, extrapolated to {len(valid)} surface pixels",
           # the host is shared with other jobs: the cores the gather actually got (process CPU time
           # over wall time) and the load average when it ran
           "cpu_seconds_per_second": cpu / max(dt, 1e-9), "loadavg_1min": os.getloadavg()[0],
           # a CPU bandwidth limit on the process's cgroup, and how long it held the gather back
           "cgroup_quota_cores": cg1["quota_cores"],
           "cgroup_throttled_s": (cg1["throttled_s"] - cg0["throttled_s"]) if cg0["throttled_s"] is not None else None,
           "cgroup_nr_throttled": (cg1["nr_throttled"] - cg0["nr_throttled"]) if cg0["nr_throttled"] is not None else None,
           # the host's CPUs during the sample, and how often the kernel took a core from a gather
           # thread (involuntary) or a thread gave it up (voluntary)
           "host_cpu": host,
           "context_switches": {"involuntary": ru1.ru_nivcsw - ru0.ru_nivcsw, "voluntary": ru1.ru_nvcsw - ru0.ru_nvcsw}}
    if single is not None:
        out["single_thread"] = single
    if ref64 is not None:
        out["fp64_image_vs_oracle_rel_rmse"] = check
    return out


def scene_leg(ctx, api, scene, wl, desc, avpls, pos, nrm, stream) -> dict:
    """The benchmark frame's inputs made on the GPU (arc_scene_trace_avpls_device,
    arc_scene_gbuffer_device) against the CPU generator that made them (all host threads): times,
    whether the G-buffers are the same bits, and how far the AVPLs are from the CPU's (the azimuth's
    cos / sin come from different math libraries)."""
    import torch

    N, H, W = len(avpls), pos.shape[0], pos.shape[1]
    t0 = time.perf_counter()
    cpu_av, _ = scene.trace_avpls(desc, wl.avpl_seed, N, wl.max_bounces)
    cpu_av_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    scene.gbuffer(desc, W, H)
    cpu_gb_ms = (time.perf_counter() - t0) * 1e3
    dv, _ = scene.trace_avpls_device(ctx, desc, wl.avpl_seed, N, wl.max_bounces)  # warm-up
    gb = scene.gbuffer_device(ctx, desc, W, H)
    assert ctx.synchronize() == 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dv, _ = scene.trace_avpls_device(ctx, desc, wl.avpl_seed, N, wl.max_bounces)
    e1.record(stream)
    torch.cuda.synchronize()
    gpu_av_ms = e0.elapsed_time(e1)
    e0.record(stream)
    gb = scene.gbuffer_device(ctx, desc, W, H)
    e1.record(stream)
    torch.cuda.synchronize()
    gpu_gb_ms = e0.elapsed_time(e1)
    assert ctx.synchronize() == 0
    got = dv.to_host()
    same_ints = all(np.array_equal(got[k], avpls[k]) for k in ("bounce", "materialIndex"))
    pos_diff = float(np.abs(got["position"].astype(np.float64) - avpls["position"]).max()) if same_ints else None
    gb_equal = np.array_equal(gb.pos.cpu().numpy(), pos) and np.array_equal(gb.nrm.cpu().numpy(), nrm)
    return {"avpls": N, "resolution": [W, H], "gpu_ms_avpls": gpu_av_ms, "gpu_ms_gbuffer": gpu_gb_ms,
            "cpu_ms_avpls": cpu_av_ms, "cpu_ms_gbuffer": cpu_gb_ms, "cpu_threads": os.cpu_count(),
            "gbuffer_bit_equal": bool(gb_equal), "avpl_bounces_materials_equal": bool(same_ints),
            "avpl_max_position_diff": pos_diff}


def post_leg(ctx, api, L, out, stream, hbm_gbs: float) -> dict:
    """After the gather, at the frame's resolution: accumulating the frame's three planes into FP64
    sums (arc_accumulate), normalising them (arc_accum_normalize) and the image error against
    another plane (arc_image_error); device times and the accumulation's HBM roofline
    (3 float4 read, 9 doubles read and written = 192 B per pixel)."""
    import torch

    W, H = out.width, out.height
    acc = api.Accumulator(ctx, W, H)
    norm = api.Outputs(W, H, fp64=False, parts=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    acc.add(out, paths=1)  # warm-up
    reps = 10
    e0.record(stream)
    for _ in range(reps):
        acc.add(out, paths=1)
    e1.record(stream)
    torch.cuda.synchronize()
    acc_ms = e0.elapsed_time(e1) / reps
    e0.record(stream)
    acc.normalize(norm)
    e1.record(stream)
    torch.cuda.synchronize()
    norm_ms = e0.elapsed_time(e1)
    e0.record(stream)
    err, _ = api.image_error(ctx, out.result, norm.result, L.ARC_ERROR_RMSE)
    e1.record(stream)
    torch.cuda.synchronize()
    err_ms = e0.elapsed_time(e1)
    assert ctx.synchronize() == 0
    gbs = 192.0 * W * H / (acc_ms * 1e-3) / 1e9
    return {"accumulate_ms": acc_ms, "normalize_ms": norm_ms, "image_error_ms_incl_readback": err_ms,
            "accumulate_roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm_gbs, "unit": "GB/s",
                                    "frac": gbs / hbm_gbs}, "frames_averaged_error": err}


def clustered_leg(ctx, api, scene, L, desc, mats, dv, gb, cam, stream) -> dict:
    """Disk antiradiance of the benchmark frame (radius 2% of the scene extent, the reference's
    photonRadiusScale 2) through screen clusters and light lists (arc_antiradiance_clustered)
    against the brute-force disk antiradiance (antiradiance plane of arc_gather_bruteforce):
    device times, list entries and the relative RMSE between the two."""
    import torch

    ctx.upload_materials(mats)  # the frame's materials (the batch leg uploads its own scene's)
    r = 2.0 * scene.scene_extent(desc) / 100.0
    prm = api.gather_params(L.ARC_AR_DISK, 30.0, 0.0, disk_radius=r)
    cp = L.ArcClusterParams(0.1, math.radians(0.5 * desc.camera_fov_deg))
    W, H = gb.width, gb.height
    out = api.Outputs(W, H, fp64=False, parts=True)
    ref = api.Outputs(W, H, fp64=False, parts=True)
    info = L.ArcClusterInfo()

    def clustered():
        L.check(ctx.lib.arc_antiradiance_clustered(ctx.handle, C.byref(dv), C.byref(gb.view()), L.f3(cam), C.byref(cp),
                                                   C.byref(prm), C.byref(out.view()), C.byref(info)),
                "arc_antiradiance_clustered")

    clustered()  # warm-up
    word = ctx.synchronize()
    assert word == 0, f"device error word 0x{word:x} in the clustered antiradiance"
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    clustered()
    e1.record(stream)
    torch.cuda.synchronize()
    cl_ms = e0.elapsed_time(e1)
    e0.record(stream)
    api.gather_bruteforce(ctx, dv, gb, cam, prm, ref)
    e1.record(stream)
    torch.cuda.synchronize()
    bf_ms = e0.elapsed_time(e1)
    assert ctx.synchronize() == 0
    a = out.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3).astype(np.float64)
    b = ref.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3).astype(np.float64)
    rel = float(np.max(np.sqrt(np.mean((a - b) ** 2, 0)) / (np.sqrt(np.mean(b ** 2, 0)) + 1e-300)))
    return {"disk_radius": r, "clustered_ms_incl_list_readback": cl_ms, "bruteforce_disk_ms": bf_ms,
            "list_entries": int(info.list_entries), "rel_rmse_vs_bruteforce": rel}


# compulsory DRAM bytes per AVPL of an LBVH build (the survey's minimum: bbox read 12, Morton 16,
# sort 4 passes x 16 with histograms, payload permute 128, Karras writes 12, bottom-up 204)
LBVH_MIN_BYTES_PER_AVPL = 470


def lbvh_sweep_leg(ctx, api, scene, L, desc, sizes, hbm_gbs: float, stream) -> dict:
    """LBVH build time per stage at several AVPL counts (AVPLs made by the GPU light tracer), with
    the achieved bandwidth against both the survey's compulsory 470 B/AVPL and this design's
    itemised bytes (lbvh_bytes_per_avpl)."""
    import torch

    design = sum(lbvh_bytes_per_avpl().values())
    names = C.create_string_buffer(4096)
    st_ms = (C.c_float * 256)()
    nst = C.c_int32()
    rows = []
    for n in sizes:
        dv, _ = scene.trace_avpls_device(ctx, desc, 7, n, 3)
        bvh = api.AvplBvh(ctx)
        bvh.build(dv.param)  # warm-up (sizes the arena)
        assert ctx.synchronize() == 0
        reps = 3
        ctx.lib.arc_context_profile(ctx.handle, 1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            bvh.build(dv.param)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        ctx.lib.arc_context_stage_times(ctx.handle, names, 4096, st_ms, 256, C.byref(nst))
        ctx.lib.arc_context_profile(ctx.handle, 0)
        stages = {}
        for nme, v in zip(names.value.decode().split(","), list(st_ms)[: nst.value]):
            stages[nme] = stages.get(nme, 0.0) + v / reps
        assert ctx.synchronize() == 0
        gbs_min = LBVH_MIN_BYTES_PER_AVPL * n / (ms * 1e-3) / 1e9
        gbs_design = design * n / (ms * 1e-3) / 1e9
        rows.append({"avpls": n, "ms": ms, "stage_ms": stages,
                     "achieved_gbs_at_470_b": gbs_min, "frac_at_470_b": gbs_min / hbm_gbs,
                     "achieved_gbs_at_design_b": gbs_design, "frac_at_design_b": gbs_design / hbm_gbs})
        bvh.close()
        del dv
        torch.cuda.empty_cache()
    return {"sizes": rows, "bytes_per_avpl_min": LBVH_MIN_BYTES_PER_AVPL, "bytes_per_avpl_design": design,
            "peak_gbs": hbm_gbs, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}


def seeds_leg(ctx, model, error_bound: float, seeds) -> dict:
    """The headline comparison on more than one scene: for each room variant seed at 1920x1080 with
    1,048,576 AVPLs, the learned cut (the model's calibrated threshold), the analytic cut (at its
    calibrated bound) and the exact brute-force gather, each timed on the GPU and scored against
    the scene's all-FP64 image (relative RMSE and max relative error).  The operating points were
    chosen on other scenes (the validation seeds), so none of these is a tuning scene."""
    from antiradiancecuts_b200 import api, learned

    rows = []
    for s in seeds:
        sc = learned.EvalScene(ctx, s)
        pool = sc.tiles * 65536
        lc = sc.cut(learned.cut_params(model, cut_pool_entries=pool), reps=3) if model is not None else None
        an = sc.cut(api.cut_params(api.L.ARC_CUT_ERROR_BOUND, error_bound=error_bound,
                                   ar_uncertain_factor=learned.PREACCEPT_K, cut_pool_entries=pool), reps=2)
        ex = sc.exact(reps=1)
        row = {"seed": s, "surface_pixels": sc.surface_pixels, "exact": ex, "analytic": an}
        if lc is not None:
            row["learned"] = lc
            row["speedup_learned_vs_exact"] = ex["ms"] / lc["ms"]
        row["speedup_analytic_vs_exact"] = ex["ms"] / an["ms"]
        rows.append(row)
        sc.close()
        del sc
    return {"scenes": rows, "analytic_error_bound": error_bound,
            "mlp_threshold": model.threshold if model is not None else None,
            "all_learned_within_1pct": all(r["learned"]["rel_rmse"] <= 0.01 for r in rows) if model else None}


def batch_leg(ctx, api, scene, L, stream, num_views: int, model=None) -> dict:
    """Multi-view batch: views of the room + 2 boxes scene drawn with seed 4 (resolutions from
    {256^2, 512^2, 1280x720, 1920x1080}, 8,192 - 262,144 AVPLs each, log-uniform, camera inside the
    room), each with its own AVPL set; per view an LBVH build and an error-bound cut gather (eps
    0.01).  Timed as the views one after another on the context's stream (serial), as a batch on
    concurrent lanes (eager), and as one recorded CUDA graph launch; with a model, the learned cut's
    batch recorded into a graph too."""
    import torch

    desc = scene.scene_desc(L.ARC_SCENE_ROOM_2BOXES, 2, 2)
    mats, _, _, _ = scene.materials(desc)
    ctx.upload_materials(mats)
    items, keep = [], []
    pixels = avpl_total = 0
    for v in scene.batch_views(desc, 4, num_views):
        avpls, pos, nrm = scene.view_inputs(desc, v)
        dv = api.DeviceAvpls(avpls)
        out = api.Outputs(v.width, v.height, fp64=False, parts=False)
        keep.append((dv, out))
        items.append((dv.param, api.GBuffer(pos, nrm), (v.camera_position.x, v.camera_position.y, v.camera_position.z),
                      out))
        pixels += v.width * v.height
        avpl_total += v.num_avpls
    views = api.Batch.views(items)
    lp, gp = api.lbvh_params(), api.gather_params(L.ARC_AR_CONE, 30.0, 0.01)
    cp = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.01)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    # serial: one view after another on the context's stream
    bvh = api.AvplBvh(ctx)

    def serial():
        for av, gbv, cam, out in items:
            L.check(ctx.lib.arc_lbvh_build(bvh.handle, C.byref(av), C.byref(lp)), "arc_lbvh_build")
            api.gather_cut(ctx, bvh, av, gbv, cam, gp, cp, out)

    serial()
    assert ctx.synchronize() == 0
    e0.record(stream)
    for _ in range(reps):
        serial()
    e1.record(stream)
    torch.cuda.synchronize()
    serial_ms = e0.elapsed_time(e1) / reps
    bvh.close()
    b = api.Batch(ctx)
    b.render(views, lp, gp, cp)  # warm-up (sizes every buffer)
    assert ctx.synchronize() == 0
    e0.record(stream)
    for _ in range(reps):
        b.render(views, lp, gp, cp)
    e1.record(stream)
    torch.cuda.synchronize()
    eager = e0.elapsed_time(e1) / reps
    b.capture(views, lp, gp, cp)
    b.launch()
    assert ctx.synchronize() == 0
    e0.record(stream)
    for _ in range(reps):
        b.launch()
    e1.record(stream)
    torch.cuda.synchronize()
    graph = e0.elapsed_time(e1) / reps
    assert ctx.synchronize() == 0
    learned_graph = None
    if model is not None:
        from antiradiancecuts_b200 import learned

        b.capture(views, lp, gp, learned.cut_params(model))
        b.launch()
        assert ctx.synchronize() == 0
        e0.record(stream)
        for _ in range(reps):
            b.launch()
        e1.record(stream)
        torch.cuda.synchronize()
        learned_graph = e0.elapsed_time(e1) / reps
        assert ctx.synchronize() == 0
    b.close()
    return {"views": num_views, "pixels": pixels, "avpls": avpl_total, "ms_per_batch_serial": serial_ms,
            "ms_per_batch_eager": eager, "ms_per_batch_graph": graph, "graph_launches_per_batch": 1,
            "lanes": 4, "cut": "error bound 0.01", "views_per_s": num_views * 1000.0 / graph,
            "ms_per_batch_graph_learned": learned_graph}


def run_reference(args):
    """--impl reference: the CPU gather on the host cores (rank 0 only)."""
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    # the inputs come from the scene generator's source built without the GPU library
    # (oracle/libinputs.so): this process loads no GPU code
    from antiradiancecuts_b200 import _lib as L
    from antiradiancecuts_b200 import scene
    from oracle import oracle as O

    if not os.path.exists(O.INPUTS_LIB):
        O.build()
    wl = scene.WORKLOADS[args.workload]
    desc, avpls, paths, pos, nrm = wl.build(lib=L.load_scene_library(O.INPUTS_LIB))
    _, dif, spe, ex = scene.materials(desc)
    cam = (desc.camera_position.x, desc.camera_position.y, desc.camera_position.z)
    threads = host_threads()
    per = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    vals, cores, thr = [], [], []
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(wl, desc, avpls, pos, nrm, dif, spe, ex, cam, per, threads)
        if i >= args.warmup:
            vals.append(b["value"])
            cores.append(b["cpu_seconds_per_second"])
            thr.append(b["cgroup_throttled_s"])
    v = float(np.median(vals))
    b["value"] = v
    b["per_step_values"] = [round(x, 1) for x in vals]
    b["per_step_cpu_seconds_per_second"] = [round(x, 2) for x in cores]
    b["per_step_cgroup_throttled_s"] = [None if x is None else round(x, 2) for x in thr]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "resolution": [wl.width, wl.height], "avpls": wl.num_avpls,
                       "method": "exact brute-force gather on the CPU (the reference has no CPU gather: scalar "
                                 "FP32 restatement of cudaGather.cu / Gather.frag formulas)"},
            "cpu_baseline": b, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="variant500_1080p_1m")
    ap.add_argument("--method", default="auto", choices=["auto", "learned", "error_bound"])
    ap.add_argument("--error-bound", type=float, default=None,
                    help="analytic cut bound (default: the one calibrated on the validation scenes)")
    ap.add_argument("--seeds", default="500,501,502,503", help="scenes of the per-scene comparison ('' = none)")
    ap.add_argument("--autotune", action="store_true",
                    help="time every brute-force launch shape and store the best in models/autotune.json")
    ap.add_argument("--small", action="store_true", help="640x360 / 262,144 AVPLs, no extras (profiling)")
    ap.add_argument("--no-extras", action="store_true", help="skip exact / FP64 / CPU legs")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="all-core CPU baseline sample")
    ap.add_argument("--cpu-single-seconds", type=float, default=5.0, help="single-thread CPU baseline sample")
    ap.add_argument("--batch-views", type=int, default=32, help="views of the multi-view batch leg")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.error_bound is None:
        args.error_bound = calibrated_error_bound()

    import torch

    from antiradiancecuts_b200 import _lib as L
    from antiradiancecuts_b200 import api, scene

    world, rank, local = dist_init()
    if world > 1:
        # replicas: the extra legs (exact and FP64 gathers, analytic cut, batch, scene, post,
        # clustered) repeat one GPU's measurements on every rank, and the CPU baseline belongs to
        # the single-GPU run, where no other rank loads the host cores
        args.no_extras = True
    torch.cuda.set_device(local)
    ctx = api.Context(local)
    lib = ctx.lib
    wl = scene.WORKLOADS[args.workload]
    if args.small:
        W, H, N = 640, 360, 262144
        args.no_extras = True
    else:
        W, H, N = wl.width, wl.height, wl.num_avpls
    desc, avpls, paths, pos, nrm = wl.build(W, H, N)
    mats, dif, spe, ex = scene.materials(desc)
    cam = (desc.camera_position.x, desc.camera_position.y, desc.camera_position.z)
    ctx.upload_materials(mats)
    dv = ctx.upload_avpls(avpls)
    gb = api.GBuffer(pos, nrm)
    out = api.Outputs(W, H)
    bvh = api.AvplBvh(ctx)
    prm = api.gather_params(wl.ar_kind, wl.cone_half_angle_deg, wl.dist_clamp)

    method = args.method
    model = None
    from antiradiancecuts_b200 import learned

    if method in ("auto", "learned"):
        try:
            model = learned.load_default_model(ctx)
            method = "learned"
        except Exception as e:  # no trained model available
            if args.method == "learned":
                raise
            method = "error_bound"
            model_error = str(e)
    kind = L.ARC_CUT_LEARNED if method == "learned" else L.ARC_CUT_ERROR_BOUND
    tiles = ((W + 7) // 8) * ((H + 7) // 8)
    pool = tiles * 65536
    if model is not None:
        cut = learned.cut_params(model, cut_pool_entries=pool)
    else:
        cut = api.cut_params(kind, error_bound=args.error_bound, cut_pool_entries=pool)

    stream = ctx.stream  # the context's stream (also torch's current stream)

    def frame():
        bvh.build(dv)
        api.gather_cut(ctx, bvh, None, gb, cam, prm, cut, out)

    for _ in range(args.warmup):
        frame()
    word = ctx.synchronize()
    assert word == 0, f"device error word 0x{word:x} during warm-up"
    barrier(world)
    torch.cuda.synchronize()
    lib.arc_context_profile(ctx.handle, 1)
    launches0 = lib.arc_context_launch_count(ctx.handle)
    rows0 = lib.arc_context_learned_rows(ctx.handle)
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        frame()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    launches = lib.arc_context_launch_count(ctx.handle) - launches0
    rows_per_frame = (lib.arc_context_learned_rows(ctx.handle) - rows0) / args.steps
    names = C.create_string_buffer(4096)
    st_ms = (C.c_float * 256)()
    nst = C.c_int32()
    lib.arc_context_stage_times(ctx.handle, names, 4096, st_ms, 256, C.byref(nst))
    lib.arc_context_profile(ctx.handle, 0)
    stage_names = names.value.decode().split(",") if nst.value else []
    per_stage = {}
    for nme, v in zip(stage_names, list(st_ms)[: nst.value]):
        per_stage[nme] = per_stage.get(nme, 0.0) + v / args.steps
    assert ctx.synchronize() == 0, "device error during the timed frames"
    barrier(world)
    ms = max_over_ranks(world, ms)

    # ---- roofline of the dominant kernel ----
    counts = api.cut_counts(ctx).astype(np.int64)
    valid_px = (nrm[..., 3] > 0)
    tiles_x, tiles_y = (W + 7) // 8, (H + 7) // 8
    vp = np.zeros((tiles_y * 8, tiles_x * 8), np.int64)
    vp[:H, :W] = valid_px
    valid_per_tile = vp.reshape(tiles_y, 8, tiles_x, 8).sum(axis=(1, 3)).ravel()
    pairs = int((counts * valid_per_tile).sum())
    cut_stats = {"mean": float(counts.mean()), "p50": float(np.median(counts)), "p99": float(np.percentile(counts, 99)),
                 "max": int(counts.max()), "pairs": pairs, "exact_pairs": int(valid_px.sum()) * N}
    sc, pk = C.c_double(), C.c_double()
    L.check(lib.arc_measure_fp32_peak(ctx.handle, C.byref(sc), C.byref(pk)), "arc_measure_fp32_peak")
    fp32_peak = max(sc.value, pk.value)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}
    dom = max(per_stage, key=per_stage.get) if per_stage else "cut_eval"
    eval_roof = None
    if "cut_eval" in per_stage:
        ach = pairs * FLOP_PER_PAIR[wl.ar_kind] / (per_stage["cut_eval"] * 1e-3) / 1e12
        eval_roof = {"kernel": "cut_eval", "bound": "fp32", "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": ach / fp32_peak, "traffic": None, "ms": per_stage["cut_eval"],
                     "peak_source": "measured FFMA microbenchmark (arc_measure_fp32_peak), max of scalar/packed"}
    if dom == "cut_eval":
        roof = dict(eval_roof)
    elif dom == "cut_learned":
        # the fused level kernel's algorithmic work is the network's forward pass over the scored
        # rows (feature computation and frontier expansion are counted as overhead)
        bf16 = peaks.get("bf16_tflops", 1590.0)
        ach = rows_per_frame * FLOP_PER_ROW / (per_stage[dom] * 1e-3) / 1e12
        roof = {"kernel": "learned_level", "bound": "tensor", "achieved": ach, "peak": bf16, "unit": "TFLOP/s",
                "frac": ach / bf16, "traffic": LEARNED_LEVEL_DRAM_BYTES_PER_ROW * rows_per_frame,
                "traffic_scope": "bytes of the frame's 96 level launches (the unit `achieved` is taken over): "
                                 f"{LEARNED_LEVEL_DRAM_BYTES_PER_ROW} B per scored row from a 640x360 capture "
                                 "x rows_per_frame",
                "rows_per_frame": rows_per_frame,
                "flop_per_row": FLOP_PER_ROW, "ms": per_stage[dom],
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if "bf16_tflops" in peaks else "fallback"}
    elif dom.startswith("lbvh"):
        b = lbvh_bytes_per_avpl()[dom] * N
        ach = b / (per_stage[dom] * 1e-3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"], "traffic": None, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
    else:
        roof = {"kernel": dom, "bound": "latency", "achieved": None, "peak": None, "unit": None, "frac": None,
                "traffic": None}
    lb_ms = sum(v for k, v in per_stage.items() if k.startswith("lbvh"))
    lb_bytes = sum(lbvh_bytes_per_avpl().values()) * N
    lbvh_roof = {"achieved": lb_bytes / (lb_ms * 1e-3) / 1e9 if lb_ms else None, "peak": peaks["hbm_gbs"],
                 "unit": "GB/s", "frac": (lb_bytes / (lb_ms * 1e-3) / 1e9) / peaks["hbm_gbs"] if lb_ms else None,
                 "ms": lb_ms, "bytes_per_avpl": sum(lbvh_bytes_per_avpl().values()),
                 "frac_at_470_b": (LBVH_MIN_BYTES_PER_AVPL * N / (lb_ms * 1e-3) / 1e9) / peaks["hbm_gbs"]
                 if lb_ms else None}

    result = {}
    cut_img = out.result64.cpu().numpy().reshape(-1, 3).copy()
    if not args.no_extras:
        # ---- exact brute-force gather (same GPU), in the launch shape the autotuner chose for this
        # workload (models/autotune.json; --autotune times every shape and updates the file) ----
        prm_bf = api.gather_params(wl.ar_kind, wl.cone_half_angle_deg, wl.dist_clamp)
        out_bf = api.Outputs(W, H)
        tcache = api.TuningCache(TUNING)
        tkey = api.TuningCache.key(W, H, N, prm_bf.ar_kind, prm_bf.precision)
        tuned = tcache.get(tkey)
        if args.autotune or tuned is not None:
            tuned, _ = api.autotune_bruteforce(ctx, dv, gb, cam, prm_bf, out_bf, cache=None if args.autotune else tcache)
            if args.autotune:
                tcache.put(tkey, tuned, _)
                tcache.save()
        api.gather_bruteforce(ctx, dv, gb, cam, prm_bf, out_bf)  # warm-up
        torch.cuda.synchronize()
        lib.arc_context_profile(ctx.handle, 1)
        e0.record(stream)
        for _ in range(2):
            api.gather_bruteforce(ctx, dv, gb, cam, prm_bf, out_bf)
        e1.record(stream)
        torch.cuda.synchronize()
        exact_ms = e0.elapsed_time(e1) / 2
        lib.arc_context_stage_times(ctx.handle, names, 4096, st_ms, 256, C.byref(nst))
        lib.arc_context_profile(ctx.handle, 0)
        bf_stage = {}
        for nme, v in zip(names.value.decode().split(","), list(st_ms)[: nst.value]):
            bf_stage[nme] = bf_stage.get(nme, 0.0) + v / 2
        bf_pairs = int(valid_px.sum()) * N
        bf_ach = bf_pairs * FLOP_PER_PAIR[wl.ar_kind] / (bf_stage.get("bf_gather", exact_ms) * 1e-3) / 1e12
        # ---- FP64 image (all-FP64 GPU gather), checked against the CPU FP64 oracle on a sample ----
        prm64 = api.gather_params(wl.ar_kind, wl.cone_half_angle_deg, wl.dist_clamp, precision=L.ARC_PREC_FP64)
        out64 = api.Outputs(W, H)
        api.gather_bruteforce(ctx, dv, gb, cam, prm64, out64)
        assert ctx.synchronize() == 0
        ref64 = out64.result64.cpu().numpy().reshape(-1, 3)
        exact_img = out_bf.result64.cpu().numpy().reshape(-1, 3)

        def rel_rmse(a, b):
            return float(np.max(np.sqrt(np.mean((a - b) ** 2, 0)) / (np.sqrt(np.mean(b ** 2, 0)) + 1e-300)))

        # ---- the analytic error-bound cut at the bound that keeps it within 1% (the method the
        # learned cut is measured against) ----
        out_an = api.Outputs(W, H)
        cut_an = api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=args.error_bound, cut_pool_entries=pool)

        def frame_an():
            bvh.build(dv)
            api.gather_cut(ctx, bvh, None, gb, cam, prm, cut_an, out_an)

        frame_an()
        assert ctx.synchronize() == 0
        e0.record(stream)
        for _ in range(2):
            frame_an()
        e1.record(stream)
        torch.cuda.synchronize()
        an_ms = e0.elapsed_time(e1) / 2
        an_nodes = float(api.cut_counts(ctx).mean())
        assert ctx.synchronize() == 0
        result = {
            "analytic_cut": {"error_bound": args.error_bound, "ms_per_frame": an_ms,
                             "rel_rmse_vs_fp64": rel_rmse(out_an.result64.cpu().numpy().reshape(-1, 3), ref64),
                             "nodes_per_tile": an_nodes},
            "exact_ms_per_frame": exact_ms,
            "exact_tile_config": tuned if tuned is not None else "built-in",
            "speedup_vs_exact": exact_ms / ms,
            "rel_rmse_vs_fp64": rel_rmse(cut_img, ref64),
            "exact_rel_rmse_vs_fp64": rel_rmse(exact_img, ref64),
            "exact_roofline": {"kernel": "bf_gather", "bound": "fp32", "achieved": bf_ach, "peak": fp32_peak,
                               "unit": "TFLOP/s", "frac": bf_ach / fp32_peak},
        }

    # ---- e2e through the public API: CudaGather::run with host AVPLs, result read back ----
    g = api.CudaGather(ctx, gb, mats, outputs=api.Outputs(W, H, fp64=False, parts=False))
    rcfg = api.run_config(useLightCuts=1, cut_kind=kind, error_bound=cut.error_bound, ar_kind=wl.ar_kind,
                          cone_half_angle=math.radians(wl.cone_half_angle_deg), dist_clamp=wl.dist_clamp,
                          model=model.handle.value if model else None, ar_uncertain_factor=cut.ar_uncertain_factor,
                          mlp_threshold=cut.mlp_threshold, mlp_band=cut.mlp_band, cut_pool_entries=pool)
    host_out = torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True)
    for _ in range(args.warmup):
        g.run(avpls, cam, scene.scene_extent(desc), rcfg)
        host_out.copy_(g.outputs.result, non_blocking=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        g.run(avpls, cam, scene.scene_extent(desc), rcfg)
        host_out.copy_(g.outputs.result, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1) / args.steps)

    cpu = None
    if rank == 0 and not args.no_extras:
        cpu = cpu_baseline(wl, desc, avpls, pos, nrm, dif, spe, ex, cam, args.cpu_seconds, host_threads(),
                           ref64=ref64, single_s=args.cpu_single_seconds)
        result["fp64_image_vs_cpu_oracle_rel_rmse"] = cpu.pop("fp64_image_vs_oracle_rel_rmse")

    batch = gen = post = clus = seeds = sweep = None
    if not args.no_extras and args.seeds:
        seeds = seeds_leg(ctx, model, args.error_bound, [int(x) for x in args.seeds.split(",")])
        ctx.upload_materials(mats)
    if not args.no_extras:
        torch.cuda.empty_cache()  # the per-scene leg's tensors: the batch's lanes allocate outside torch
        batch = batch_leg(ctx, api, scene, L, stream, args.batch_views, model)
        gen = scene_leg(ctx, api, scene, wl, desc, avpls, pos, nrm, stream)
        post = post_leg(ctx, api, L, out, stream, lbvh_roof["peak"])
        clus = clustered_leg(ctx, api, scene, L, desc, mats, dv, gb, cam, stream)
        sweep = lbvh_sweep_leg(ctx, api, scene, L, desc, (1 << 20, 1 << 22, 1 << 24), lbvh_roof["peak"], stream)
        ctx.upload_materials(mats)

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload if not args.small else args.workload + "_small",
                       "resolution": [W, H], "avpls": N, "light_paths": paths, "method": method,
                       "error_bound": cut.error_bound, "ar_uncertain_factor": cut.ar_uncertain_factor,
                       "mlp_threshold": cut.mlp_threshold if model else None,
                       "mlp_band": cut.mlp_band if model else None, "antiradiance": "cone", "cone_half_angle_deg":
                           wl.cone_half_angle_deg, "dist_clamp": wl.dist_clamp,
                       "l2": "inputs larger than L2 (AVPLs 71 MB, G-buffer 66 MB, tree ~0.9 GB); no flush",
                       "parallelism": f"replicas x{world}", "frames_per_s_all_gpus": world * 1000.0 / ms},
            "stage_ms": per_stage, "cut_nodes_per_tile": cut_stats, "gpu_launches": int(launches), "launches_per_frame": launches / args.steps,
            "roofline": roof, "cut_eval_roofline": eval_roof, "lbvh_roofline": lbvh_roof, **result,
            "e2e": {"value": e2e_ms, "unit": UNIT, "h2d_bytes_per_step": int(68 * N),
                    "d2h_bytes_per_step": int(W * H * 16)},
            "cpu_baseline": cpu, "clocks": clk, "batch": batch, "scene_generation": gen, "post": post,
            "clustered_antiradiance": clus, "scenes": seeds, "lbvh_sweep": sweep,
        }
        if method != "learned" and args.method == "auto":
            line["config"]["learned_unavailable"] = model_error[:200]
        print(json.dumps(line))
    barrier(world)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
