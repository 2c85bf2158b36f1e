#!/usr/bin/env python
"""Precision-stress report (high cancellation): the brute-force gather in every precision mode
against FP64 references, per channel.

Workload (defaults): room with 16 random boxes (PCG32 seed 3), 1920x1080, 262,144 AVPLs
(<= 5 bounces), cone antiradiance 60 deg, distance clamp 0.005.  Modes:
    NAIVE         FP32 terms, plain FP32 sums, FP32 combine (the reference's arithmetic)
    KAHAN         FP32 terms, per-chunk FP32 partials folded into Kahan sums, FP64 combine (default)
    KAHAN_STRICT  FP32 terms, every term Kahan-added, FP64 combine
    FP64          every operation in FP64
References: the all-FP64 GPU image over the full frame, and the CPU FP64 oracle on a seeded sample
of surface pixels (which also pins the FP64 GPU image).  Errors are per channel: relative RMSE
(RMSE / RMS of the reference), and the maximum relative error over pixels,
|x - ref| / max(|ref|, 1e-3 RMS(ref)).

    python tests/precision_report.py [--width W] [--height H] [--avpls N] [--sample K]

prints a Markdown report (the summary under profiles/ was made with the defaults on one B200).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

MODES = [("NAIVE", 2), ("KAHAN", 0), ("KAHAN_STRICT", 1), ("FP64", 3)]


def channel_errors(x: np.ndarray, ref: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(relative RMSE, max relative error) per channel of [k, 3] images."""
    x = np.asarray(x, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    rms = np.sqrt(np.mean(ref ** 2, axis=0))
    rel_rmse = np.sqrt(np.mean((x - ref) ** 2, axis=0)) / rms
    floor = 1e-3 * rms
    max_rel = np.max(np.abs(x - ref) / np.maximum(np.abs(ref), floor), axis=0)
    return rel_rmse, max_rel


def measure(width=1920, height=1080, num_avpls=262144, sample=4096, workload="boxes16_1080p_256k"):
    """Images and timings of every mode plus the oracle sample; returns a dict of results."""
    import torch

    from antiradiancecuts_b200 import _lib as L
    from antiradiancecuts_b200 import api, scene
    from oracle import oracle as O

    ctx = api.Context(0)
    wl = scene.WORKLOADS[workload]
    desc, avpls, _, pos, nrm = wl.build(width, height, num_avpls)
    mats, dif, spe, ex = scene.materials(desc)
    cam = (desc.camera_position.x, desc.camera_position.y, desc.camera_position.z)
    ctx.upload_materials(mats)
    dv = ctx.upload_avpls(avpls)
    gb = api.GBuffer(pos, nrm)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    images, times, parts = {}, {}, {}
    for name, prec in MODES:
        prm = api.gather_params(wl.ar_kind, wl.cone_half_angle_deg, wl.dist_clamp, precision=prec)
        out = api.Outputs(width, height)
        api.gather_bruteforce(ctx, dv, gb, cam, prm, out)
        assert ctx.synchronize() == 0
        e0.record(ctx.stream)
        api.gather_bruteforce(ctx, dv, gb, cam, prm, out)
        e1.record(ctx.stream)
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1)
        images[name] = out.result64.cpu().numpy().reshape(-1, 3).copy()
        parts[name] = (out.radiance.cpu().numpy()[..., :3].reshape(-1, 3).astype(np.float64),
                       out.antiradiance.cpu().numpy()[..., :3].reshape(-1, 3).astype(np.float64))
    valid = np.nonzero(nrm.reshape(-1, 4)[:, 3] > 0)[0]
    rng = np.random.default_rng(3)
    px = rng.choice(valid, size=min(sample, len(valid)), replace=False)
    t0 = time.perf_counter()
    _, _, oracle = O.gather_fp64(pos, nrm, px, avpls, dif, spe, ex, cam,
                                 O.params(wl.ar_kind, wl.cone_half_angle_deg, wl.dist_clamp))
    oracle_s = time.perf_counter() - t0
    rad64, ar64 = parts["FP64"]
    cancel = np.sqrt(np.mean(rad64[valid] ** 2, 0)) / np.sqrt(np.mean(images["FP64"][valid] ** 2, 0))
    return {"width": width, "height": height, "avpls": num_avpls, "surface_pixels": len(valid), "sample": len(px),
            "cone_half_angle_deg": wl.cone_half_angle_deg, "dist_clamp": wl.dist_clamp, "times_ms": times,
            "vs_fp64_gpu": {n: channel_errors(images[n][valid], images["FP64"][valid]) for n, _ in MODES},
            "vs_oracle": {n: channel_errors(images[n][px], oracle) for n, _ in MODES},
            "rad_over_result_rms": cancel, "oracle_seconds": oracle_s}


def report(r) -> str:
    fmt = lambda v: " / ".join(f"{x:.2e}" for x in v)  # noqa: E731
    lines = [f"Workload: {r['width']}x{r['height']}, {r['avpls']:,} AVPLs, cone {r['cone_half_angle_deg']} deg, "
             f"distance clamp {r['dist_clamp']}; {r['surface_pixels']:,} surface pixels.  Cancellation: RMS of the "
             f"radiance / RMS of the result = {fmt(r['rad_over_result_rms'])} (R / G / B).",
             "",
             "| mode | ms/frame | rel. RMSE vs FP64 GPU (R / G / B) | max rel. error vs FP64 GPU | "
             f"rel. RMSE vs CPU FP64 oracle ({r['sample']} px) | max rel. error vs oracle |",
             "|---|---:|---|---|---|---|"]
    for n, _ in MODES:
        a, b = r["vs_fp64_gpu"][n], r["vs_oracle"][n]
        lines.append(f"| {n} | {r['times_ms'][n]:.1f} | {fmt(a[0])} | {fmt(a[1])} | {fmt(b[0])} | {fmt(b[1])} |")
    return "\n".join(lines)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--avpls", type=int, default=262144)
    ap.add_argument("--sample", type=int, default=4096)
    a = ap.parse_args(argv)
    print(report(measure(a.width, a.height, a.avpls, a.sample)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
