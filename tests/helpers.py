"""Shared helpers of the test suite: cached workloads and image error metrics."""
from __future__ import annotations

import functools
import math

import numpy as np

from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import scene


@functools.lru_cache(maxsize=None)
def workload(name: str, width: int | None = None, height: int | None = None, num_avpls: int | None = None):
    w = scene.WORKLOADS[name]
    desc, avpls, paths, pos, nrm = w.build(width, height, num_avpls)
    mats, dif, spe, ex = scene.materials(desc)
    cam = (desc.camera_position.x, desc.camera_position.y, desc.camera_position.z)
    return {"w": w, "desc": desc, "avpls": avpls, "paths": paths, "pos": pos, "nrm": nrm, "mats": mats, "dif": dif,
            "spe": spe, "ex": ex, "cam": cam}


def rel_rmse(img, ref) -> float:
    """max over channels of RMSE(img - ref) / RMS(ref)."""
    img = np.asarray(img, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    num = np.sqrt(np.mean((img - ref) ** 2, axis=0))
    den = np.sqrt(np.mean(ref ** 2, axis=0)) + 1e-300
    return float(np.max(num / den))


def pixel_rel_err(img, ref, scale) -> np.ndarray:
    """Per-pixel max-channel |img - ref| / scale, scale = |radiance| + |antiradiance| of the oracle."""
    img = np.asarray(img, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    s = np.asarray(scale, np.float64).reshape(-1, 3)
    return np.max(np.abs(img - ref) / (s + 1e-30), axis=1)


def disk_radius(desc) -> float:
    return 2.0 * scene.scene_extent(desc) / 100.0
