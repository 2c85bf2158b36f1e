"""Generates the golden fixtures of tests/golden/.

    python tests/golden/make_golden.py

morton_ref.npz
    Points and the Morton codes the reference's own morton.h computes for them (MortonCode3D,
    and MortonCode6D truncated to 32 bits), via oracle/_ref/libref_morton.so, which
    oracle/Makefile compiles from the reference tree.  Needs that library, i.e. the reference
    tree, when it is regenerated; the tests only read the frozen file.
gather_kat.json
    Known-answer gather cases whose expected radiance / antiradiance follow in closed form from
    the reference's formulas (cudaGather.cu:45-144, Shaders/Gather.frag:149-208): one pixel, one
    AVPL, geometry chosen so every cosine, distance and reflection is exact.
scene_gen.json
    SHA-256 digests of the synthetic-scene generator's outputs (G-buffer planes and traced AVPLs
    of the preset scenes at small sizes), so that a change to the generator's arithmetic, which
    would move every benchmark and training input, shows in the CPU tests.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def make_morton():
    from oracle import oracle as O

    rng = np.random.default_rng(20240611)
    pts = rng.random((4096, 3), dtype=np.float32)
    # edge values: exact cell boundaries, 0, 1, and values just below 1
    edge = np.array([[0, 0, 0], [1, 1, 1], [0.5, 0.25, 0.125], [1023 / 1024, 1 / 1024, 0.999999],
                     [np.nextafter(np.float32(1), np.float32(0))] * 3, [-0.1, 1.1, 0.5]], dtype=np.float32)
    pts = np.concatenate([edge, pts]).astype(np.float32)
    nrm = rng.random((len(pts), 3), dtype=np.float32)
    c3 = O.ref_morton3d(pts)
    c6 = O.ref_morton6d(pts, nrm)
    if c3 is None:
        raise SystemExit("oracle/_ref/libref_morton.so missing: run `make -C oracle` with the reference tree present")
    np.savez_compressed(os.path.join(HERE, "morton_ref.npz"), points=pts, normals01=nrm, codes3=c3, codes6=c6)


def make_kat():
    inv_pi = 1.0 / math.pi
    cases = []
    rho = 0.5     # receiver albedo (material 1)
    rho_a = 0.7   # AVPL albedo (material 2)
    base = {"materials": [[0, 0, 0], [rho, rho, rho], [rho_a, rho_a, rho_a]], "specular": [[0, 0, 0]] * 3,
            "exponent": [1, 1, 1], "pixel_pos": [0, 0, 0], "pixel_nrm": [0, 1, 0], "pixel_mat": 1,
            "cam": [0, 1, -1]}
    # 1: AVPL straight above, facing down: G = 1, rad = L rho_a/pi rho/pi; cone AR accepted with G_A = 1
    L, A = [1.0, 2.0, 3.0], [4.0, 5.0, 6.0]
    c = dict(base, name="above_facing_down", avpl_pos=[0, 1, 0], avpl_nrm=[0, -1, 0], avpl_w=[0, -1, 0], L=L, A=A,
             avpl_mat=2, ar_kind=2, half_angle_deg=30.0, clamp=0.0)
    c["rad"] = [x * rho_a * inv_pi * rho * inv_pi for x in L]
    c["ar"] = [x * rho * inv_pi for x in A]
    cases.append(c)
    # 2: same at distance 2: G = 1/4, G_A = 1/4
    c = dict(c, name="above_dist2", avpl_pos=[0, 2, 0])
    c["rad"] = [x * rho_a * inv_pi * rho * inv_pi / 4 for x in L]
    c["ar"] = [x * rho * inv_pi / 4 for x in A]
    cases.append(c)
    # 3: distance 0.005 with clamp 0.01: 1/d^2 -> 1/0.01^2
    c = dict(c, name="clamped", avpl_pos=[0, 0.005, 0], clamp=0.01)
    c["rad"] = [x * rho_a * inv_pi * rho * inv_pi * 1e4 for x in L]
    c["ar"] = [x * rho * inv_pi * 1e4 for x in A]
    cases.append(c)
    # 4: AVPL at 45 deg: w straight down, so the pixel is 45 deg off the cone axis
    s = 1 / math.sqrt(2)
    c = dict(base, name="cone_reject_45", avpl_pos=[-s, s, 0], avpl_nrm=[s, -s, 0], avpl_w=[0, -1, 0], L=L, A=A,
             avpl_mat=2, ar_kind=2, half_angle_deg=30.0, clamp=0.0)
    # n . w^ = cos 45, n_a . (-w^) = 1, d = 1  -> G = cos 45
    c["rad"] = [x * rho_a * inv_pi * rho * inv_pi * s for x in L]
    c["ar"] = [0.0, 0.0, 0.0]
    cases.append(c)
    c = dict(c, name="cone_accept_60", half_angle_deg=60.0)
    c["ar"] = [x * rho * inv_pi * s for x in A]  # G_A = n.(-avpl_to_pos) / d^2 = cos 45
    cases.append(c)
    # 6: AVPL above facing up (light passed through it): radiance 0 (n_a faces away), disk AR hit at the
    # pixel itself: A rho/pi / (pi r^2); cone AR: G_A = 1
    r = 0.25
    c = dict(base, name="disk_hit", avpl_pos=[0, 1, 0], avpl_nrm=[0, 1, 0], avpl_w=[0, -1, 0], L=L, A=A, avpl_mat=2,
             ar_kind=1, disk_radius=r, half_angle_deg=30.0, clamp=0.0)
    c["rad"] = [0.0, 0.0, 0.0]
    c["ar"] = [x * rho * inv_pi / (math.pi * r * r) for x in A]
    cases.append(c)
    c = dict(c, name="disk_miss", avpl_pos=[0.3, 1, 0])  # hit point 0.3 from the pixel > r
    c["ar"] = [0.0, 0.0, 0.0]
    cases.append(c)
    c = dict(c, name="cone_behind", avpl_pos=[0, 1, 0], ar_kind=2)
    c["ar"] = [x * rho * inv_pi for x in A]
    cases.append(c)
    # 9: light-source AVPL (w = 0): brdf_light = 1 (cudaGather.cu:88-90)
    c = dict(base, name="light_source_avpl", avpl_pos=[0, 1, 0], avpl_nrm=[0, -1, 0], avpl_w=[0, 0, 0], L=L,
             A=[0, 0, 0], avpl_mat=2, ar_kind=2, half_angle_deg=30.0, clamp=0.0)
    c["rad"] = [x * rho * inv_pi for x in L]
    c["ar"] = [0.0, 0.0, 0.0]
    cases.append(c)
    # 10: specular receiver, mirror configuration: reflect(-w_i, n) == w_o, cos = 1
    e = 8.0
    ks = 0.3
    c = dict(base, name="specular_mirror", materials=[[0, 0, 0], [rho, rho, rho], [rho_a, rho_a, rho_a]],
             specular=[[0, 0, 0], [ks, ks, ks], [0, 0, 0]], exponent=[1, e, 1], avpl_pos=[-s, s, 0],
             avpl_nrm=[s, -s, 0], avpl_w=[s, -s, 0], L=L, A=[0, 0, 0], avpl_mat=2, ar_kind=0, half_angle_deg=30.0,
             clamp=0.0, cam=[1, 1, 0])
    fr = rho * inv_pi + 0.5 * inv_pi * (e + 2) * ks
    c["rad"] = [x * rho_a * inv_pi * fr * s for x in L]
    c["ar"] = [0.0, 0.0, 0.0]
    cases.append(c)
    with open(os.path.join(HERE, "gather_kat.json"), "w") as f:
        json.dump(cases, f, indent=1)


SCENE_CASES = [(0, 0, 0), (1, 2, 2), (2, 3, 16), (3, 500, 0)]  # (preset, seed, boxes)


def scene_digests() -> dict:
    """Digests of scene.gbuffer (40 x 24) and scene.trace_avpls (4096 AVPLs, seed 7, 3 bounces)
    for each preset case."""
    import hashlib

    from antiradiancecuts_b200 import scene

    out = {}
    for preset, seed, boxes in SCENE_CASES:
        desc = scene.scene_desc(preset, seed, boxes)
        pos, nrm = scene.gbuffer(desc, 40, 24)
        av, paths = scene.trace_avpls(desc, 7, 4096, 3)
        key = f"{preset}/{seed}/{boxes}"
        out[key] = {"gbuffer": hashlib.sha256(pos.tobytes() + nrm.tobytes()).hexdigest(),
                    "avpls": hashlib.sha256(av.tobytes()).hexdigest(), "paths": int(paths)}
    return out


def make_scene():
    with open(os.path.join(HERE, "scene_gen.json"), "w") as f:
        json.dump(scene_digests(), f, indent=1)


if __name__ == "__main__":
    if "--scene-only" not in sys.argv:
        make_morton()
        make_kat()
    make_scene()
    print("wrote", os.listdir(HERE))
