"""numpy interface to the CPU oracle (oracle.c -> liboracle.so) and to the reference's own
Morton code functions (_ref/libref_morton.so, compiled from the reference's morton.h).

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the benchmark's CPU-baseline leg use
this module as the checker / the timed CPU restatement.  The product (antiradiancecuts_b200)
never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_morton.so")

_lib = None
_ref = None


class OracleParams(C.Structure):
    _fields_ = [("ar_kind", C.c_int32), ("disk_radius", C.c_float), ("cone_half_angle", C.c_float),
                ("dist_clamp", C.c_float), ("geo_limit_radiance", C.c_float), ("geo_limit_antiradiance", C.c_float)]


INPUTS_LIB = os.path.join(HERE, "libinputs.so")


def build() -> None:
    """Compile liboracle.so, libinputs.so and, when the reference's Framework/ directory is found
    (environment variable ARC_REFERENCE_FRAMEWORK, else the checkout this recipe was written
    against), the reference Morton wrapper in _ref/."""
    ref = os.environ.get("ARC_REFERENCE_FRAMEWORK") or "/root/reference/Framework"
    cmd = ["make", "-s", "-C", HERE]
    if os.path.exists(os.path.join(ref, "morton.h")):
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
    return _lib


def ref_lib() -> C.CDLL | None:
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        _ref = C.CDLL(REF_LIB)
    return _ref


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def params(ar_kind=2, cone_half_angle_deg=30.0, dist_clamp=0.0, disk_radius=0.0, geo_limit_radiance=0.0,
           geo_limit_antiradiance=0.0) -> OracleParams:
    return OracleParams(ar_kind, disk_radius, math.radians(cone_half_angle_deg), dist_clamp, geo_limit_radiance,
                        geo_limit_antiradiance)


def _avpl_arrays(avpls):
    return (_f32(avpls["position"]), _f32(avpls["normal"]), _f32(avpls["incDirection"]), _f32(avpls["incRadiance"]),
            _f32(avpls["antiradiance"]), _i32(avpls["materialIndex"]))


def gather_fp64(pos4, nrm4, pixels, avpls, diffuse, specular, exponent, cam, prm: OracleParams, threads=0):
    """FP64 exact gather at the listed linear pixel indices -> (rad, antirad, result) [k,3]."""
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    pixels = _i32(pixels)
    k = len(pixels)
    a = _avpl_arrays(avpls)
    rad, ar, res = (np.zeros((k, 3), np.float64) for _ in range(3))
    cam = _f32(cam)
    dif, spe, ex = _f32(diffuse), _f32(specular), _f32(exponent)
    threads = threads or os.cpu_count() or 1
    lib().oracle_gather_fp64(_p(pos4), _p(nrm4), C.c_int32(0), _p(pixels), C.c_int32(k), *[_p(x) for x in a],
                             C.c_int32(len(avpls)), _p(dif), _p(spe), _p(ex), C.c_int32(len(dif)), _p(cam),
                             C.byref(prm), _p(rad), _p(ar), _p(res), C.c_int32(threads))
    return rad, ar, res


def clustered_disk_ar(pos4, nrm4, avpls, diffuse, specular, exponent, cam, z_near, theta, prm: OracleParams):
    """Clustered deferred disk antiradiance (oracle_clustered_disk_ar) over a whole [H, W] G-buffer
    -> (antiradiance [H*W, 3] FP64, number of clusters, list entries)."""
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    h, w = pos4.shape[:2]
    a = _avpl_arrays(avpls)
    out = np.zeros((h * w, 3), np.float64)
    dif, spe, ex = _f32(diffuse), _f32(specular), _f32(exponent)
    nc = C.c_int32(0)
    f = lib().oracle_clustered_disk_ar
    f.restype = C.c_int64
    entries = f(_p(pos4), _p(nrm4), C.c_int32(w), C.c_int32(h), _p(a[0]), _p(a[1]), _p(a[2]), _p(a[4]),
                C.c_int32(len(avpls)), _p(dif), _p(spe), _p(ex), C.c_int32(len(dif)), _p(_f32(cam)),
                C.c_float(z_near), C.c_float(theta), C.byref(prm), _p(out), C.byref(nc))
    return out, nc.value, int(entries)


def gather_fp32(pos4, nrm4, pixels, avpls, diffuse, specular, exponent, cam, prm: OracleParams, threads=1):
    """Scalar FP32 gather (the reference's arithmetic) -> result [k,3] float32."""
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    pixels = _i32(pixels)
    k = len(pixels)
    a = _avpl_arrays(avpls)
    res = np.zeros((k, 3), np.float32)
    cam = _f32(cam)
    dif, spe, ex = _f32(diffuse), _f32(specular), _f32(exponent)
    lib().oracle_gather_fp32(_p(pos4), _p(nrm4), C.c_int32(0), _p(pixels), C.c_int32(k), *[_p(x) for x in a],
                             C.c_int32(len(avpls)), _p(dif), _p(spe), _p(ex), C.c_int32(len(dif)), _p(cam),
                             C.byref(prm), _p(res), C.c_int32(threads))
    return res


def morton(pos, nrm=None, consider_normals=False, bbox_mode=0, scene_min=(0, 0, 0), scene_max=(1, 1, 1)):
    pos = _f32(pos)
    nrm = _f32(nrm if nrm is not None else np.zeros_like(pos))
    out = np.zeros(len(pos), np.uint32)
    smin, smax = _f32(scene_min), _f32(scene_max)  # kept alive across the call
    lib().oracle_morton(_p(pos), _p(nrm), C.c_int32(len(pos)), C.c_int32(int(consider_normals)), C.c_int32(bbox_mode),
                        _p(smin), _p(smax), _p(out))
    return out


def ref_morton3d(xyz):
    """The reference's MortonCode3D on points already in [0,1]^3 (None without _ref)."""
    r = ref_lib()
    if r is None:
        return None
    xyz = _f32(xyz)
    out = np.zeros(len(xyz), np.uint32)
    r.ref_morton3d(_p(xyz), C.c_int(len(xyz)), _p(out))
    return out


def ref_morton6d(a, b):
    r = ref_lib()
    if r is None:
        return None
    a, b = _f32(a), _f32(b)
    out = np.zeros(len(a), np.uint32)
    r.ref_morton6d_u32(_p(a), _p(b), C.c_int(len(a)), _p(out))
    return out


def stable_sort(keys):
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    perm = np.zeros(len(keys), np.int32)
    lib().oracle_stable_sort(_p(keys), C.c_int32(len(keys)), _p(perm))
    return perm


def karras(sorted_codes):
    m = np.ascontiguousarray(sorted_codes, dtype=np.uint32)
    n = len(m)
    left, right = np.zeros(n - 1, np.int32), np.zeros(n - 1, np.int32)
    parents = np.zeros(2 * n - 1, np.int32)
    lib().oracle_karras(_p(m), C.c_int32(n), _p(left), _p(right), _p(parents))
    return left, right, parents


def topdown(sorted_codes):
    m = np.ascontiguousarray(sorted_codes, dtype=np.uint32)
    n = len(m)
    left, right = np.zeros(n - 1, np.int32), np.zeros(n - 1, np.int32)
    lib().oracle_topdown(_p(m), C.c_int32(n), _p(left), _p(right))
    return left, right


def check_tree(left, right, parents):
    ms = C.c_int32(0)
    left, right, parents = _i32(left), _i32(right), _i32(parents)
    rc = lib().oracle_check_tree(_p(left), _p(right), _p(parents), C.c_int32(len(left) + 1), C.byref(ms))
    return int(rc), int(ms.value)


def bottom_up(sorted_avpls, diffuse, left, right, seed):
    """Bottom-up pass over sorted leaves -> dict of bounds / node data / records."""
    n = len(sorted_avpls)
    t = 2 * n - 1
    pos, nrm, w, L, A, mat = _avpl_arrays(sorted_avpls)
    diffuse, left, right = _f32(diffuse), _i32(left), _i32(right)
    out = {
        "bounds": np.zeros((max(n - 1, 1), 16), np.float32),
        "size": np.zeros(t, np.int32),
        "materialIndex": np.zeros(t, np.int32),
        "randomNumbers": np.zeros(t, np.float32),
        "position": np.zeros((t, 3), np.float32),
        "normal": np.zeros((t, 3), np.float32),
        "incRadiance": np.zeros((t, 3), np.float32),
        "incDirection": np.zeros((t, 3), np.float32),
        "records": np.zeros((t, 16), np.float32),
        "dirstat": np.zeros((t, 4), np.float32),
    }
    lib().oracle_bottom_up(C.c_int32(n), _p(pos), _p(nrm), _p(w), _p(L), _p(A), _p(mat), _p(diffuse),
                           _p(left), _p(right), C.c_uint32(seed), _p(out["bounds"]), _p(out["size"]),
                           _p(out["materialIndex"]), _p(out["randomNumbers"]), _p(out["position"]), _p(out["normal"]),
                           _p(out["incRadiance"]), _p(out["incDirection"]), _p(out["records"]), _p(out["dirstat"]))
    out["bounds"] = out["bounds"][: n - 1]
    return out


def build_tree(avpls, diffuse, seed=5489, bbox_mode=0, scene_min=(0, 0, 0), scene_max=(1, 1, 1),
               consider_normals=False):
    """Whole CPU LBVH: codes, stable order, Karras topology and bottom-up data."""
    codes = morton(avpls["position"], avpls["normal"], consider_normals, bbox_mode, scene_min, scene_max)
    perm = stable_sort(codes)
    sc = codes[perm]
    left, right, parents = karras(sc)
    bu = bottom_up(avpls[perm], diffuse, left, right, seed)
    return {"morton": sc, "sorted_index": perm, "left": left, "right": right, "parents": parents, **bu}


def cut_solid_angle(pos4, nrm4, pixels, tree, diffuse, specular, exponent, cam, thresh, dist_clamp=0.0, stack_cap=64,
                    threads=0):
    """Per-pixel solid-angle lightcut over `tree` (from build_tree or the GPU's host_arrays)."""
    pos4, nrm4, pixels = _f32(pos4), _f32(nrm4), _i32(pixels)
    n = len(tree["morton"])
    k = len(pixels)
    out = np.zeros((k, 3), np.float64)
    err = np.zeros(k, np.int32)
    b = _f32(tree["bounds"])
    npos, nnrm, nw, nL = (_f32(tree[x]) for x in ("position", "normal", "incDirection", "incRadiance"))
    nmat = _i32(tree["materialIndex"])
    dif, spe, ex, cam = _f32(diffuse), _f32(specular), _f32(exponent), _f32(cam)
    threads = threads or os.cpu_count() or 1
    lib().oracle_cut_solid_angle(_p(pos4), _p(nrm4), _p(pixels), C.c_int32(k), C.c_int32(n), _p(b), _p(npos), _p(nnrm),
                                 _p(nw), _p(nL), _p(nmat), _p(dif), _p(spe), _p(ex), C.c_int32(len(dif)), _p(cam),
                                 C.c_float(thresh), C.c_float(dist_clamp), C.c_int32(stack_cap), _p(out), _p(err),
                                 C.c_int32(threads))
    return out, err


def tile_cut(pos4, nrm4, tree, diffuse, eps_bound, dist_clamp, ar_kind, cone_half_angle_deg, disk_radius=0.0,
             max_cut=16384, ar_uncertain=16.0, threads=0):
    """Error-bound tile cuts -> (list of sorted node arrays per tile, tau per tile, overflow count)."""
    H, W = pos4.shape[:2]
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    n = len(tree["morton"])
    tiles = ((W + 7) // 8) * ((H + 7) // 8)
    nodes = np.zeros((tiles, max_cut), np.int32)
    counts = np.zeros(tiles, np.int32)
    tau = np.zeros(tiles, np.float32)
    b, r, dif = _f32(tree["bounds"]), _f32(tree["records"]), _f32(diffuse)
    threads = threads or os.cpu_count() or 1
    ov = lib().oracle_tile_cut(_p(pos4), _p(nrm4), C.c_int32(W), C.c_int32(H), C.c_int32(n), _p(b), _p(r), _p(dif),
                               C.c_int32(len(dif)), C.c_float(eps_bound), C.c_float(dist_clamp), C.c_int32(ar_kind),
                               C.c_float(math.radians(cone_half_angle_deg)), C.c_float(disk_radius),
                               C.c_float(ar_uncertain), C.c_int32(max_cut), _p(nodes), _p(counts), _p(tau),
                               C.c_int32(threads))
    return [np.sort(nodes[t, :counts[t]]) for t in range(tiles)], tau, int(ov)


def eval_cut(pos4, nrm4, tree, cuts, diffuse, ar_kind, cone_half_angle_deg, dist_clamp, disk_radius=0.0, threads=0):
    """FP64 evaluation of per-tile cuts -> (rad, antirad, result) [H*W, 3]."""
    H, W = pos4.shape[:2]
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    stride = max(1, max((len(c) for c in cuts), default=1))
    nodes = np.zeros((len(cuts), stride), np.int32)
    counts = np.zeros(len(cuts), np.int32)
    for t, c in enumerate(cuts):
        nodes[t, :len(c)] = c
        counts[t] = len(c)
    rad, ar, res = (np.zeros((H * W, 3), np.float64) for _ in range(3))
    r, dif = _f32(tree["records"]), _f32(diffuse)
    threads = threads or os.cpu_count() or 1
    lib().oracle_eval_cut(_p(pos4), _p(nrm4), C.c_int32(W), C.c_int32(H), _p(r), _p(nodes), _p(counts),
                          C.c_int32(stride), _p(dif), C.c_int32(len(dif)), C.c_int32(ar_kind),
                          C.c_float(math.radians(cone_half_angle_deg)), C.c_float(dist_clamp), C.c_float(disk_radius),
                          _p(rad), _p(ar), _p(res), C.c_int32(threads))
    return rad, ar, res


def node_bound(pos4, nrm4, tree, diffuse, tile, inner, eps_bound, dist_clamp, ar_kind, cone_half_angle_deg,
               ar_uncertain=16.0):
    """(bound, geom[7], tile info[14]) of one (tile, inner node) pair."""
    H, W = pos4.shape[:2]
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    n = len(tree["morton"])
    b, r, dif = _f32(tree["bounds"]), _f32(tree["records"]), _f32(diffuse)
    geom, tinfo = np.zeros(7, np.float32), np.zeros(14, np.float32)
    f = lib().oracle_node_bound
    f.restype = C.c_float
    m = f(_p(pos4), _p(nrm4), C.c_int32(W), C.c_int32(H), C.c_int32(tile), C.c_int32(n), _p(b), _p(r), _p(dif),
          C.c_int32(len(dif)), C.c_float(eps_bound), C.c_float(dist_clamp), C.c_int32(ar_kind),
          C.c_float(math.radians(cone_half_angle_deg)), C.c_float(ar_uncertain), C.c_int32(inner), _p(geom),
          _p(tinfo))
    return float(m), geom, tinfo


# --- learned cut ---------------------------------------------------------------------------------
# tile record columns: tmin(3) tmax(3) ncone(4) kdl tau mean valid rt sn
TREC_TAU, TREC_MEAN, TREC_VALID = 11, 12, 13


def tile_records(pos4, nrm4, tree, diffuse, eps_bound, dist_clamp, threads=0):
    """Per 8x8 tile: the quantities of the GPU's tile set-up -> float32 [tiles, 16]."""
    H, W = pos4.shape[:2]
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    n = len(tree["morton"])
    tiles = ((W + 7) // 8) * ((H + 7) // 8)
    out = np.zeros((tiles, 16), np.float32)
    b, r, dif = _f32(tree["bounds"]), _f32(tree["records"]), _f32(diffuse)
    lib().oracle_tile_records(_p(pos4), _p(nrm4), C.c_int32(W), C.c_int32(H), C.c_int32(n), _p(b), _p(r), _p(dif),
                              C.c_int32(len(dif)), C.c_float(eps_bound), C.c_float(dist_clamp), _p(out),
                              C.c_int32(threads or os.cpu_count() or 1))
    return out


def pair_features(trec, tiles, nodes, depths, tree, dist_clamp, ar_kind, cone_half_angle_deg, disk_radius=0.0,
                  ar_uncertain=16.0, threads=0):
    """(bound M [k], features [k, 16], conditioning [k, 4]) of (tile, inner node) pairs; nodes in
    record index space (inner k at n + k).  Conditioning: |rad - rad_l - rad_r| s, (|rad| + |rad_l| +
    |rad_r|) s and the same for antiradiance (features 12 and 13 are logs of the differences)."""
    tiles, nodes, depths = _i32(tiles), _i32(nodes), _i32(depths)
    k = len(tiles)
    n = len(tree["morton"])
    M = np.zeros(k, np.float32)
    F = np.zeros((k, 16), np.float32)
    A = np.zeros((k, 4), np.float32)
    b, r, ds = _f32(tree["bounds"]), _f32(tree["records"]), _f32(tree["dirstat"])
    trec = _f32(trec)
    lib().oracle_pair_features(_p(trec), C.c_int32(k), _p(tiles), _p(nodes), _p(depths), C.c_int32(n), _p(b), _p(r),
                               _p(ds), C.c_float(dist_clamp), C.c_int32(ar_kind),
                               C.c_float(math.radians(cone_half_angle_deg)), C.c_float(disk_radius),
                               C.c_float(ar_uncertain), _p(M), _p(F), _p(A), C.c_int32(threads or os.cpu_count() or 1))
    return M, F, A


def training_samples(pos4, nrm4, tree, diffuse, eps_bound, dist_clamp, ar_kind, cone_half_angle_deg, band, delta,
                     disk_radius=0.0, ar_uncertain=16.0, capacity=1 << 20, threads=0):
    """The learned cut's labelling walk with FP64 exact node contributions -> (keys [k, 2] = (tile,
    node), features [k, 16] float32, labels [k], errors [k]), tile after tile."""
    H, W = pos4.shape[:2]
    pos4, nrm4 = _f32(pos4), _f32(nrm4)
    n = len(tree["morton"])
    keys = np.zeros((capacity, 2), np.int32)
    F = np.zeros((capacity, 16), np.float32)
    lab = np.zeros(capacity, np.float32)
    err = np.zeros(capacity, np.float32)
    b, r, ds, dif = _f32(tree["bounds"]), _f32(tree["records"]), _f32(tree["dirstat"]), _f32(diffuse)
    f = lib().oracle_training_samples
    f.restype = C.c_int32
    k = f(_p(pos4), _p(nrm4), C.c_int32(W), C.c_int32(H), C.c_int32(n), _p(b), _p(r), _p(ds), _p(dif),
          C.c_int32(len(dif)), C.c_float(eps_bound), C.c_float(dist_clamp), C.c_int32(ar_kind),
          C.c_float(math.radians(cone_half_angle_deg)), C.c_float(disk_radius), C.c_float(ar_uncertain),
          C.c_float(band), C.c_float(delta), C.c_int32(capacity), _p(keys), _p(F), _p(lab), _p(err),
          C.c_int32(threads or os.cpu_count() or 1))
    k = min(k, capacity)
    return keys[:k], F[:k], lab[:k], err[:k]


def learned_cut(pos4, nrm4, tree, diffuse, params, eps_bound, ar_uncertain, band, thr_logit, dist_clamp, ar_kind,
                cone_half_angle_deg, disk_radius=0.0, threads=0, act="gelu"):
    """The learned cut selection, level by level: leaves and nodes whose bound is within tau are
    accepted, nodes above band * tau refined, the rest scored by the network (hidden activation
    `act`; BF16 rounding points of the tensor-core kernels, FP64 otherwise) and refined iff the
    logit reaches thr_logit.
    -> (sorted node array per tile, scored (tile, node, logit) rows)."""
    from . import mlp_oracle

    n = len(tree["morton"])
    trec = tile_records(pos4, nrm4, tree, diffuse, eps_bound, dist_clamp, threads)
    tiles_n = trec.shape[0]
    bounds = np.asarray(tree["bounds"], np.float32)
    lc = bounds[:, 3].view(np.int32)
    rc = bounds[:, 7].view(np.int32)
    lc = np.where(lc >= 0, lc, n - (lc + 1))
    rc = np.where(rc >= 0, rc, n - (rc + 1))
    ft = np.nonzero(trec[:, TREC_VALID] > 0)[0].astype(np.int32)
    fn = np.full(len(ft), n, np.int32)
    depth = 0
    acc_t, acc_n, scored = [], [], []
    band32 = np.float32(band)
    while len(ft):
        leaf = fn < n
        acc_t.append(ft[leaf])
        acc_n.append(fn[leaf])
        it, inn = ft[~leaf], fn[~leaf]
        M, F, _ = pair_features(trec, it, inn, np.full(len(it), depth, np.int32), tree, dist_clamp, ar_kind,
                                cone_half_angle_deg, disk_radius, ar_uncertain, threads)
        tau = trec[it, TREC_TAU]
        accept = ~(M > tau)
        refine = (M > band32 * tau) & ~accept
        score = ~accept & ~refine
        if score.any():
            y = mlp_oracle.forward_bf16(params, F[score], act)
            refine[np.nonzero(score)[0][y >= thr_logit]] = True
            scored.append(np.stack([it[score], inn[score], y], 1))
        done = ~refine
        acc_t.append(it[done])
        acc_n.append(inn[done])
        k = inn[refine] - n
        ft = np.concatenate([it[refine], it[refine]]).astype(np.int32)
        fn = np.concatenate([lc[k], rc[k]]).astype(np.int32)
        depth += 1
    at, an = np.concatenate(acc_t), np.concatenate(acc_n)
    order = np.lexsort((an, at))
    at, an = at[order], an[order]
    starts = np.searchsorted(at, np.arange(tiles_n + 1))
    cuts = [an[starts[t]:starts[t + 1]] for t in range(tiles_n)]
    return cuts, (np.concatenate(scored) if scored else np.zeros((0, 3)))
