// Tile-level cut decision math shared by the error-bound and learned cut selections.  Every
// operation is explicitly rounded and ordered so that the CPU oracle reproduces each decision
// bit for bit.
#ifndef ARC_CUT_BOUNDS_CUH_
#define ARC_CUT_BOUNDS_CUH_

#include "arc_internal.h"
#include "device_common.cuh"

namespace arc {

struct TileInfo {
    float tmin[3], tmax[3];  // bounding box of the tile's valid pixel positions
    float4 ncone;            // union of the valid pixels' normal cones
    float kdl;               // max luminance of the receivers' diffuse/pi
    float tau;               // error threshold: eps * mean coarse estimate
    int valid;               // valid pixel count
    float rt;                // half-diagonal of the box (half_diagonal)
    float sn;                // sine of the normal cone's half-angle (cone_sine)
};

// Per inner node, the pair-independent parts of node_geom / node_bound, computed once per cut
// selection (cut_node_extra) with the same rounded operations, so the results are unchanged.
struct NodeExtra {
    float rn;   // half-diagonal of the node's box
    float snc;  // sine of the normal cone's half-angle
    float swc;  // sine of the direction cone's half-angle
    float Ls;   // luminance of the summed radiance
    float As;   // luminance of the summed antiradiance
    float cn[3];  // centre of the node's box, 0.5 (bmin + bmax)
};

// two float4 per inner node: {rn, snc, swc, Ls}, {As, centre}
__device__ __forceinline__ NodeExtra load_node_extra(const float4* ext, int k) {
    const float4 e0 = ext[2 * (size_t)k], e1 = ext[2 * (size_t)k + 1];
    return NodeExtra{e0.x, e0.y, e0.z, e0.w, e1.x, {e1.y, e1.z, e1.w}};
}

struct BoundParams {
    float clamp2;    // dist clamp squared (0 = off)
    int ar_kind;
    float cos_thr;   // cone: max(cos(half angle), 0.001)
    float eps_cone;  // 0.001
    float disk_scale;
    float ar_uncertain;  // bound multiplier when the cone test may differ between the node's pairs
};

__device__ __forceinline__ float lum3(float r, float g, float b) {
    return rn_add(rn_add(rn_mul(0.2126f, r), rn_mul(0.7152f, g)), rn_mul(0.0722f, b));
}

// sin of a cone's half-angle from its cosine
__device__ __forceinline__ float cone_sine(float c) { return rn_sqrt(fmaxf(0.0f, rn_sub(1.0f, rn_mul(c, c)))); }

// half the length of a box's diagonal (extents ex, ey, ez)
__device__ __forceinline__ float half_diagonal(float ex, float ey, float ez) {
    return rn_mul(0.5f, rn_sqrt(rn_dot(ex, ey, ez, ex, ey, ez)));
}

// max over members of two cones of cos(angle between them), clamped to [0, 1] is left to the
// caller; returns 1 when the cones overlap.  (a1, c1, s1), (a2, c2, s2): axis, cos and sin
// (cone_sine) of the half-angle.
__device__ __forceinline__ float cone_max_cos(float a1x, float a1y, float a1z, float c1, float s1, float a2x, float a2y,
                                              float a2z, float c2, float s2) {
    if (c1 <= -1.0f || c2 <= -1.0f) return 1.0f;
    float cb = rn_dot(a1x, a1y, a1z, a2x, a2y, a2z);
    cb = fminf(fmaxf(cb, -1.0f), 1.0f);
    const float cg = rn_sub(rn_mul(c1, c2), rn_mul(s1, s2));
    const float sg = rn_add(rn_mul(s1, c2), rn_mul(c1, s2));
    if (sg < 0.0f) return 1.0f;   // combined half-angles exceed pi
    if (cb >= cg) return 1.0f;    // axes closer than the combined half-angles
    const float sb = cone_sine(cb);  // (only needed past the early returns)
    return rn_add(rn_mul(cb, cg), rn_mul(sb, sg));
}

// min over members of two cones of cos(angle between them); -1 when they can point opposite.
__device__ __forceinline__ float cone_min_cos(float a1x, float a1y, float a1z, float c1, float s1, float a2x, float a2y,
                                              float a2z, float c2, float s2) {
    if (c1 <= -1.0f || c2 <= -1.0f) return -1.0f;
    float cb = rn_dot(a1x, a1y, a1z, a2x, a2y, a2z);
    cb = fminf(fmaxf(cb, -1.0f), 1.0f);
    const float cg = rn_sub(rn_mul(c1, c2), rn_mul(s1, s2));
    const float sg = rn_add(rn_mul(s1, c2), rn_mul(c1, s2));
    if (sg < 0.0f) return -1.0f;
    if (cg < -cb) return -1.0f;
    const float sb = cone_sine(cb);
    return rn_sub(rn_mul(cb, cg), rn_mul(sb, sg));
}

// Geometry quantities of (tile, inner node) used by the bound and by the learned features.
struct NodeGeom {
    float d2c;      // clamped squared box-to-box distance
    float cos1;     // receiver cosine bound in [0,1]
    float cos2;     // emitter cosine bound in [0,1]
    float ar_ok;    // 0: no antiradiance reaches the tile; 1: all pairs pass the cone test; else uncertain
    float dc;       // centre distance
    float rs;       // sum of the half-diagonals
    float rn;       // node half-diagonal
};

__device__ __forceinline__ NodeGeom node_geom(const TileInfo& t, float4 b0, float4 b1, float4 nc, float4 wc,
                                              const NodeExtra& ne, const BoundParams& bp) {
    NodeGeom g;
    const float bmin[3] = {b0.x, b0.y, b0.z}, bmax[3] = {b1.x, b1.y, b1.z};
    float d2 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float gap = fmaxf(0.0f, fmaxf(rn_sub(bmin[k], t.tmax[k]), rn_sub(t.tmin[k], bmax[k])));
        d2 = rn_add(d2, rn_mul(gap, gap));
    }
    g.d2c = fmaxf(d2, bp.clamp2);
    // direction cone node -> tile
    float v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float ct = rn_mul(0.5f, rn_add(t.tmin[k], t.tmax[k]));
        v[k] = rn_sub(ct, ne.cn[k]);
    }
    const float dc = rn_sqrt(rn_dot(v[0], v[1], v[2], v[0], v[1], v[2]));
    const float rn = ne.rn;
    const float rs = rn_add(rn, t.rt);
    g.dc = dc;
    g.rs = rs;
    g.rn = rn;
    // direction cone node -> tile: axis v / dc, sine rs / dc, cosine from the sine (ca = -1: the
    // boxes are too close for a cone)
    float ca = -1.0f, sa = 0.0f, ax = 0.0f, ay = 0.0f, az = 0.0f;
    if (dc > rs) {
        const float inv = rn_div(1.0f, dc);
        sa = rn_mul(rs, inv);
        ca = cone_sine(sa);
        ax = rn_mul(v[0], inv);
        ay = rn_mul(v[1], inv);
        az = rn_mul(v[2], inv);
    }
    const float sa2 = sa;
    const float c2 = cone_max_cos(nc.x, nc.y, nc.z, nc.w, ne.snc, ax, ay, az, ca, sa2);
    const float c1 = cone_max_cos(t.ncone.x, t.ncone.y, t.ncone.z, t.ncone.w, t.sn, -ax, -ay, -az, ca, sa2);
    g.cos2 = fminf(fmaxf(c2, 0.0f), 1.0f);
    g.cos1 = fminf(fmaxf(c1, 0.0f), 1.0f);
    g.ar_ok = 0.0f;
    if (bp.ar_kind == ARC_AR_CONE) {
        const float cw = cone_max_cos(wc.x, wc.y, wc.z, wc.w, ne.swc, ax, ay, az, ca, sa2);
        if (cw > bp.cos_thr && g.cos1 > bp.eps_cone) {
            // 1 when every (pixel, AVPL) pair of the two boxes passes the cone test, else the
            // uncertainty multiplier: the representative's test then stands for a mixed set
            const float cwmin = cone_min_cos(wc.x, wc.y, wc.z, wc.w, ne.swc, ax, ay, az, ca, sa2);
            const float c1min = cone_min_cos(t.ncone.x, t.ncone.y, t.ncone.z, t.ncone.w, t.sn, -ax, -ay, -az, ca, sa2);
            g.ar_ok = (cwmin > bp.cos_thr && c1min > bp.eps_cone) ? 1.0f : bp.ar_uncertain;
        }
    } else if (bp.ar_kind == ARC_AR_DISK) {
        g.ar_ok = 1.0f;
    }
    return g;
}

// Upper bound of the node's contribution (luminance) to any pixel of the tile.
__device__ __forceinline__ float node_bound(const TileInfo& t, const NodeGeom& g, float Ls, float As,
                                            const BoundParams& bp) {
    if (!(g.d2c > 0.0f)) return INFINITY;
    const float id2 = rn_div(1.0f, g.d2c);
    const float grad = rn_mul(rn_mul(g.cos1, g.cos2), id2);
    float m = rn_mul(Ls, grad);
    if (bp.ar_kind == ARC_AR_CONE) {
        m = rn_add(m, rn_mul(As, rn_mul(g.ar_ok, rn_mul(g.cos1, id2))));
    } else if (bp.ar_kind == ARC_AR_DISK) {
        m = rn_add(m, rn_mul(As, bp.disk_scale));
    }
    return rn_mul(t.kdl, m);
}

// Appends one warp's accepted nodes to its tile's chunked list in the cut pool.  Warp-uniform
// state; every lane of the warp calls append() with the same `mask`.
struct CutWriter {
    static constexpr int kChunk = 1024;
    CutPool pool;
    int32_t* table;
    int count = 0;
    int chunk_id = -1;  // pool chunk holding entry count - 1
    bool overflow = false;

    __device__ CutWriter(const CutPool& p, int tile) : pool(p), table(p.tables + (size_t)tile * p.max_chunks) {}

    __device__ __forceinline__ void append(unsigned mask, bool mine, int node, int lane) {
        const int n = __popc(mask);
        if (n == 0) return;
        const int first_new = count % kChunk == 0 ? count / kChunk : count / kChunk + 1;
        const int last = (count + n - 1) / kChunk;
        int new_id = -1;
        if (last >= first_new) {  // the batch starts a new chunk (at most one: n <= 32 < kChunk)
            if (lane == 0) {
                new_id = last < pool.max_chunks ? atomicAdd(pool.next, 1) : pool.num_chunks;
                if (new_id < pool.num_chunks) table[last] = new_id;
            }
            new_id = __shfl_sync(0xffffffffu, new_id, 0);
            if (new_id >= pool.num_chunks) overflow = true;
        }
        if (mine) {
            const int pos = count + __popc(mask & ((1u << lane) - 1u));
            const int id = pos / kChunk == last && last >= first_new ? new_id : chunk_id;
            if (id >= 0 && id < pool.num_chunks) pool.entries[(size_t)id * kChunk + pos % kChunk] = node;
        }
        if (last >= first_new) chunk_id = new_id;
        if (overflow) {
            count = min(count + n, last * kChunk);  // keep only entries that landed in a chunk
        } else {
            count += n;
        }
    }
};

}  // namespace arc

#endif  // ARC_CUT_BOUNDS_CUH_
