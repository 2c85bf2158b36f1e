// Cut gathers over the LBVH.
//
// ARC_CUT_SOLID_ANGLE: the lightcut of kernel_bvh (cudaGather.cu:316-444), one thread per pixel:
//   DFS from the root; a leaf adds its exact radiance; an inner node is skipped when both of its
//   box corners lie behind the receiver (cudaGather.cu:405-408), used whole when the solid angle
//   2 pi (1 - d / sqrt(r^2 + d^2)) of its bounding sphere seen from the representative is below
//   the threshold, and refined otherwise.  The stack holds 64 entries (the reference's 32
//   overflows for large trees); overflow paints the reference's magenta pixel and sets
//   ARC_DEVERR_STACK_OVERFLOW.  Antiradiance comes from the brute-force pass, as in the
//   reference's non-clustered run() path.
// ARC_CUT_ERROR_BOUND: one cut per 8x8 pixel tile, chosen by one warp that walks the tree
//   cooperatively (32 nodes per step, ballot/popc compaction of accepted nodes and of the
//   children to push).  A node is refined while an upper bound of its contribution to any pixel
//   of the tile exceeds eps times the tile's coarse radiance estimate.  Every pixel of the tile
//   then evaluates the same node list, so the evaluation is fully coherent.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>

#include "arc_internal.h"
#include "cut_bounds.cuh"
#include "device_common.cuh"
#include "pair_math.cuh"

namespace arc {

arc_status launch_antiradiance_only(arc_context* ctx, const GatherLaunch& g, double* ar64);
arc_status launch_cut_select_learned(arc_context* ctx, const arc_lbvh* bvh, const ArcGatherParams* gp,
                                     const ArcCutParams* cp, const float4* tiles_info, const float4* extra,
                                     int tiles_x, int tiles_y, const CutPool& pool);

namespace {

constexpr int kTile = 8;
constexpr int kSolidStack = 64;
constexpr int kChunkSize = 1024;  // cut entries per pool chunk
constexpr int kSelWarps = 4;
constexpr int kSelStack = 4096;
constexpr int kCoarseDepth = 5;

struct MatSmem {
    MaterialRecord m[ARC_MAX_MATERIALS];
};

// ---------------------------------------------------------------------------------------
// Solid-angle lightcut (reference semantics)
// ---------------------------------------------------------------------------------------
struct SolidArgs {
    const float4* gpos;
    const float4* gnrm;
    int64_t gpitch;
    int width, height;
    const MaterialRecord* mats;
    int num_mats;
    float3 cam;
    int n;
    const float4* bounds;
    ArcAvplBvhNodeDataParam nd;
    float thresh;
    float clamp2;
    double* rad64;
    float4* out_rad;
    int64_t opitch;
    int dbg_x, dbg_y;
    int32_t* used;
    uint32_t* err;
};

__device__ __forceinline__ float3 brdf_f(float3 w_i, float3 w_o, float3 n, const MaterialRecord& m) {
    float3 d = f3(kOneOverPi * m.diffuse_exp.x, kOneOverPi * m.diffuse_exp.y, kOneOverPi * m.diffuse_exp.z);
    if (m.specular_flag.w != 0.0f) {
        const float3 I = -1.0f * w_i;
        const float3 r = I - (2.0f * dot(n, I)) * n;
        const float c = fmaxf(0.0f, dot(r, w_o));
        const float e = m.diffuse_exp.w;
        const float f = 0.5f * kOneOverPi * (e + 2.0f) * powf(c, e);
        d = d + f * f3(m.specular_flag.x, m.specular_flag.y, m.specular_flag.z);
    }
    return d;
}

__device__ __forceinline__ float3 norm3(float3 v) { return rsqrtf(dot(v, v)) * v; }

// getRadiance (cudaGather.cu:78-95) for node-data element idx
__device__ __forceinline__ float3 node_radiance(const SolidArgs& a, const MatSmem& sm, float3 p, float3 n, int mat,
                                                float3 w_o, int idx) {
    const float3 pa = ld3(a.nd.position, idx), na = ld3(a.nd.normal, idx), wa = ld3(a.nd.incDirection, idx);
    const float3 L = ld3(a.nd.incRadiance, idx);
    int ma = a.nd.materialIndex[idx];
    if (ma < 0 || ma >= a.num_mats) ma = 0;
    const float3 v = pa - p;
    const float l2 = dot(v, v);
    if (!(l2 > 0.0f)) return f3(0, 0, 0);
    const float3 w = rsqrtf(l2) * v;
    float3 fl = f3(1, 1, 1);
    if (dot(wa, wa) != 0.0f) fl = brdf_f(-1.0f * wa, -1.0f * w, norm3(na), sm.m[ma]);
    const float3 fr = brdf_f(w, w_o, n, sm.m[mat]);
    const float c1 = fminf(fmaxf(dot(n, w), 0.0f), 1.0f);
    const float c2 = fminf(fmaxf(-dot(norm3(na), w), 0.0f), 1.0f);
    const float g = c1 * c2 / fmaxf(l2, a.clamp2);
    return f3(L.x * fl.x * fr.x * g, L.y * fl.y * fr.y * g, L.z * fl.z * fr.z * g);
}

__global__ void __launch_bounds__(256) cut_solid_angle_kernel(SolidArgs a) {
    __shared__ MatSmem sm;
    for (int i = threadIdx.x; i < a.num_mats; i += blockDim.x) sm.m[i] = a.mats[i];
    __syncthreads();
    const int x = blockIdx.x * 16 + threadIdx.x % 16;
    const int y = blockIdx.y * 16 + threadIdx.x / 16;
    if (x >= a.width || y >= a.height) return;
    const float4 gp = a.gpos[(int64_t)y * a.gpitch + x];
    const float4 gn = a.gnrm[(int64_t)y * a.gpitch + x];
    const int mat = (int)gn.w;
    const int64_t o = (int64_t)y * a.opitch + x;
    float s[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    bool error = false;
    if (mat != 0 && !(mat > 0 && mat < a.num_mats)) set_error(a.err, ARC_DEVERR_BAD_MATERIAL);
    if (mat > 0 && mat < a.num_mats) {
        const float3 p = f3(gp.x, gp.y, gp.z);
        const float3 nraw = f3(gn.x, gn.y, gn.z);
        const float3 n = norm3(nraw);
        const float3 w_o = norm3(a.cam - p);
        const bool dbg = a.used && x == a.dbg_x && y == a.dbg_y;
        int stack[kSolidStack];
        stack[0] = -1;
        int sp = 1;
        const float two_pi = rn_mul(2.0f, kPi);
        // every node is visited at most once in a valid tree: 2n - 1 pops bound the walk
        int budget = 2 * a.n;
        while (sp > 0) {
            if (--budget < 0) {
                error = true;
                set_error(a.err, ARC_DEVERR_BAD_NODE);
                break;
            }
            const int node = stack[--sp];
            if (node >= a.n) {
                error = true;
                set_error(a.err, ARC_DEVERR_BAD_NODE);
                break;
            }
            int idx;
            if (node >= 0) {
                idx = node;
            } else {
                const int k = -(node + 1);
                if (k >= a.n - 1) {
                    error = true;
                    set_error(a.err, ARC_DEVERR_BAD_NODE);
                    break;
                }
                const float4 b0 = a.bounds[4 * (size_t)k], b1 = a.bounds[4 * (size_t)k + 1];
                // visibility of the box corners (cudaGather.cu:405-408); the sign of
                // n.normalize(v) is the sign of n.v
                const bool vis = rn_dot(nraw.x, nraw.y, nraw.z, rn_sub(b1.x, p.x), rn_sub(b1.y, p.y), rn_sub(b1.z, p.z)) >
                                     0.0f ||
                                 rn_dot(nraw.x, nraw.y, nraw.z, rn_sub(b0.x, p.x), rn_sub(b0.y, p.y), rn_sub(b0.z, p.z)) >
                                     0.0f;
                if (!vis) continue;
                idx = a.n + k;
                const float3 pr = ld3(a.nd.position, idx);
                const float ex = rn_sub(b1.x, b0.x), ey = rn_sub(b1.y, b0.y), ez = rn_sub(b1.z, b0.z);
                const float radius = rn_mul(0.5f, rn_sqrt(rn_dot(ex, ey, ez, ex, ey, ez)));
                const float vx = rn_sub(pr.x, p.x), vy = rn_sub(pr.y, p.y), vz = rn_sub(pr.z, p.z);
                const float dist = rn_sqrt(rn_dot(vx, vy, vz, vx, vy, vz));
                const float solid = rn_mul(
                    two_pi,
                    rn_sub(1.0f, rn_div(dist, rn_sqrt(rn_add(rn_mul(radius, radius), rn_mul(dist, dist))))));
                if (!(solid < a.thresh)) {
                    if (sp + 2 > kSolidStack) {
                        error = true;
                        set_error(a.err, ARC_DEVERR_STACK_OVERFLOW);
                        break;
                    }
                    stack[sp++] = __float_as_int(b0.w);
                    stack[sp++] = __float_as_int(b1.w);
                    continue;
                }
            }
            const float3 t = node_radiance(a, sm, p, n, mat, w_o, idx);
            kahan_add(s[0], c[0], t.x);
            kahan_add(s[1], c[1], t.y);
            kahan_add(s[2], c[2], t.z);
            if (dbg) a.used[idx] = 1;
        }
    }
    double r[3];
    for (int q = 0; q < 3; ++q) r[q] = (double)s[q] - (double)c[q];
    if (error) {
        r[0] = 100000.0;
        r[1] = 0.0;
        r[2] = 100000.0;
    }
    a.rad64[3 * o + 0] = r[0];
    a.rad64[3 * o + 1] = r[1];
    a.rad64[3 * o + 2] = r[2];
    if (a.out_rad) a.out_rad[o] = make_float4((float)r[0], (float)r[1], (float)r[2], 1.0f);
}

// ---------------------------------------------------------------------------------------
// Tile set-up: bounds of the tile, receiver normal cone, max receiver albedo, coarse estimate
// ---------------------------------------------------------------------------------------
struct TileArgs {
    const float4* gpos;
    const float4* gnrm;
    int64_t gpitch;
    int width, height;
    const MaterialRecord* mats;
    int num_mats;
    int n;
    const float4* bounds;
    const float4* records;
    float eps_bound;
    float clamp2;
    int tiles_x, tiles_y;
    float4* info;  // [tiles][4]
    uint32_t* err;
};

__device__ __forceinline__ float coarse_g(float px, float py, float pz, float nx, float ny, float nz, const float4 q0,
                                          const float4 q1, float clamp2) {
    const float dx = rn_sub(q0.x, px), dy = rn_sub(q0.y, py), dz = rn_sub(q0.z, pz);
    const float l2 = rn_dot(dx, dy, dz, dx, dy, dz);
    if (!(l2 > 0.0f)) return 0.0f;
    const float r = rn_div(1.0f, rn_sqrt(l2));
    const float c1 = fmaxf(0.0f, rn_mul(rn_dot(nx, ny, nz, dx, dy, dz), r));
    const float c2 = fmaxf(0.0f, rn_mul(-rn_dot(q0.w, q1.x, q1.y, dx, dy, dz), r));
    return rn_div(rn_mul(c1, c2), fmaxf(l2, clamp2));
}

__global__ void __launch_bounds__(32 * kSelWarps) cut_tile_setup(TileArgs a) {
    __shared__ float sp[kSelWarps][64][7];  // p.xyz, n.xyz, valid
    __shared__ float skd[kSelWarps][64][3];
    __shared__ float sest[kSelWarps][64];
    __shared__ int scoarse[kSelWarps][1 << kCoarseDepth];
    __shared__ int sncoarse[kSelWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kSelWarps + warp;
    if (tile >= a.tiles_x * a.tiles_y) return;
    const int tx0 = (tile % a.tiles_x) * kTile, ty0 = (tile / a.tiles_x) * kTile;
    float tmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, tmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float kdl = 0.0f;
    int nvalid = 0;
    for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        const int x = tx0 + i % kTile, y = ty0 + i / kTile;
        float4 gp = make_float4(0, 0, 0, 0), gn = make_float4(0, 0, 0, 0);
        bool v = x < a.width && y < a.height;
        if (v) {
            gp = a.gpos[(int64_t)y * a.gpitch + x];
            gn = a.gnrm[(int64_t)y * a.gpitch + x];
            const int m = (int)gn.w;
            v = m > 0 && m < a.num_mats;
            if (!v && m != 0) set_error(a.err, ARC_DEVERR_BAD_MATERIAL);  // gathers 0, as brute force does
            if (v) {
                const float4 d = a.mats[m].diffuse_exp;
                skd[warp][i][0] = rn_mul(kOneOverPi, d.x);
                skd[warp][i][1] = rn_mul(kOneOverPi, d.y);
                skd[warp][i][2] = rn_mul(kOneOverPi, d.z);
                kdl = fmaxf(kdl, lum3(skd[warp][i][0], skd[warp][i][1], skd[warp][i][2]));
                tmin[0] = fminf(tmin[0], gp.x); tmin[1] = fminf(tmin[1], gp.y); tmin[2] = fminf(tmin[2], gp.z);
                tmax[0] = fmaxf(tmax[0], gp.x); tmax[1] = fmaxf(tmax[1], gp.y); tmax[2] = fmaxf(tmax[2], gp.z);
                nvalid += 1;
            }
        }
        sp[warp][i][0] = gp.x; sp[warp][i][1] = gp.y; sp[warp][i][2] = gp.z;
        sp[warp][i][3] = gn.x; sp[warp][i][4] = gn.y; sp[warp][i][5] = gn.z;
        sp[warp][i][6] = v ? 1.0f : 0.0f;
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int k = 0; k < 3; ++k) {
            tmin[k] = fminf(tmin[k], __shfl_xor_sync(0xffffffffu, tmin[k], o));
            tmax[k] = fmaxf(tmax[k], __shfl_xor_sync(0xffffffffu, tmax[k], o));
        }
        kdl = fmaxf(kdl, __shfl_xor_sync(0xffffffffu, kdl, o));
        nvalid += __shfl_xor_sync(0xffffffffu, nvalid, o);
    }
    // coarse cut: the nodes at depth kCoarseDepth (or leaves above it), left-first DFS order
    if (lane == 0) {
        int st[2 * kCoarseDepth + 2][2];
        int top = 0, cnt = 0;
        st[top][0] = a.n;  // root inner node 0 in node-record index space
        st[top][1] = 0;
        ++top;
        while (top > 0) {
            --top;
            const int node = st[top][0], depth = st[top][1];
            if (node < a.n || depth == kCoarseDepth) {
                scoarse[warp][cnt++] = node;
                continue;
            }
            const int k = node - a.n;
            const float4 b0 = a.bounds[4 * (size_t)k], b1 = a.bounds[4 * (size_t)k + 1];
            const int lc = __float_as_int(b0.w), rc = __float_as_int(b1.w);
            st[top][0] = rc >= 0 ? rc : a.n - (rc + 1);
            st[top][1] = depth + 1;
            ++top;
            st[top][0] = lc >= 0 ? lc : a.n - (lc + 1);
            st[top][1] = depth + 1;
            ++top;
        }
        sncoarse[warp] = cnt;
    }
    __syncwarp();
    const int ncoarse = sncoarse[warp];
    for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        float est = 0.0f;
        if (sp[warp][i][6] != 0.0f) {
            for (int j = 0; j < ncoarse; ++j) {
                const int node = scoarse[warp][j];
                const float4 q0 = a.records[4 * (size_t)node], q1 = a.records[4 * (size_t)node + 1];
                const float4 q2 = a.records[4 * (size_t)node + 2];
                const float g = coarse_g(sp[warp][i][0], sp[warp][i][1], sp[warp][i][2], sp[warp][i][3], sp[warp][i][4],
                                         sp[warp][i][5], q0, q1, a.clamp2);
                const float l = lum3(rn_mul(skd[warp][i][0], q2.y), rn_mul(skd[warp][i][1], q2.z),
                                     rn_mul(skd[warp][i][2], q2.w));
                est = rn_add(est, rn_mul(l, g));
            }
        }
        sest[warp][i] = est;
    }
    __syncwarp();
    if (lane == 0) {
        float sum = 0.0f;
        float4 cone = make_float4(0, 0, 0, -2.0f);  // -2: empty
        for (int i = 0; i < 64; ++i) {
            if (sp[warp][i][6] == 0.0f) continue;
            sum = rn_add(sum, sest[warp][i]);
            const float4 ci = make_float4(sp[warp][i][3], sp[warp][i][4], sp[warp][i][5], 1.0f);
            if (cone.w < -1.5f) {
                cone = ci;
            } else {
                // cone union (same as the bottom-up build)
                if (cone.w <= -1.0f) continue;
                const float sx = rn_add(cone.x, ci.x), sy = rn_add(cone.y, ci.y), sz = rn_add(cone.z, ci.z);
                const float l2 = rn_dot(sx, sy, sz, sx, sy, sz);
                if (!(l2 > 1e-12f)) {
                    cone = make_float4(0, 0, 0, -1.0f);
                    continue;
                }
                const float inv = rn_div(1.0f, rn_sqrt(l2));
                const float ax = rn_mul(sx, inv), ay = rn_mul(sy, inv), az = rn_mul(sz, inv);
                float res = 1.0f;
                const float4 cc[2] = {cone, ci};
                for (int q = 0; q < 2; ++q) {
                    float d = rn_dot(ax, ay, az, cc[q].x, cc[q].y, cc[q].z);
                    d = fminf(fmaxf(d, -1.0f), 1.0f);
                    const float sd = rn_sqrt(fmaxf(0.0f, rn_sub(1.0f, rn_mul(d, d))));
                    const float si = rn_sqrt(fmaxf(0.0f, rn_sub(1.0f, rn_mul(cc[q].w, cc[q].w))));
                    const float v = cc[q].w < -d ? -1.0f : rn_sub(rn_mul(d, cc[q].w), rn_mul(sd, si));
                    res = fminf(res, v);
                }
                cone = make_float4(ax, ay, az, res);
            }
        }
        if (cone.w < -1.5f) cone = make_float4(0, 0, 0, -1.0f);
        const float mean = nvalid > 0 ? rn_div(sum, (float)nvalid) : 0.0f;
        float4* info = a.info + 4 * (size_t)tile;
        info[0] = make_float4(tmin[0], tmin[1], tmin[2], kdl);
        info[1] = make_float4(tmax[0], tmax[1], tmax[2], rn_mul(a.eps_bound, mean));
        info[2] = cone;
        info[3] = make_float4(__int_as_float(nvalid), mean,
                              half_diagonal(rn_sub(tmax[0], tmin[0]), rn_sub(tmax[1], tmin[1]), rn_sub(tmax[2], tmin[2])),
                              cone_sine(cone.w));
    }
}

// NodeExtra of every inner node k (bounds at 4 k, record at 4 (n + k)), for node_geom / node_bound
__global__ void cut_node_extra(int n, const float4* bounds, const float4* records, float4* ext) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n - 1) return;
    const float4 b0 = bounds[4 * (size_t)k], b1 = bounds[4 * (size_t)k + 1];
    const float4 nc = bounds[4 * (size_t)k + 2], wc = bounds[4 * (size_t)k + 3];
    const float4 q2 = records[4 * ((size_t)n + k) + 2], q3 = records[4 * ((size_t)n + k) + 3];
    const float rn = half_diagonal(rn_sub(b1.x, b0.x), rn_sub(b1.y, b0.y), rn_sub(b1.z, b0.z));
    ext[2 * (size_t)k] = make_float4(rn, cone_sine(nc.w), cone_sine(wc.w), lum3(q2.y, q2.z, q2.w));
    ext[2 * (size_t)k + 1] = make_float4(lum3(q3.x, q3.y, q3.z), rn_mul(0.5f, rn_add(b0.x, b1.x)),
                                         rn_mul(0.5f, rn_add(b0.y, b1.y)), rn_mul(0.5f, rn_add(b0.z, b1.z)));
}

__device__ __forceinline__ TileInfo load_tile(const float4* info, int tile) {
    const float4 i0 = info[4 * (size_t)tile], i1 = info[4 * (size_t)tile + 1], i2 = info[4 * (size_t)tile + 2],
                 i3 = info[4 * (size_t)tile + 3];
    TileInfo t;
    t.tmin[0] = i0.x; t.tmin[1] = i0.y; t.tmin[2] = i0.z; t.kdl = i0.w;
    t.tmax[0] = i1.x; t.tmax[1] = i1.y; t.tmax[2] = i1.z; t.tau = i1.w;
    t.ncone = i2;
    t.valid = __float_as_int(i3.x);
    t.rt = i3.z;
    t.sn = i3.w;
    return t;
}

// ---------------------------------------------------------------------------------------
// Error-bound cut selection: one warp per tile
// ---------------------------------------------------------------------------------------
struct SelArgs {
    int n;
    const float4* bounds;
    const float4* records;
    const float4* info;
    const float4* extra;  // NodeExtra per inner node
    BoundParams bp;
    int tiles;
    CutPool pool;
    uint32_t* err;
};

__global__ void __launch_bounds__(32 * kSelWarps) cut_select_bound(SelArgs a) {
    extern __shared__ int sstack[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kSelWarps + warp;
    if (tile >= a.tiles) return;
    int* stack = sstack + warp * kSelStack;
    const TileInfo t = load_tile(a.info, tile);
    CutWriter cw(a.pool, tile);
    if (t.valid == 0) {
        if (lane == 0) a.pool.counts[tile] = 0;
        return;
    }
    const unsigned lt = (1u << lane) - 1u;
    int sp = 1;
    if (lane == 0) stack[0] = a.n;  // root
    __syncwarp();
    bool overflow = false;
    int budget = 2 * a.n;  // node visits of a valid tree
    while (sp > 0) {
        if (budget <= 0) {
            if (lane == 0) set_error(a.err, ARC_DEVERR_BAD_NODE);
            break;
        }
        const int m = min(32, sp);
        budget -= m;
        int node = -1;
        if (lane < m) node = stack[sp - 1 - lane];
        __syncwarp();
        sp -= m;
        bool accept = false, refine = false;
        int lc = 0, rc = 0;
        if (lane < m) {
            if (node < a.n) {
                accept = node >= 0;
            } else {
                const int k = node - a.n;
                const float4 b0 = a.bounds[4 * (size_t)k], b1 = a.bounds[4 * (size_t)k + 1];
                const float4 nc = a.bounds[4 * (size_t)k + 2], wc = a.bounds[4 * (size_t)k + 3];
                const NodeExtra ne = load_node_extra(a.extra, k);
                const NodeGeom g = node_geom(t, b0, b1, nc, wc, ne, a.bp);
                const float M = node_bound(t, g, ne.Ls, ne.As, a.bp);
                if (M > t.tau) {
                    refine = true;
                    const int l = __float_as_int(b0.w), r = __float_as_int(b1.w);
                    lc = l >= 0 ? l : a.n - (l + 1);
                    rc = r >= 0 ? r : a.n - (r + 1);
                } else {
                    accept = true;
                }
            }
        }
        unsigned rmask = __ballot_sync(0xffffffffu, refine);
        const int nref = __popc(rmask);
        if (sp + 2 * nref > kSelStack) {  // no room: use the nodes whole
            if (refine) {
                refine = false;
                accept = true;
            }
            rmask = 0;
            overflow = true;
        }
        const unsigned amask = __ballot_sync(0xffffffffu, accept);
        cw.append(amask, accept, node, lane);
        if (refine) {
            const int q = sp + 2 * __popc(rmask & lt);
            stack[q] = rc;
            stack[q + 1] = lc;
        }
        sp += 2 * __popc(rmask);
        __syncwarp();
    }
    if (lane == 0) {
        if (cw.overflow || overflow) set_error(a.err, ARC_DEVERR_CUT_OVERFLOW);
        a.pool.counts[tile] = cw.count;
    }
}

// ---------------------------------------------------------------------------------------
// Cut evaluation: one 64-thread block per tile, one pixel per thread
// ---------------------------------------------------------------------------------------
struct EvalArgs {
    const float4* gpos;
    const float4* gnrm;
    int64_t gpitch;
    int width, height;
    const MaterialRecord* mats;
    int num_mats;
    const float4* records;
    int tiles_x;
    CutPool pool;
    PairConsts pc;
    float disk_scale;
    float4* out_res;
    float4* out_rad;
    float4* out_ar;
    double* out_res64;
    int64_t opitch;
    const int* order;  // block b evaluates tile order[b]
};

// Tiles in decreasing order of cut size (buckets of floor(log2(count)), empty tiles last), so that
// the blocks with the longest cuts start first and the short ones fill the tail of the launch.
// One block; the order within a bucket is arbitrary (each tile's result does not depend on it).
__global__ void __launch_bounds__(1024) tile_order_kernel(const int32_t* counts, int tiles, int* order) {
    __shared__ int hist[33], off[33];
    const int t = threadIdx.x;
    if (t < 33) hist[t] = 0;
    __syncthreads();
    for (int i = t; i < tiles; i += blockDim.x) {
        const int c = counts[i];
        atomicAdd(&hist[c > 0 ? 32 - __clz(c) : 0], 1);
    }
    __syncthreads();
    if (t == 0) {
        int s = 0;
        for (int b = 32; b >= 0; --b) {
            off[b] = s;
            s += hist[b];
        }
    }
    __syncthreads();
    for (int i = t; i < tiles; i += blockDim.x) {
        const int c = counts[i];
        order[atomicAdd(&off[c > 0 ? 32 - __clz(c) : 0], 1)] = i;
    }
}

template <int AR>
__global__ void __launch_bounds__(64) cut_eval_kernel(EvalArgs a) {
    constexpr int kChunk = 256;
    __shared__ float4 srec[kChunk * 4];
    const int tile = a.order[blockIdx.x];
    const int i = threadIdx.x;
    const int x = (tile % a.tiles_x) * kTile + i % kTile, y = (tile / a.tiles_x) * kTile + i / kTile;
    bool valid = x < a.width && y < a.height;
    float4 gp = make_float4(0, 0, 0, 0), gn = make_float4(0, 0, 0, 0);
    int mat = 0;
    if (valid) {
        gp = a.gpos[(int64_t)y * a.gpitch + x];
        gn = a.gnrm[(int64_t)y * a.gpitch + x];
        mat = (int)gn.w;
        valid = mat > 0 && mat < a.num_mats;
    }
    Pixel<float> px;
    px.px = gp.x;
    px.py = gp.y;
    px.pz = gp.z;
    if (valid) {
        const float l = rsqrtf(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z);
        px.nx = gn.x * l;
        px.ny = gn.y * l;
        px.nz = gn.z * l;
    } else {
        px.nx = px.ny = px.nz = 0.0f;
    }
    px.r0 = px.r1 = px.r2 = px.a0 = px.a1 = px.a2 = 0.0f;
    float ss[6] = {0, 0, 0, 0, 0, 0}, sc[6] = {0, 0, 0, 0, 0, 0};
    const int count = a.pool.counts[tile];
    for (int base = 0; base < count; base += kChunk) {
        const int cnt = min(kChunk, count - base);
        // kChunk divides kChunkSize: a sub-chunk never straddles two pool chunks
        const int32_t* nodes = a.pool.entries + (size_t)a.pool.tables[(size_t)tile * a.pool.max_chunks + base / kChunkSize] *
                                                    kChunkSize + base % kChunkSize;
        __syncthreads();
        for (int j = i; j < cnt * 4; j += 64) {
            const int node = nodes[j / 4];
            float4 q = a.records[4 * (size_t)node + (j & 3)];
            if (AR == ARC_AR_DISK && (j & 3) == 3) {
                const float4 q1 = a.records[4 * (size_t)node + 1], q2 = a.records[4 * (size_t)node + 2];
                const float ww = q1.z * q1.z + q1.w * q1.w + q2.x * q2.x;
                q.w = ww > 0.0f ? rsqrtf(ww) : 0.0f;
            }
            srec[j] = q;
        }
        __syncthreads();
        for (int j = 0; j < cnt; ++j) {
            float g, ga;
            const float4* q = srec + 4 * j;
            pair_terms<AR, float>(q[0], q[1], q[2], q[3], px, a.pc, g, ga);
            px.r0 += q[2].y * g;
            px.r1 += q[2].z * g;
            px.r2 += q[2].w * g;
            px.a0 += q[3].x * ga;
            px.a1 += q[3].y * ga;
            px.a2 += q[3].z * ga;
        }
        kahan_add(ss[0], sc[0], px.r0);
        kahan_add(ss[1], sc[1], px.r1);
        kahan_add(ss[2], sc[2], px.r2);
        kahan_add(ss[3], sc[3], px.a0);
        kahan_add(ss[4], sc[4], px.a1);
        kahan_add(ss[5], sc[5], px.a2);
        px.r0 = px.r1 = px.r2 = px.a0 = px.a1 = px.a2 = 0.0f;
    }
    if (x >= a.width || y >= a.height) return;
    double rad[3] = {0, 0, 0}, ar[3] = {0, 0, 0};
    if (valid) {
        const float4 d = a.mats[mat].diffuse_exp;
        const double kd[3] = {(double)(kOneOverPi * d.x), (double)(kOneOverPi * d.y), (double)(kOneOverPi * d.z)};
        const double as = AR == ARC_AR_DISK ? (double)a.disk_scale : 1.0;
        for (int c = 0; c < 3; ++c) {
            rad[c] = kd[c] * ((double)ss[c] - (double)sc[c]);
            ar[c] = kd[c] * as * ((double)ss[3 + c] - (double)sc[3 + c]);
        }
    }
    const int64_t o = (int64_t)y * a.opitch + x;
    const double res[3] = {rad[0] - ar[0], rad[1] - ar[1], rad[2] - ar[2]};
    if (a.out_res) a.out_res[o] = make_float4((float)res[0], (float)res[1], (float)res[2], 1.0f);
    if (a.out_rad) a.out_rad[o] = make_float4((float)rad[0], (float)rad[1], (float)rad[2], 1.0f);
    if (a.out_ar) a.out_ar[o] = make_float4((float)ar[0], (float)ar[1], (float)ar[2], 1.0f);
    if (a.out_res64) {
        a.out_res64[3 * o + 0] = res[0];
        a.out_res64[3 * o + 1] = res[1];
        a.out_res64[3 * o + 2] = res[2];
    }
}

// Cut evaluation with packed FP32 pairs (no or cone antiradiance): each thread (one pixel) takes
// two cut nodes per step with f32x2 arithmetic.  The records are staged 128 nodes at a time,
// interleaved by node pair: float pair * 32 + 2 f + h holds field f (0..15 of the packed record)
// of node 2 pair + h, so one 16-byte shared load brings two fields of both nodes.  Staging is
// asynchronous and double-buffered: a warp copies a whole pair block per instruction, lane t
// moving float t (field t / 2 of node 2 pair + t % 2) with a 4-byte cp.async -- the 32 lanes read
// the two 64-byte records (4 sectors) and write 32 consecutive banks.  The node ids of each stage
// arrive in shared memory one stage ahead with the copies before it, so the copies of stage s + 1
// are issued from shared memory and fly while stage s is evaluated.  An odd count is padded with
// a zero record, which contributes exactly 0.  Same terms as pair_terms; the even and odd nodes'
// partial sums are added before each stage's Kahan step.
template <int AR>
__global__ void __launch_bounds__(64) cut_eval_packed_kernel(EvalArgs a) {
    constexpr int kSub = 128;  // nodes per stage; divides kChunkSize, so a stage never straddles two pool chunks
    __shared__ __align__(16) float srec[2][kSub * 16];
    __shared__ int32_t sids[2][kSub];
    const int tile = a.order[blockIdx.x];
    const int i = threadIdx.x, lane = i & 31, warp = i >> 5;
    const int x = (tile % a.tiles_x) * kTile + i % kTile, y = (tile / a.tiles_x) * kTile + i / kTile;
    const int count = a.pool.counts[tile];
    const int nsub = (count + kSub - 1) / kSub;
    const int32_t* table = a.pool.tables + (size_t)tile * a.pool.max_chunks;
    const float* recf = reinterpret_cast<const float*>(a.records);
    // node ids of stage s into sids[s & 1]: two per thread
    auto copy_ids = [&](int s) {
        const int base = s * kSub;
        const int cnt = min(kSub, count - base);
        const int32_t* nodes = a.pool.entries + (size_t)table[base / kChunkSize] * kChunkSize + base % kChunkSize;
        if (i < cnt) cp_async4(&sids[s & 1][i], nodes + i);
        if (i + 64 < cnt) cp_async4(&sids[s & 1][i + 64], nodes + i + 64);
    };
    // records of stage s (ids already in sids[s & 1]) into srec[s & 1]: warp w copies pairs
    // w, w + 2, ...; the pad half of an odd count's last pair gets a zero
    auto copy_records = [&](int s) {
        const int cnt = min(kSub, count - s * kSub);
        const int pairs = (cnt + 1) >> 1;
        float* buf = srec[s & 1];
        const int h = lane & 1, f = lane >> 1;
        for (int pr = warp; pr < pairs; pr += 2) {
            const int nl = 2 * pr + h;
            if (nl < cnt)
                cp_async4(buf + pr * 32 + lane, recf + 16 * (size_t)sids[s & 1][nl] + f);
            else
                buf[pr * 32 + lane] = 0.0f;
        }
    };
    if (nsub > 0) {
        copy_ids(0);
        cp_async_commit();
        if (nsub > 1) copy_ids(1);
        cp_async_commit();
        cp_async_wait<1>();  // this thread's ids of stage 0
        __syncthreads();     // everyone's
        copy_records(0);
        cp_async_commit();
    }

    bool valid = x < a.width && y < a.height;
    float4 gp = make_float4(0, 0, 0, 0), gn = make_float4(0, 0, 0, 0);
    int mat = 0;
    if (valid) {
        gp = a.gpos[(int64_t)y * a.gpitch + x];
        gn = a.gnrm[(int64_t)y * a.gpitch + x];
        mat = (int)gn.w;
        valid = mat > 0 && mat < a.num_mats;
    }
    float nx = 0.0f, ny = 0.0f, nz = 0.0f;
    if (valid) {
        const float l = rsqrtf(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z);
        nx = gn.x * l;
        ny = gn.y * l;
        nz = gn.z * l;
    }
    const uint64_t PX = f2(-gp.x, -gp.x), PY = f2(-gp.y, -gp.y), PZ = f2(-gp.z, -gp.z);
    const uint64_t NX = f2(nx, nx), NY = f2(ny, ny), NZ = f2(nz, nz);
    const float cos_thr = a.pc.cos_thr, eps = a.pc.eps, inv_clamp2 = a.pc.inv_clamp2;
    // distance floor folded into the FMA chain: l2 + 1e-30 equals max(l2, 1e-30) for l2 above ~1e-23
    const uint64_t kTiny2 = f2(1e-30f, 1e-30f);
    float ss[6] = {0, 0, 0, 0, 0, 0}, sc[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < nsub; ++s) {
        // stage s's records and stage s + 1's ids have landed for every thread, and every thread
        // is done with stage s - 1, whose buffers the next copies overwrite
        cp_async_wait<0>();
        __syncthreads();
        if (s + 1 < nsub) copy_records(s + 1);
        if (s + 2 < nsub) copy_ids(s + 2);
        cp_async_commit();
        const int cnt = min(kSub, count - s * kSub);
        const int pairs = (cnt + 1) >> 1;
        const float* srs = srec[s & 1];
        uint64_t R0 = 0, R1 = 0, R2 = 0, A0 = 0, A1 = 0, A2 = 0;  // packed zeros
#pragma unroll 2
        for (int pr = 0; pr < pairs; ++pr) {
            const ulonglong2* s2 = reinterpret_cast<const ulonglong2*>(srs + pr * 32);
            const ulonglong2 f01 = s2[0], f23 = s2[1], f45 = s2[2], f67 = s2[3], f89 = s2[4], f1011 = s2[5];
            const uint64_t dx = f2_add(f01.x, PX), dy = f2_add(f01.y, PY), dz = f2_add(f23.x, PZ);
            const uint64_t l2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_fma(dx, dx, kTiny2)));  // >= 1e-30
            float l2a, l2b;
            f2_split(l2, l2a, l2b);
            const uint64_t r = f2(rsqrtf(l2a), rsqrtf(l2b));
            const uint64_t c1 = f2_mul(f2_fma(NZ, dz, f2_fma(NY, dy, f2_mul(NX, dx))), r);
            const uint64_t c2n = f2_mul(f2_fma(f45.y, dz, f2_fma(f45.x, dy, f2_mul(f23.y, dx))), r);  // -c2
            float c1a, c1b, c2a, c2b, rra, rrb, ia, ib;
            f2_split(c1, c1a, c1b);
            f2_split(c2n, c2a, c2b);
            f2_split(f2_mul(r, r), rra, rrb);
            const uint64_t inv = f2(fminf(rra, inv_clamp2), fminf(rrb, inv_clamp2));
            // c1 / max(d^2, clamp^2): the radiance term's receiver factor and the cone term itself
            f2_split(f2_mul(c1, inv), ia, ib);
            const uint64_t g = f2_mul(f2(fmaxf(ia, 0.0f), fmaxf(ib, 0.0f)), f2(fmaxf(-c2a, 0.0f), fmaxf(-c2b, 0.0f)));
            R0 = f2_fma(f89.y, g, R0);
            R1 = f2_fma(f1011.x, g, R1);
            R2 = f2_fma(f1011.y, g, R2);
            if (AR == ARC_AR_CONE) {
                const ulonglong2 f1213 = s2[6], f1415 = s2[7];
                const uint64_t wdr = f2_mul(f2_fma(f89.x, dz, f2_fma(f67.y, dy, f2_mul(f67.x, dx))), r);  // -cw
                float wa, wb;
                f2_split(wdr, wa, wb);
                const uint64_t ga = f2((-wa > cos_thr && c1a > eps) ? ia : 0.0f, (-wb > cos_thr && c1b > eps) ? ib : 0.0f);
                A0 = f2_fma(f1213.x, ga, A0);
                A1 = f2_fma(f1213.y, ga, A1);
                A2 = f2_fma(f1415.x, ga, A2);
            }
        }
        const uint64_t acc[6] = {R0, R1, R2, A0, A1, A2};
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            float lo, hi;
            f2_split(acc[c], lo, hi);
            kahan_add(ss[c], sc[c], lo + hi);
        }
    }
    if (x >= a.width || y >= a.height) return;
    double rad[3] = {0, 0, 0}, ar[3] = {0, 0, 0};
    if (valid) {
        const float4 d = a.mats[mat].diffuse_exp;
        const double kd[3] = {(double)(kOneOverPi * d.x), (double)(kOneOverPi * d.y), (double)(kOneOverPi * d.z)};
        for (int c = 0; c < 3; ++c) {
            rad[c] = kd[c] * ((double)ss[c] - (double)sc[c]);
            ar[c] = kd[c] * ((double)ss[3 + c] - (double)sc[3 + c]);
        }
    }
    const int64_t o = (int64_t)y * a.opitch + x;
    const double res[3] = {rad[0] - ar[0], rad[1] - ar[1], rad[2] - ar[2]};
    if (a.out_res) a.out_res[o] = make_float4((float)res[0], (float)res[1], (float)res[2], 1.0f);
    if (a.out_rad) a.out_rad[o] = make_float4((float)rad[0], (float)rad[1], (float)rad[2], 1.0f);
    if (a.out_ar) a.out_ar[o] = make_float4((float)ar[0], (float)ar[1], (float)ar[2], 1.0f);
    if (a.out_res64) {
        a.out_res64[3 * o + 0] = res[0];
        a.out_res64[3 * o + 1] = res[1];
        a.out_res64[3 * o + 2] = res[2];
    }
}

// result = radiance - antiradiance in FP64 (kernel_combine, cudaGather.cu:782-803)
__global__ void combine_kernel(const double* rad64, const double* ar64, int width, int height, float4* out_res,
                               float4* out_ar, double* out_res64, int64_t opitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    const int64_t o = (int64_t)y * opitch + x;
    double r[3];
    for (int c = 0; c < 3; ++c) r[c] = rad64[3 * o + c] - (ar64 ? ar64[3 * o + c] : 0.0);
    if (out_res) out_res[o] = make_float4((float)r[0], (float)r[1], (float)r[2], 1.0f);
    if (out_ar) {
        if (ar64)
            out_ar[o] = make_float4((float)ar64[3 * o], (float)ar64[3 * o + 1], (float)ar64[3 * o + 2], 1.0f);
        else
            out_ar[o] = make_float4(0, 0, 0, 1.0f);
    }
    if (out_res64)
        for (int c = 0; c < 3; ++c) out_res64[3 * o + c] = r[c];
}

}  // namespace

arc_status launch_tile_setup(arc_context* ctx, const arc_lbvh* bvh, const ArcGBufferView* gb, const ArcGatherParams* gp,
                             const ArcCutParams* cp, float4** info_out, float4** extra_out) {
    const int W = gb->width, H = gb->height;
    const int tiles_x = (W + kTile - 1) / kTile, tiles_y = (H + kTile - 1) / kTile, tiles = tiles_x * tiles_y;
    float4* info = nullptr;
    ARC_TRY(ctx->arena.get("tile_info", (size_t)tiles * 4 * sizeof(float4), reinterpret_cast<void**>(&info)));
    TileArgs ta;
    ta.gpos = reinterpret_cast<const float4*>(gb->position);
    ta.gnrm = reinterpret_cast<const float4*>(gb->normal);
    ta.gpitch = gb->pitch;
    ta.width = W;
    ta.height = H;
    ta.mats = ctx->d_materials;
    ta.num_mats = ctx->num_materials;
    ta.n = bvh->n;
    ta.bounds = reinterpret_cast<const float4*>(bvh->view.bounds);
    ta.records = reinterpret_cast<const float4*>(bvh->view.records);
    ta.eps_bound = cp->error_bound;
    ta.clamp2 = gp->dist_clamp > 0.0f ? gp->dist_clamp * gp->dist_clamp : 0.0f;
    ta.tiles_x = tiles_x;
    ta.tiles_y = tiles_y;
    ta.info = info;
    ta.err = ctx->d_error;
    float4* extra = nullptr;
    ARC_TRY(ctx->arena.get("node_extra", (size_t)(bvh->n - 1) * 2 * sizeof(float4), reinterpret_cast<void**>(&extra)));
    stage_begin(ctx, "cut_setup");
    cut_tile_setup<<<(tiles + kSelWarps - 1) / kSelWarps, 32 * kSelWarps, 0, ctx->stream>>>(ta);
    cut_node_extra<<<(bvh->n - 1 + 255) / 256, 256, 0, ctx->stream>>>(bvh->n, ta.bounds, ta.records, extra);
    stage_end(ctx, 2);
    ARC_TRY_CUDA(cudaGetLastError());
    *info_out = info;
    *extra_out = extra;
    return ARC_OK;
}

arc_status launch_gather_cut(arc_context* ctx, const arc_lbvh* bvh, const ArcAvplsGpuParam* avpls,
                             const ArcGBufferView* gb, float3 cam, const ArcGatherParams* gp, const ArcCutParams* cp,
                             const ArcOutputView* out) {
    ARC_CHECK_ARG(bvh->n >= 2, "LBVH not built");
    ARC_CHECK_ARG(cp->kind >= 0 && cp->kind <= 2, "cut kind out of range");
    ARC_CHECK_ARG(gp->ar_kind >= 0 && gp->ar_kind <= 2, "ar_kind out of range");
    ARC_CHECK_ARG(gb->width > 0 && gb->height > 0 && gb->pitch >= gb->width && gb->position && gb->normal,
                  "bad G-buffer view");
    ARC_CHECK_ARG(out->pitch >= gb->width, "bad output view");
    ARC_CHECK_ARG(ctx->num_materials > 0, "materials not uploaded");
    cudaStream_t st = ctx->stream;
    const int W = gb->width, H = gb->height;
    const float clamp2 = gp->dist_clamp > 0.0f ? gp->dist_clamp * gp->dist_clamp : 0.0f;

    if (cp->kind == ARC_CUT_SOLID_ANGLE) {
        double *rad64 = nullptr, *ar64 = nullptr;
        const size_t np = (size_t)H * out->pitch;
        ARC_TRY(ctx->arena.get("cut_rad64", np * 3 * sizeof(double), reinterpret_cast<void**>(&rad64)));
        SolidArgs a;
        a.gpos = reinterpret_cast<const float4*>(gb->position);
        a.gnrm = reinterpret_cast<const float4*>(gb->normal);
        a.gpitch = gb->pitch;
        a.width = W;
        a.height = H;
        a.mats = ctx->d_materials;
        a.num_mats = ctx->num_materials;
        a.cam = cam;
        a.n = bvh->n;
        a.bounds = reinterpret_cast<const float4*>(bvh->view.bounds);
        a.nd = bvh->view.node_data;
        a.thresh = cp->solid_angle_threshold;
        a.clamp2 = clamp2;
        a.rad64 = rad64;
        a.out_rad = reinterpret_cast<float4*>(out->radiance);
        a.opitch = out->pitch;
        a.dbg_x = cp->debug_pixel_x;
        a.dbg_y = cp->debug_pixel_y;
        a.used = cp->used_nodes;
        a.err = ctx->d_error;
        dim3 grid((W + 15) / 16, (H + 15) / 16);
        stage_begin(ctx, "cut_solid_angle");
        cut_solid_angle_kernel<<<grid, 256, 0, st>>>(a);
        stage_end(ctx, 1);
        ARC_TRY_CUDA(cudaGetLastError());
        if (gp->ar_kind != ARC_AR_NONE) {
            ARC_CHECK_ARG(avpls != nullptr, "ARC_CUT_SOLID_ANGLE with antiradiance needs the AVPL arrays");
            ARC_TRY(ctx->arena.get("cut_ar64", np * 3 * sizeof(double), reinterpret_cast<void**>(&ar64)));
            GatherLaunch g{avpls, gb, cam, gp, out};
            ARC_TRY(launch_antiradiance_only(ctx, g, ar64));
        }
        dim3 cg((W + 31) / 32, (H + 7) / 8);
        stage_begin(ctx, "combine");
        combine_kernel<<<cg, dim3(32, 8), 0, st>>>(rad64, ar64, W, H, reinterpret_cast<float4*>(out->result),
                                                  reinterpret_cast<float4*>(out->antiradiance), out->result_fp64,
                                                  out->pitch);
        stage_end(ctx, 1);
        ARC_TRY_CUDA(cudaGetLastError());
        return ARC_OK;
    }

    // tile cuts
    const int tiles_x = (W + kTile - 1) / kTile, tiles_y = (H + kTile - 1) / kTile, tiles = tiles_x * tiles_y;
    const int max_cut = cp->max_cut_nodes > 0 ? cp->max_cut_nodes : (1 << 20);
    CutPool pool;
    pool.max_chunks = (max_cut + kChunkSize - 1) / kChunkSize;
    const int64_t pool_entries = cp->cut_pool_entries > 0 ? cp->cut_pool_entries : (int64_t)tiles * 32768;
    pool.num_chunks = (int32_t)std::min<int64_t>((pool_entries + kChunkSize - 1) / kChunkSize, INT32_MAX / kChunkSize);
    ARC_TRY(ctx->arena.get("cut_pool", (size_t)pool.num_chunks * kChunkSize * sizeof(int32_t),
                           reinterpret_cast<void**>(&pool.entries)));
    ARC_TRY(ctx->arena.get("cut_tables", (size_t)tiles * pool.max_chunks * sizeof(int32_t),
                           reinterpret_cast<void**>(&pool.tables)));
    ARC_TRY(ctx->arena.get("cut_counts", (size_t)tiles * sizeof(int32_t), reinterpret_cast<void**>(&pool.counts)));
    ARC_TRY(ctx->arena.get("cut_pool_next", sizeof(int32_t), reinterpret_cast<void**>(&pool.next)));
    ARC_TRY_CUDA(cudaMemsetAsync(pool.next, 0, sizeof(int32_t), st));
    float4* info = nullptr;
    float4* extra = nullptr;
    ARC_TRY(launch_tile_setup(ctx, bvh, gb, gp, cp, &info, &extra));
    TileArgs ta;
    ta.gpos = reinterpret_cast<const float4*>(gb->position);
    ta.gnrm = reinterpret_cast<const float4*>(gb->normal);
    ta.bounds = reinterpret_cast<const float4*>(bvh->view.bounds);
    ta.records = reinterpret_cast<const float4*>(bvh->view.records);

    if (cp->kind == ARC_CUT_ERROR_BOUND) {
        SelArgs sa;
        sa.n = bvh->n;
        sa.bounds = ta.bounds;
        sa.records = ta.records;
        sa.info = info;
        sa.extra = extra;
        sa.bp.clamp2 = clamp2;
        sa.bp.ar_kind = gp->ar_kind;
        sa.bp.eps_cone = 0.001f;
        sa.bp.cos_thr = fmaxf(cosf(gp->cone_half_angle), 0.001f);
        sa.bp.disk_scale = gp->disk_radius > 0.0f ? 1.0f / (kPi * gp->disk_radius * gp->disk_radius) : 0.0f;
        sa.bp.ar_uncertain = cp->ar_uncertain_factor;
        sa.tiles = tiles;
        sa.pool = pool;
        sa.err = ctx->d_error;
        const size_t smem = (size_t)kSelWarps * kSelStack * sizeof(int);
        ARC_TRY_CUDA(cudaFuncSetAttribute(cut_select_bound, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        stage_begin(ctx, "cut_select");
        cut_select_bound<<<(tiles + kSelWarps - 1) / kSelWarps, 32 * kSelWarps, smem, st>>>(sa);
        stage_end(ctx, 1);
        ARC_TRY_CUDA(cudaGetLastError());
    } else {
        ARC_CHECK_ARG(cp->model != nullptr, "ARC_CUT_LEARNED needs a model");
        ARC_TRY(launch_cut_select_learned(ctx, bvh, gp, cp, info, extra, tiles_x, tiles_y, pool));
    }

    EvalArgs ea;
    ea.gpos = ta.gpos;
    ea.gnrm = ta.gnrm;
    ea.gpitch = gb->pitch;
    ea.width = W;
    ea.height = H;
    ea.mats = ctx->d_materials;
    ea.num_mats = ctx->num_materials;
    ea.records = ta.records;
    ea.tiles_x = tiles_x;
    ea.pool = pool;
    ea.pc.cos_thr = fmaxf(cosf(gp->cone_half_angle), 0.001f);
    ea.pc.eps = 0.001f;
    ea.pc.inv_clamp2 = clamp2 > 0.0f ? 1.0f / clamp2 : INFINITY;
    ea.pc.disk_r2 = gp->disk_radius * gp->disk_radius;
    ea.disk_scale = gp->disk_radius > 0.0f ? 1.0f / (kPi * gp->disk_radius * gp->disk_radius) : 0.0f;
    ea.out_res = reinterpret_cast<float4*>(out->result);
    ea.out_rad = reinterpret_cast<float4*>(out->radiance);
    ea.out_ar = reinterpret_cast<float4*>(out->antiradiance);
    ea.out_res64 = out->result_fp64;
    ea.opitch = out->pitch;
    int* order = nullptr;
    ARC_TRY(ctx->arena.get("cut_order", (size_t)tiles * sizeof(int), reinterpret_cast<void**>(&order)));
    ea.order = order;
    stage_begin(ctx, "cut_eval");
    tile_order_kernel<<<1, 1024, 0, st>>>(pool.counts, tiles, order);
    if (gp->ar_kind == 0) cut_eval_packed_kernel<0><<<tiles, 64, 0, st>>>(ea);
    if (gp->ar_kind == 1) cut_eval_kernel<1><<<tiles, 64, 0, st>>>(ea);
    if (gp->ar_kind == 2) cut_eval_packed_kernel<2><<<tiles, 64, 0, st>>>(ea);
    stage_end(ctx, 2);
    ARC_TRY_CUDA(cudaGetLastError());
    ctx->last_cut.num_tiles = tiles;
    ctx->last_cut.pool = pool;
    return ARC_OK;
}

}  // namespace arc
