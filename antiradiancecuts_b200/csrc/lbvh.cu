// LBVH build over AVPLs (AvplBvh / Bvh::create, bvh.cu:325-454, 673-808; morton.h).
//
//   1. lbvh_bbox        min/max reduction (only for the reference's AVPL-box normalisation and
//                       for 6D codes), ordered-integer atomics
//   2. lbvh_morton      normalise with IEEE division (bvh.cu:73-81), quantise and interleave
//                       (morton.h:82-107), write (code, index) and the digit histograms of all
//                       four sort passes
//   3. radix sort       4 x 8-bit stable LSD passes, one kernel each: tiles ranked with warp
//                       match/ballot, tile offsets by decoupled look-back with bounded waits
//   4. lbvh_karras      Karras inner node i (bvh.cu:189-266) fused with the gather of sorted
//                       leaf i (the reference's zip-iterator payload sort, bvh.cu:793-808)
//   5. lbvh_bottom_up   second-arriving thread merges the two children (kernel_innerNodes +
//                       cluster, bvh.cu:280-316, 726-744) with release/acquire ordering that
//                       the reference lacks (no fence before its atomic)
//
// Every floating-point result is computed with explicitly rounded operations in a fixed order,
// so codes, topology, bounds, sums, representatives and cones equal the CPU build bit for bit.
#include <cfloat>
#include <cstdio>

#include "arc_internal.h"
#include "device_common.cuh"
#include "pcg32.h"

namespace arc {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortKPT = 8;  // keys per thread
constexpr int kSortTile = kSortThreads * kSortKPT;
constexpr int kSortWarps = kSortThreads / 32;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;

__device__ __forceinline__ uint32_t float_to_ordered(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u) {
    const uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return __uint_as_float(b);
}

// bbox slots: [0..2] pos min, [3..5] pos max, [6..8] normal min, [9..11] normal max
__global__ void lbvh_bbox_init(uint32_t* bb) {
    const int t = threadIdx.x;
    if (t < 12) {
        const int which = (t / 3) % 2;  // 0 = min, 1 = max
        // max is seeded with FLT_MIN as numeric_limits<float>::min() in bvh.cu:349-350, 357-358
        bb[t] = which == 0 ? float_to_ordered(FLT_MAX) : float_to_ordered(FLT_MIN);
    }
}

__global__ void lbvh_bbox(ArcAvplsGpuParam a, uint32_t* bb, int with_normals) {
    float mn[6], mx[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        mn[k] = FLT_MAX;
        mx[k] = FLT_MIN;
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.numAvpls;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float3 p = ld3(a.position, i);
        mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
        mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
        if (with_normals) {
            const float3 n = ld3(a.normal, i);
            mn[3] = fminf(mn[3], n.x); mn[4] = fminf(mn[4], n.y); mn[5] = fminf(mn[5], n.z);
            mx[3] = fmaxf(mx[3], n.x); mx[4] = fmaxf(mx[4], n.y); mx[5] = fmaxf(mx[5], n.z);
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(&bb[k], float_to_ordered(mn[k]));
            atomicMax(&bb[3 + k], float_to_ordered(mx[k]));
            if (with_normals) {
                atomicMin(&bb[6 + k], float_to_ordered(mn[3 + k]));
                atomicMax(&bb[9 + k], float_to_ordered(mx[3 + k]));
            }
        }
    }
}

__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t quant10(float v) {
    const float q = fminf(fmaxf(rn_mul(v, 1024.0f), 0.0f), 1023.0f);
    return (uint32_t)q;
}

struct MortonArgs {
    ArcAvplsGpuParam a;
    const uint32_t* bb;  // ordered-int bbox (when computed)
    float3 smin, smax;   // scene box
    int use_avpl_box;
    int consider_normals;
    uint32_t* keys;
    int32_t* vals;
    uint32_t* hist;  // [4][256]
};

__global__ void __launch_bounds__(256) lbvh_morton(MortonArgs m) {
    __shared__ uint32_t sh[4][256];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) (&sh[0][0])[i] = 0;
    __syncthreads();
    float mn[3], mx[3], nmn[3], nmx[3];
    if (m.use_avpl_box) {
        for (int k = 0; k < 3; ++k) {
            mn[k] = ordered_to_float(m.bb[k]);
            mx[k] = ordered_to_float(m.bb[3 + k]);
        }
    } else {
        mn[0] = m.smin.x; mn[1] = m.smin.y; mn[2] = m.smin.z;
        mx[0] = m.smax.x; mx[1] = m.smax.y; mx[2] = m.smax.z;
    }
    if (m.consider_normals)
        for (int k = 0; k < 3; ++k) {
            nmn[k] = ordered_to_float(m.bb[6 + k]);
            nmx[k] = ordered_to_float(m.bb[9 + k]);
        }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m.a.numAvpls;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float3 p = ld3(m.a.position, i);
        const float pv[3] = {p.x, p.y, p.z};
        uint32_t q[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) q[k] = quant10(rn_div(rn_sub(pv[k], mn[k]), rn_sub(mx[k], mn[k])));
        uint32_t code;
        if (!m.consider_normals) {
            code = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
        } else {
            // six 10-bit values interleaved into 64 bits (bit i of value k -> bit 6i + k),
            // truncated to the low 32 bits (MC_SIZE uint32_t, bvh.h:17)
            const float3 n = ld3(m.a.normal, i);
            const float nv[3] = {n.x, n.y, n.z};
            uint32_t u[6] = {q[0], q[1], q[2], 0, 0, 0};
#pragma unroll
            for (int k = 0; k < 3; ++k) u[3 + k] = quant10(rn_div(rn_sub(nv[k], nmn[k]), rn_sub(nmx[k], nmn[k])));
            uint64_t c = 0;
#pragma unroll
            for (int b = 0; b < 10; ++b)
#pragma unroll
                for (int k = 0; k < 6; ++k) c |= (uint64_t)((u[k] >> b) & 1u) << (6 * b + k);
            code = (uint32_t)c;
        }
        m.keys[i] = code;
        m.vals[i] = (int32_t)i;
#pragma unroll
        for (int pass = 0; pass < 4; ++pass) atomicAdd(&sh[pass][(code >> (8 * pass)) & 0xffu], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) {
        const uint32_t v = (&sh[0][0])[i];
        if (v) atomicAdd(&m.hist[i], v);
    }
}

// exclusive scan of each pass's 256-bin histogram (in place), one block of 256 threads
__global__ void lbvh_scan_hist(uint32_t* hist) {
    __shared__ uint32_t s[256];
    for (int pass = 0; pass < 4; ++pass) {
        const uint32_t v = hist[pass * 256 + threadIdx.x];
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 256; o <<= 1) {
            const uint32_t t = threadIdx.x >= o ? s[threadIdx.x - o] : 0u;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        hist[pass * 256 + threadIdx.x] = s[threadIdx.x] - v;
        __syncthreads();
    }
}

struct SortPassArgs {
    const uint32_t* keys_in;
    const int32_t* vals_in;
    uint32_t* keys_out;
    int32_t* vals_out;
    const uint32_t* digit_base;  // 256 exclusive offsets of this pass
    uint32_t* status;            // [tiles][256]
    uint32_t* tile_counter;
    int32_t n;
    int shift;
    int pass;
    uint32_t spin_limit;  // polls of the look-back before it gives up
    uint32_t* abort;      // the build's abort word: 1 + the pass whose look-back gave up, or 0
    uint32_t* err;
};

__global__ void __launch_bounds__(kSortThreads) lbvh_sort_pass(SortPassArgs s) {
    __shared__ uint32_t warp_cnt[kSortWarps][256];
    __shared__ uint32_t tile_off[256];
    __shared__ int tile_sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // An earlier pass gave up (its output is not a permutation, so this pass's digit offsets,
    // counted from the unsorted keys, no longer bound its writes): the build stops here.  CTAs of
    // the pass that gave up keep going, so that none of its tiles waits on a tile that left.
    const uint32_t ab = *reinterpret_cast<volatile uint32_t*>(s.abort);
    if (ab != 0u && ab <= (uint32_t)s.pass) return;
    if (tid == 0) tile_sh = (int)atomicAdd(s.tile_counter, 1u);
    for (int i = tid; i < kSortWarps * 256; i += kSortThreads) (&warp_cnt[0][0])[i] = 0;
    __syncthreads();
    const int tile = tile_sh;
    const int64_t base = (int64_t)tile * kSortTile + (int64_t)warp * 32 * kSortKPT;

    uint32_t key[kSortKPT], digit[kSortKPT], rank[kSortKPT];
    int32_t val[kSortKPT];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kSortKPT; ++j) {
        const int64_t idx = base + j * 32 + lane;
        const bool in = idx < s.n;
        key[j] = in ? s.keys_in[idx] : 0xffffffffu;
        val[j] = in ? s.vals_in[idx] : 0;
        digit[j] = in ? ((key[j] >> s.shift) & 0xffu) : 256u;
        const unsigned active = __ballot_sync(0xffffffffu, in);
        rank[j] = 0;
        if (in) {
            const unsigned peers = __match_any_sync(active, digit[j]);
            const int leader = __ffs(peers) - 1;
            uint32_t before = 0;
            if (lane == leader) {
                before = warp_cnt[warp][digit[j]];
                warp_cnt[warp][digit[j]] = before + __popc(peers);
            }
            before = __shfl_sync(peers, before, leader);
            rank[j] = before + __popc(peers & lt);
        }
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive offsets across warps, tile total, then decoupled look-back
    {
        const int d = tid;  // 256 threads, one digit each
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = warp_cnt[w][d];
            warp_cnt[w][d] = run;
            run += c;
        }
        const uint32_t total = run;
        volatile uint32_t* st = s.status;
        uint32_t excl = 0;
        if (tile == 0) {
            st[d] = kFlagPrefix | total;
        } else {
            st[(size_t)tile * 256 + d] = kFlagAgg | total;
            int t = tile - 1;
            uint32_t spins = 0;
            while (t >= 0) {
                const uint32_t v = st[(size_t)t * 256 + d];
                if ((v & ~kValueMask) == 0) {
                    if (++spins > s.spin_limit) {
                        // publish what was summed: later tiles' offsets stay within the digit's
                        // range, and the passes after this one do not run
                        set_error(s.err, ARC_DEVERR_TIMEOUT);
                        atomicMax(s.abort, (uint32_t)s.pass + 1u);
                        break;
                    }
                    continue;
                }
                excl += v & kValueMask;
                if (v & kFlagPrefix) break;
                --t;
            }
            __threadfence();
            st[(size_t)tile * 256 + d] = kFlagPrefix | (excl + total);
        }
        tile_off[d] = s.digit_base[d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortKPT; ++j) {
        if (digit[j] < 256u) {
            const uint32_t pos = tile_off[digit[j]] + warp_cnt[warp][digit[j]] + rank[j];
            s.keys_out[pos] = key[j];
            s.vals_out[pos] = val[j];
        }
    }
}

// delta(i, j) (cuda_delta, bvh.cu:124-135)
__device__ __forceinline__ int kdelta(const uint32_t* __restrict__ m, int num_nodes, int i, int64_t j) {
    if (j < 0 || j > num_nodes) return -1;
    int d = __clz(m[i] ^ m[j]);
    if (d == 32) d += __clz((uint32_t)(i ^ (int)j));
    return d;
}

struct KarrasArgs {
    const uint32_t* morton;
    const int32_t* sorted_index;
    ArcAvplsGpuParam a;
    const MaterialRecord* mats;
    int32_t num_mats;
    int32_t n;
    uint32_t seed;
    int32_t* left;
    int32_t* right;
    int32_t* parents;
    int32_t* range;
    float4* records;   // [2N-1][4]
    float4* cones;     // [2N-1][2] {normal axis, cos}, {direction axis, cos}
    float4* dirstat;   // [2N-1] {S.xyz, a}: a = sum of antiradiance luminances, S = sum of a_i w_i / |w_i|
    float4* bbox;      // [2N-1][2] scratch: {min, 0}, {max, 0} of leaf boxes then inner boxes
    ArcAvplBvhNodeDataParam nd;
    ArcFloat3* sorted_pos;
    ArcFloat3* sorted_nrm;
    const uint32_t* abort;  // set when the sort gave up: its order is not a permutation
    uint32_t* err;
};

__global__ void __launch_bounds__(256) lbvh_karras(KarrasArgs k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = k.n, num_nodes = n - 1;
    if (i >= n || *k.abort != 0u) return;
    // ---- inner node i ----
    if (i < num_nodes) {
        const uint32_t* m = k.morton;
        const int d = (kdelta(m, num_nodes, i, i + 1) - kdelta(m, num_nodes, i, i - 1)) < 0 ? -1 : 1;
        const int delta_min = kdelta(m, num_nodes, i, i - d);
        int64_t l_max = 128;
        while (kdelta(m, num_nodes, i, i + l_max * d) > delta_min) l_max *= 4;
        int64_t l = 0;
        for (int64_t t = l_max / 2; t > 0; t /= 2)
            if (kdelta(m, num_nodes, i, i + (l + t) * d) > delta_min) l += t;
        const int64_t j = i + l * d;
        const int delta_node = kdelta(m, num_nodes, i, j);
        int64_t s = 0, kk = 2, t = (l + kk - 1) / kk;
        while (true) {
            if (kdelta(m, num_nodes, i, i + (s + t) * d) > delta_node) s += t;
            if (t <= 1) break;
            kk *= 2;
            t = (l + kk - 1) / kk;
        }
        const int split = (int)(i + s * d + min(d, 0));
        const int lo = (int)min((int64_t)i, j), hi = (int)max((int64_t)i, j);
        const int lc = lo == split ? split : -(split + 1);
        const int rc = hi == split + 1 ? split + 1 : -(split + 2);
        k.left[i] = lc;
        k.right[i] = rc;
        k.range[2 * i] = lo;
        k.range[2 * i + 1] = hi;
        k.parents[lc >= 0 ? lc : n - (lc + 1)] = i;
        k.parents[rc >= 0 ? rc : n - (rc + 1)] = i;
        if (i == 0) k.parents[n] = -1;
    }
    // ---- sorted leaf i ----
    const int src = k.sorted_index[i];
    const float3 p = ld3(k.a.position, src), nr = ld3(k.a.normal, src), w = ld3(k.a.incDirection, src);
    const float3 L = ld3(k.a.incRadiance, src), A = ld3(k.a.antiradiance, src);
    int mat = k.a.materialIndex[src];
    if (mat < 0 || mat >= k.num_mats) {
        set_error(k.err, ARC_DEVERR_BAD_MATERIAL);
        mat = 0;
    }
    const float4 dif = k.mats[mat].diffuse_exp;
    const bool light = (w.x == 0.0f && w.y == 0.0f && w.z == 0.0f);
    float4* r = k.records + 4 * (size_t)i;
    r[0] = make_float4(p.x, p.y, p.z, nr.x);
    r[1] = make_float4(nr.y, nr.z, w.x, w.y);
    r[2] = make_float4(w.z, light ? L.x : rn_mul(L.x, rn_mul(kOneOverPi, dif.x)),
                       light ? L.y : rn_mul(L.y, rn_mul(kOneOverPi, dif.y)),
                       light ? L.z : rn_mul(L.z, rn_mul(kOneOverPi, dif.z)));
    r[3] = make_float4(A.x, A.y, A.z, 1.0f);
    // leaf cones: (n, 1) and (w/|w|, 1), or the whole sphere when w = 0
    float4* c = k.cones + 2 * (size_t)i;
    c[0] = make_float4(nr.x, nr.y, nr.z, 1.0f);
    const float ww = rn_dot(w.x, w.y, w.z, w.x, w.y, w.z);
    const float a_lum = rn_add(rn_add(rn_mul(0.2126f, A.x), rn_mul(0.7152f, A.y)), rn_mul(0.0722f, A.z));
    if (ww > 0.0f) {
        const float inv = rn_div(1.0f, rn_sqrt(ww));
        c[1] = make_float4(rn_mul(w.x, inv), rn_mul(w.y, inv), rn_mul(w.z, inv), 1.0f);
        k.dirstat[i] = make_float4(rn_mul(a_lum, c[1].x), rn_mul(a_lum, c[1].y), rn_mul(a_lum, c[1].z), a_lum);
    } else {
        c[1] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        k.dirstat[i] = make_float4(0.0f, 0.0f, 0.0f, a_lum);
    }
    k.bbox[2 * (size_t)i] = make_float4(p.x, p.y, p.z, 0.0f);
    k.bbox[2 * (size_t)i + 1] = make_float4(p.x, p.y, p.z, 0.0f);
    // reference node-data layout (AvplBvhNodeData, bvh.cu:673-724, sorted as bvh.cu:793-808)
    k.nd.size[i] = 1;
    k.nd.materialIndex[i] = mat;
    k.nd.randomNumbers[i] = arc_node_random(k.seed, (uint32_t)i);
    reinterpret_cast<float*>(k.nd.position)[3 * i + 0] = p.x;
    reinterpret_cast<float*>(k.nd.position)[3 * i + 1] = p.y;
    reinterpret_cast<float*>(k.nd.position)[3 * i + 2] = p.z;
    reinterpret_cast<float*>(k.nd.normal)[3 * i + 0] = nr.x;
    reinterpret_cast<float*>(k.nd.normal)[3 * i + 1] = nr.y;
    reinterpret_cast<float*>(k.nd.normal)[3 * i + 2] = nr.z;
    reinterpret_cast<float*>(k.nd.incRadiance)[3 * i + 0] = L.x;
    reinterpret_cast<float*>(k.nd.incRadiance)[3 * i + 1] = L.y;
    reinterpret_cast<float*>(k.nd.incRadiance)[3 * i + 2] = L.z;
    reinterpret_cast<float*>(k.nd.incDirection)[3 * i + 0] = w.x;
    reinterpret_cast<float*>(k.nd.incDirection)[3 * i + 1] = w.y;
    reinterpret_cast<float*>(k.nd.incDirection)[3 * i + 2] = w.z;
    k.sorted_pos[i] = ArcFloat3{p.x, p.y, p.z};
    k.sorted_nrm[i] = ArcFloat3{nr.x, nr.y, nr.z};
}

// union of two cones; same operation order as the CPU build's cone_union
__device__ __forceinline__ float4 cone_union(float4 c1, float4 c2) {
    if (c1.w <= -1.0f || c2.w <= -1.0f) return make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    const float sx = rn_add(c1.x, c2.x), sy = rn_add(c1.y, c2.y), sz = rn_add(c1.z, c2.z);
    const float l2 = rn_dot(sx, sy, sz, sx, sy, sz);
    if (!(l2 > 1e-12f)) return make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    const float inv = rn_div(1.0f, rn_sqrt(l2));
    const float ax = rn_mul(sx, inv), ay = rn_mul(sy, inv), az = rn_mul(sz, inv);
    float res = 1.0f;
    const float4 ci[2] = {c1, c2};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float d = rn_dot(ax, ay, az, ci[q].x, ci[q].y, ci[q].z);
        d = fminf(fmaxf(d, -1.0f), 1.0f);
        const float sd = rn_sqrt(fmaxf(0.0f, rn_sub(1.0f, rn_mul(d, d))));
        const float si = rn_sqrt(fmaxf(0.0f, rn_sub(1.0f, rn_mul(ci[q].w, ci[q].w))));
        const float v = ci[q].w < -d ? -1.0f : rn_sub(rn_mul(d, ci[q].w), rn_mul(sd, si));
        res = fminf(res, v);
    }
    return make_float4(ax, ay, az, res);
}

struct BottomUpArgs {
    const uint32_t* abort;  // set when the sort gave up
    uint32_t* err;
    int32_t n;
    uint32_t seed;
    const int32_t* left;
    const int32_t* right;
    const int32_t* parents;
    const int32_t* range;  // [N-1][2]: first and last leaf of each inner node
    int32_t* visit;
    float4* records;
    float4* cones;
    float4* dirstat;
    float4* bbox;
    float4* bounds;  // [N-1][4]
    ArcAvplBvhNodeDataParam nd;
};

// Loads of a child's data in the merge.  A child merged by a thread of the same block (LOCAL) was
// published with a block-scope release, so the load goes through the SM's L1; a child merged in
// another block was published with a device-scope release and is read from L2.
template <bool LOCAL, typename T>
__device__ __forceinline__ T ld_child(const T* p) {
    if (LOCAL) return *p;
    return __ldcg(p);
}

// Merges the two children of inner node k (the second thread to arrive does it); same operations
// and order as the CPU build's bottom-up pass.
template <bool LOCAL>
__device__ __forceinline__ void merge_node(const BottomUpArgs& b, int k, int lc, int rc) {
    const int n = b.n;
    const int t = n + k;
    const int l = lc >= 0 ? lc : n - (lc + 1);
    const int r = rc >= 0 ? rc : n - (rc + 1);
    // bounding box
    const float4 lmin = ld_child<LOCAL>(b.bbox + 2 * (size_t)l), lmax = ld_child<LOCAL>(b.bbox + 2 * (size_t)l + 1);
    const float4 rmin = ld_child<LOCAL>(b.bbox + 2 * (size_t)r), rmax = ld_child<LOCAL>(b.bbox + 2 * (size_t)r + 1);
    const float bt[6] = {fminf(lmin.x, rmin.x), fminf(lmin.y, rmin.y), fminf(lmin.z, rmin.z),
                         fmaxf(lmax.x, rmax.x), fmaxf(lmax.y, rmax.y), fmaxf(lmax.z, rmax.z)};
    b.bbox[2 * (size_t)t] = make_float4(bt[0], bt[1], bt[2], 0.0f);
    b.bbox[2 * (size_t)t + 1] = make_float4(bt[3], bt[4], bt[5], 0.0f);
    // representative (cluster, bvh.cu:726-744)
    const float* Lf = reinterpret_cast<const float*>(b.nd.incRadiance);
    const float Ll[3] = {ld_child<LOCAL>(Lf + 3 * l), ld_child<LOCAL>(Lf + 3 * l + 1), ld_child<LOCAL>(Lf + 3 * l + 2)};
    const float Lr[3] = {ld_child<LOCAL>(Lf + 3 * r), ld_child<LOCAL>(Lf + 3 * r + 1), ld_child<LOCAL>(Lf + 3 * r + 2)};
    const float i1 = rn_sqrt(rn_dot(Ll[0], Ll[1], Ll[2], Ll[0], Ll[1], Ll[2]));
    const float i2 = rn_sqrt(rn_dot(Lr[0], Lr[1], Lr[2], Lr[0], Lr[1], Lr[2]));
    const float rnd = arc_node_random(b.seed, (uint32_t)t);
    const int repr = rnd > rn_div(i1, rn_add(i1, i2)) ? r : l;
    const int sl = ld_child<LOCAL>(b.nd.size + l), sr = ld_child<LOCAL>(b.nd.size + r);
    b.nd.randomNumbers[t] = rnd;
    b.nd.size[t] = sl + sr;
    b.nd.materialIndex[t] = ld_child<LOCAL>(b.nd.materialIndex + repr);
    float* Lt = reinterpret_cast<float*>(b.nd.incRadiance);
    float* P = reinterpret_cast<float*>(b.nd.position);
    float* N = reinterpret_cast<float*>(b.nd.normal);
    float* W = reinterpret_cast<float*>(b.nd.incDirection);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        Lt[3 * t + q] = rn_add(Ll[q], Lr[q]);
        P[3 * t + q] = ld_child<LOCAL>(P + 3 * repr + q);
        N[3 * t + q] = ld_child<LOCAL>(N + 3 * repr + q);
        W[3 * t + q] = ld_child<LOCAL>(W + 3 * repr + q);
    }
    // direction statistics, and the antiradiance representative: drawn in proportion to
    // antiradiance luminance with the same random number; its direction is the record's w
    const float4 dl = ld_child<LOCAL>(b.dirstat + l), dr = ld_child<LOCAL>(b.dirstat + r);
    const float4 dt = make_float4(rn_add(dl.x, dr.x), rn_add(dl.y, dr.y), rn_add(dl.z, dr.z), rn_add(dl.w, dr.w));
    b.dirstat[t] = dt;
    const int arep = dt.w > 0.0f ? (rnd > rn_div(dl.w, dt.w) ? r : l) : repr;
    // packed record: representative p/n, antiradiance representative's w, summed L' and A, count
    const float* R = reinterpret_cast<const float*>(b.records);
    float rt[16];
#pragma unroll
    for (int q = 0; q < 6; ++q) rt[q] = ld_child<LOCAL>(R + 16 * (size_t)repr + q);
#pragma unroll
    for (int q = 6; q < 9; ++q) rt[q] = ld_child<LOCAL>(R + 16 * (size_t)arep + q);
#pragma unroll
    for (int q = 9; q < 15; ++q)
        rt[q] = rn_add(ld_child<LOCAL>(R + 16 * (size_t)l + q), ld_child<LOCAL>(R + 16 * (size_t)r + q));
    rt[15] = (float)(sl + sr);
    float4* rec = b.records + 4 * (size_t)t;
    rec[0] = make_float4(rt[0], rt[1], rt[2], rt[3]);
    rec[1] = make_float4(rt[4], rt[5], rt[6], rt[7]);
    rec[2] = make_float4(rt[8], rt[9], rt[10], rt[11]);
    rec[3] = make_float4(rt[12], rt[13], rt[14], rt[15]);
    // cones
    const float4 cnl = ld_child<LOCAL>(b.cones + 2 * (size_t)l), cnr = ld_child<LOCAL>(b.cones + 2 * (size_t)r);
    const float4 cwl = ld_child<LOCAL>(b.cones + 2 * (size_t)l + 1), cwr = ld_child<LOCAL>(b.cones + 2 * (size_t)r + 1);
    const float4 cn = cone_union(cnl, cnr), cw = cone_union(cwl, cwr);
    b.cones[2 * (size_t)t] = cn;
    b.cones[2 * (size_t)t + 1] = cw;
    float4* bd = b.bounds + 4 * (size_t)k;
    bd[0] = make_float4(bt[0], bt[1], bt[2], __int_as_float(lc));
    bd[1] = make_float4(bt[3], bt[4], bt[5], __int_as_float(rc));
    bd[2] = cn;
    bd[3] = cw;
}

// One thread per leaf climbs towards the root; at each inner node the first thread to arrive
// stops and the second merges the two children.  Nodes whose leaf range lies inside the block's
// kBottomUpThreads leaves are settled in shared memory with block-scope ordering (both arrivals
// come from this block); the others through the global visit counters with device-scope fences.
constexpr int kBottomUpThreads = 256;

__global__ void __launch_bounds__(kBottomUpThreads) lbvh_bottom_up(BottomUpArgs b) {
    __shared__ int arrivals[kBottomUpThreads];
    arrivals[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kBottomUpThreads;
    const int i = base + threadIdx.x;
    const int n = b.n;
    if (*b.abort != 0u) return;  // uniform over the CTA: before any barrier below
    if (i >= n) return;
    int parent = b.parents[i];
    // a valid tree reaches the root within n - 1 steps; the bound guards against a corrupt one
    for (int steps = 0; parent >= 0; ++steps) {
        if (steps >= n || parent >= n - 1) {
            set_error(b.err, ARC_DEVERR_BAD_NODE);
            return;
        }
        const int k = parent;
        const int2 rg = *reinterpret_cast<const int2*>(b.range + 2 * (size_t)k);
        const int lc = b.left[k], rc = b.right[k];
        // node k is one end of its own range, so a local node's slot k - base is in [0, 256)
        const bool local = rg.x >= base && rg.y < base + kBottomUpThreads && k >= base && k < base + kBottomUpThreads;
        if (local) {
            __threadfence_block();  // release this thread's writes (the child it just finished)
            if (atomicAdd(&arrivals[k - base], 1) == 0) return;
            __threadfence_block();  // acquire the sibling's writes
            merge_node<true>(b, k, lc, rc);
        } else {
            __threadfence();
            if (atomicAdd(&b.visit[k], 1) == 0) return;
            __threadfence();
            merge_node<false>(b, k, lc, rc);
        }
        parent = b.parents[n + k];
    }
}

__global__ void lbvh_reference_nodes(int32_t num_nodes, const float4* bounds, ArcBvhNode* nodes) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= num_nodes) return;
    const float4 b0 = bounds[4 * (size_t)k], b1 = bounds[4 * (size_t)k + 1];
    ArcBvhNode nd;
    nd.left = __float_as_int(b0.w);
    nd.right = __float_as_int(b1.w);
    nd.bbMin = ArcFloat3{b0.x, b0.y, b0.z};
    nd.bbMax = ArcFloat3{b1.x, b1.y, b1.z};
    nd.visited = 2;  // both children merged
    nodes[k] = nd;
}

template <typename T>
arc_status get(arc_lbvh* bvh, const char* name, size_t count, T** out) {
    return bvh->arena.get(name, sizeof(T) * (count > 0 ? count : 1), reinterpret_cast<void**>(out));
}

}  // namespace

arc_status launch_lbvh_build(arc_lbvh* bvh, const ArcAvplsGpuParam* avpls, const ArcLbvhParams* p) {
    arc_context* ctx = bvh->ctx;
    const int32_t n = avpls->numAvpls;
    if (n < 2) {
        set_last_error("not enough points for bvh construction (need >= 2 AVPLs)");
        return ARC_ERR_TOO_FEW_AVPLS;
    }
    ARC_CHECK_ARG(n < (1 << 29), "too many AVPLs for the LBVH (max 2^29 - 1)");
    ARC_CHECK_ARG(ctx->num_materials > 0, "materials not uploaded");
    ARC_CHECK_ARG(p->bbox_mode == ARC_BBOX_SCENE || p->bbox_mode == ARC_BBOX_AVPL_REFERENCE, "bad bbox_mode");
    cudaStream_t st = ctx->stream;
    const int total = 2 * n - 1;
    const int tiles = (n + kSortTile - 1) / kSortTile;

    uint32_t *keys0, *keys1, *hist, *status, *bb;
    int32_t *vals0, *vals1, *left, *right, *parents, *range, *visit;
    float4 *records, *cones, *bounds, *dirstat;
    float4* bbox;
    ARC_TRY(get(bvh, "keys0", n, &keys0));
    ARC_TRY(get(bvh, "keys1", n, &keys1));
    ARC_TRY(get(bvh, "vals0", n, &vals0));
    ARC_TRY(get(bvh, "vals1", n, &vals1));
    // hist[4*256] | tile counters[4] | bbox[12] | abort word share one zeroed block
    ARC_TRY(get(bvh, "hist", 1024 + 4 + 12 + 1, &hist));
    ARC_TRY(get(bvh, "status", (size_t)4 * tiles * 256, &status));
    ARC_TRY(get(bvh, "left", n - 1, &left));
    ARC_TRY(get(bvh, "right", n - 1, &right));
    ARC_TRY(get(bvh, "parents", total, &parents));
    ARC_TRY(get(bvh, "range", 2 * (n - 1), &range));
    ARC_TRY(get(bvh, "visit", n - 1, &visit));
    ARC_TRY(get(bvh, "records", (size_t)4 * total, &records));
    ARC_TRY(get(bvh, "cones", (size_t)2 * total, &cones));
    ARC_TRY(get(bvh, "dirstat", total, &dirstat));
    ARC_TRY(get(bvh, "bounds", (size_t)4 * (n - 1), &bounds));
    ARC_TRY(get(bvh, "bbox", (size_t)2 * total, &bbox));
    ArcAvplBvhNodeDataParam nd;
    ARC_TRY(get(bvh, "nd_size", total, &nd.size));
    ARC_TRY(get(bvh, "nd_mat", total, &nd.materialIndex));
    ARC_TRY(get(bvh, "nd_rand", total, &nd.randomNumbers));
    ARC_TRY(get(bvh, "nd_pos", total, &nd.position));
    ARC_TRY(get(bvh, "nd_nrm", total, &nd.normal));
    ARC_TRY(get(bvh, "nd_L", total, &nd.incRadiance));
    ARC_TRY(get(bvh, "nd_w", total, &nd.incDirection));
    ARC_TRY(get(bvh, "sorted_pos", n, &bvh->sorted_positions));
    ARC_TRY(get(bvh, "sorted_nrm", n, &bvh->sorted_normals));
    bb = hist + 1024 + 4;
    uint32_t* tile_counters = hist + 1024;
    uint32_t* abort = hist + 1024 + 4 + 12;

    ARC_TRY_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 1028, st));
    ARC_TRY_CUDA(cudaMemsetAsync(abort, 0, sizeof(uint32_t), st));
    ARC_TRY_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t) * 4 * (size_t)tiles * 256, st));
    ARC_TRY_CUDA(cudaMemsetAsync(visit, 0, sizeof(int32_t) * (size_t)(n - 1), st));

    const int grid_stride_blocks = ctx->sm_count * 4;
    stage_begin(ctx, "lbvh_morton");
    const bool need_box = p->bbox_mode == ARC_BBOX_AVPL_REFERENCE || p->consider_normals;
    if (need_box) {
        lbvh_bbox_init<<<1, 32, 0, st>>>(bb);
        lbvh_bbox<<<grid_stride_blocks, 256, 0, st>>>(*avpls, bb, p->consider_normals);
        ARC_TRY_CUDA(cudaGetLastError());
    }
    MortonArgs m;
    m.a = *avpls;
    m.bb = bb;
    m.smin = make_float3(p->scene_min.x, p->scene_min.y, p->scene_min.z);
    m.smax = make_float3(p->scene_max.x, p->scene_max.y, p->scene_max.z);
    m.use_avpl_box = p->bbox_mode == ARC_BBOX_AVPL_REFERENCE;
    m.consider_normals = p->consider_normals;
    m.keys = keys0;
    m.vals = vals0;
    m.hist = hist;
    lbvh_morton<<<grid_stride_blocks, 256, 0, st>>>(m);
    lbvh_scan_hist<<<1, 256, 0, st>>>(hist);
    stage_end(ctx, need_box ? 4 : 2);
    ARC_TRY_CUDA(cudaGetLastError());
    stage_begin(ctx, "lbvh_sort");

    uint32_t* kin = keys0;
    uint32_t* kout = keys1;
    int32_t* vin = vals0;
    int32_t* vout = vals1;
    for (int pass = 0; pass < 4; ++pass) {
        SortPassArgs s;
        s.keys_in = kin;
        s.vals_in = vin;
        s.keys_out = kout;
        s.vals_out = vout;
        s.digit_base = hist + 256 * pass;
        s.status = status + (size_t)pass * tiles * 256;
        s.tile_counter = tile_counters + pass;
        s.n = n;
        s.shift = 8 * pass;
        s.pass = pass;
        s.spin_limit = p->wait_limit ? p->wait_limit : (1u << 26);
        s.abort = abort;
        s.err = ctx->d_error;
        lbvh_sort_pass<<<tiles, kSortThreads, 0, st>>>(s);
        ARC_TRY_CUDA(cudaGetLastError());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    // after 4 passes the sorted data is back in keys0 / vals0
    stage_end(ctx, 4);
    stage_begin(ctx, "lbvh_karras");

    KarrasArgs k;
    k.morton = kin;
    k.sorted_index = vin;
    k.a = *avpls;
    k.mats = ctx->d_materials;
    k.num_mats = ctx->num_materials;
    k.n = n;
    k.seed = p->repr_seed;
    k.left = left;
    k.right = right;
    k.parents = parents;
    k.range = range;
    k.records = records;
    k.cones = cones;
    k.dirstat = dirstat;
    k.bbox = bbox;
    k.nd = nd;
    k.sorted_pos = bvh->sorted_positions;
    k.sorted_nrm = bvh->sorted_normals;
    k.abort = abort;
    k.err = ctx->d_error;
    lbvh_karras<<<(n + 255) / 256, 256, 0, st>>>(k);
    stage_end(ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());

    BottomUpArgs bu;
    bu.n = n;
    bu.seed = p->repr_seed;
    bu.left = left;
    bu.right = right;
    bu.parents = parents;
    bu.range = range;
    bu.visit = visit;
    bu.records = records;
    bu.cones = cones;
    bu.dirstat = dirstat;
    bu.bbox = bbox;
    bu.bounds = bounds;
    bu.nd = nd;
    bu.abort = abort;
    bu.err = ctx->d_error;
    stage_begin(ctx, "lbvh_bottom_up");
    lbvh_bottom_up<<<(n + kBottomUpThreads - 1) / kBottomUpThreads, kBottomUpThreads, 0, st>>>(bu);
    stage_end(ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());

    bvh->n = n;
    ArcLbvhView& v = bvh->view;
    v.num_leaves = n;
    v.num_nodes = n - 1;
    v.morton = kin;
    v.sorted_index = vin;
    v.left = left;
    v.right = right;
    v.parents = parents;
    v.range = range;
    v.bounds = reinterpret_cast<const float*>(bounds);
    v.records = reinterpret_cast<const float*>(records);
    v.node_data = nd;
    v.dirstat = reinterpret_cast<const float*>(dirstat);
    bvh->has_reference_nodes = false;
    if (p->wait_limit != 0) {
        // a caller-chosen wait limit: learn now whether the sort gave up, and if it did leave the
        // object unbuilt (its arrays hold no tree) and report the timeout
        uint32_t aborted = 0;
        ARC_TRY_CUDA(cudaMemcpyAsync(&aborted, abort, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        ARC_TRY_CUDA(cudaStreamSynchronize(st));
        if (aborted) {
            bvh->n = 0;
            set_last_error("LBVH build: the radix sort's look-back gave up after " + std::to_string(p->wait_limit) +
                           " polls (pass " + std::to_string(aborted - 1) + ")");
            return ARC_ERR_TIMEOUT;
        }
    }
    return ARC_OK;
}

arc_status launch_lbvh_reference_nodes(arc_lbvh* bvh) {
    const int32_t n = bvh->n;
    ArcBvhNode* nodes = nullptr;
    ARC_TRY(bvh->arena.get("ref_nodes", sizeof(ArcBvhNode) * (size_t)(n - 1), reinterpret_cast<void**>(&nodes)));
    stage_begin(bvh->ctx, "lbvh_reference_nodes");
    lbvh_reference_nodes<<<(n - 1 + 255) / 256, 256, 0, bvh->ctx->stream>>>(
        n - 1, reinterpret_cast<const float4*>(bvh->view.bounds), nodes);
    stage_end(bvh->ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());
    bvh->ref_param.numLeafs = n;
    bvh->ref_param.numNodes = n - 1;
    bvh->ref_param.nodes = nodes;
    bvh->ref_param.positions = bvh->sorted_positions;
    bvh->ref_param.normals = bvh->sorted_normals;
    bvh->ref_data = bvh->view.node_data;
    bvh->has_reference_nodes = true;
    return ARC_OK;
}

}  // namespace arc
