// Learned cut selection and its training data.
//
// Selection (ARC_CUT_LEARNED): a level-synchronous walk over all tiles at once.  Level l holds
// the (tile, node) pairs at depth l.  One fused launch per level (learned_level) does, for every
// pair:
//   * leaves, and inner nodes whose analytic bound is already within the tile's threshold, are
//     accepted (the learned cut is never finer than the analytic one);
//   * inner nodes whose bound exceeds mlp_band times the threshold are refined (their children go
//     to level l + 1) without the network;
//   * every other pair's 16 features (BF16) are staged as one row in shared memory; each time
//     the CTA has 256 rows (two 128-row tiles, one set of weights) they are scored on the tensor
//     cores (mlp_tile.cuh) and their pairs are refined or accepted by the logit, in the same
//     launch.
// Persistent CTAs take 256 pairs at a time from a per-level work counter (the next chunk fetched
// one ahead); pushes and accepts reserve their slots with one atomic per CTA and kind.  The walk
// reads nothing back on the host: it launches a fixed number of levels, and a launch past the
// deepest frontier returns at once.  Accepted pairs are finally grouped by tile into the chunked
// cut pool (count, scan, scatter), which the shared cut evaluation reads.
//
// Training data (arc_cut_training_samples): for a batch of tiles, label_prefix computes, per
// pixel, the FP64 prefix sums over the sorted leaves of the luminance of each leaf's signed
// contribution; a node's exact contribution is then a difference of two prefixes (its leaves form
// one contiguous range).  label_traverse walks each tile's tree with the exact decision: refine iff
// max over the tile's pixels |exact - node estimate| > delta * mean |exact tile value|, and emits
// (features, label, error) for every visited node that the selection would score: the analytic
// bound neither accepts it nor puts it above the refine band (plus one level below accepted
// nodes, so the model also sees the children it would skip).  The error is the RMS over the tile's
// pixels of |exact node contribution - node estimate|, against delta * mean |exact tile value|.
#include <cuda_bf16.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "arc_internal.h"
#include "cut_bounds.cuh"
#include "device_common.cuh"
#include "mlp_tile.cuh"
#include "pair_math.cuh"
#include "tcgen05.cuh"

namespace arc {

const float* mlp_params(const arc_mlp* m);
int32_t mlp_loss_kind(const arc_mlp* m);
int32_t mlp_activation(const arc_mlp* m);

namespace {

constexpr int kTile = 8;
constexpr int kFeat = 16;
constexpr int kChunk = 1024;

__device__ __forceinline__ TileInfo load_tile_info(const float4* info, int tile, float* mean) {
    const float4 i0 = info[4 * (size_t)tile], i1 = info[4 * (size_t)tile + 1], i2 = info[4 * (size_t)tile + 2],
                 i3 = info[4 * (size_t)tile + 3];
    TileInfo t;
    t.tmin[0] = i0.x; t.tmin[1] = i0.y; t.tmin[2] = i0.z; t.kdl = i0.w;
    t.tmax[0] = i1.x; t.tmax[1] = i1.y; t.tmax[2] = i1.z; t.tau = i1.w;
    t.ncone = i2;
    t.valid = __float_as_int(i3.x);
    *mean = i3.y;
    t.rt = i3.z;
    t.sn = i3.w;
    return t;
}

// The same record from the field-major copy the selection reads (info_t[k * tiles + tile] =
// info[4 * tile + k], tile_info_transpose): a warp whose lanes hold consecutive tiles loads each
// float4 of 32 tiles from 512 contiguous bytes instead of 32 lines 64 bytes apart.
__device__ __forceinline__ TileInfo load_tile_info_t(const float4* info_t, int tiles, int tile, float* mean) {
    const float4 i0 = info_t[tile], i1 = info_t[(size_t)tiles + tile], i2 = info_t[2 * (size_t)tiles + tile],
                 i3 = info_t[3 * (size_t)tiles + tile];
    TileInfo t;
    t.tmin[0] = i0.x; t.tmin[1] = i0.y; t.tmin[2] = i0.z; t.kdl = i0.w;
    t.tmax[0] = i1.x; t.tmax[1] = i1.y; t.tmax[2] = i1.z; t.tau = i1.w;
    t.ncone = i2;
    t.valid = __float_as_int(i3.x);
    *mean = i3.y;
    t.rt = i3.z;
    t.sn = i3.w;
    return t;
}

__global__ void tile_info_transpose(const float4* info, float4* info_t, int tiles) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) info_t[(size_t)k * tiles + t] = info[4 * (size_t)t + k];
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// features are coarse network inputs: fast hardware log2 / division / square root
__device__ __forceinline__ float safe_log2(float v) { return __log2f(fmaxf(v, 1e-30f)); }

__device__ __forceinline__ float fast_sqrt(float v) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}

// Radiance and antiradiance luminance of one packed record at a point p with unit normal n
// (receiver albedo folded into kdl by the caller): position q0.xyz, normal (q0.w, q1.x, q1.y),
// direction (q1.z, q1.w, wz), luminances L and A of the record's radiance and antiradiance.
__device__ __forceinline__ void record_at(float4 q0, float4 q1, float wz, float L, float A, float px, float py,
                                          float pz, float nx, float ny, float nz, float clamp2, float cos_thr,
                                          float& rad, float& ar) {
    const float dx = q0.x - px, dy = q0.y - py, dz = q0.z - pz;
    const float l2 = fmaxf(dx * dx + dy * dy + dz * dz, 1e-12f);
    const float r = rsqrtf(l2);
    const float c1 = (nx * dx + ny * dy + nz * dz) * r;
    const float c2 = -(q0.w * dx + q1.x * dy + q1.y * dz) * r;
    const float inv = __fdividef(1.0f, fmaxf(l2, clamp2));
    rad = L * fmaxf(c1, 0.0f) * fmaxf(c2, 0.0f) * inv;
    const float cw = -(q1.z * dx + q1.w * dy + wz * dz) * r;
    ar = (cw > cos_thr && c1 > 0.001f) ? A * c1 * inv : 0.0f;
}

__device__ __forceinline__ void record_at(const float4* q, float px, float py, float pz, float nx, float ny, float nz,
                                          float clamp2, float cos_thr, float& rad, float& ar) {
    const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
    record_at(q0, q1, q2.x, lum3(q2.y, q2.z, q2.w), lum3(q3.x, q3.y, q3.z), px, py, pz, nx, ny, nz, clamp2, cos_thr,
              rad, ar);
}

// The 16 features of (tile, inner node).  Every input is known at selection time: the tile's
// geometry and coarse estimate (mean), the node's bounds / cones / record (q0, q1, the direction's
// z, the luminances Ls and As) / direction statistics, the records of its two children (a
// one-level lookahead at the tile centre), its depth, and the analytic bound M against tau.
__device__ __forceinline__ void node_features(const TileInfo& t, float mean, const NodeGeom& g, float M, float4 nc,
                                              float4 wc, float4 q0, float4 q1, float wz, float Ls, float As,
                                              const float4* rec_l, const float4* rec_r, float4 ds, int depth,
                                              float clamp2, float cos_thr, float* f) {
    const float E = fmaxf(mean, 1e-30f);
    const float inv_dc = __fdividef(1.0f, fmaxf(g.dc, 1e-6f));
    const float rt = g.rs - g.rn;
    const float cx = 0.5f * (t.tmin[0] + t.tmax[0]), cy = 0.5f * (t.tmin[1] + t.tmax[1]),
                cz = 0.5f * (t.tmin[2] + t.tmax[2]);
    float nx = t.ncone.x, ny = t.ncone.y, nz = t.ncone.z;
    const float nl = nx * nx + ny * ny + nz * nz;
    if (nl > 0.0f) {
        const float s = rsqrtf(nl);
        nx *= s;
        ny *= s;
        nz *= s;
    }
    float rad, ar, radl, arl, radr, arr;
    record_at(q0, q1, wz, Ls, As, cx, cy, cz, nx, ny, nz, clamp2, cos_thr, rad, ar);
    record_at(rec_l, cx, cy, cz, nx, ny, nz, clamp2, cos_thr, radl, arl);
    record_at(rec_r, cx, cy, cz, nx, ny, nz, clamp2, cos_thr, radr, arr);
    const float s = __fdividef(t.kdl, E);
    f[0] = clampf((M > 0.0f ? safe_log2(__fdividef(M, fmaxf(t.tau, 1e-30f))) : -32.0f) * 0.125f, -4.0f, 4.0f);
    f[1] = clampf(safe_log2(Ls * s) * 0.125f, -4.0f, 4.0f);
    f[2] = clampf(safe_log2(As * s + 1e-20f) * 0.125f, -4.0f, 4.0f);
    f[3] = clampf(g.rn * inv_dc, 0.0f, 4.0f);
    f[4] = clampf(rt * inv_dc, 0.0f, 4.0f);
    f[5] = clampf(fast_sqrt(g.d2c) * inv_dc, 0.0f, 4.0f);
    f[6] = g.cos1;
    f[7] = g.cos2;
    f[8] = g.ar_ok == 1.0f ? 1.0f : 0.0f;
    f[9] = g.ar_ok > 0.0f ? 1.0f : 0.0f;
    f[10] = nc.w;
    f[11] = wc.w;
    f[12] = clampf(safe_log2(fabsf(rad - radl - radr) * s + 1e-20f) * 0.125f, -4.0f, 4.0f);
    f[13] = clampf(safe_log2(fabsf(ar - arl - arr) * s + 1e-20f) * 0.125f, -4.0f, 4.0f);
    f[14] = depth * (1.0f / 32.0f);
    // mean resultant length of the antiradiance directions, in [-1, 1]
    const float sl = fast_sqrt(ds.x * ds.x + ds.y * ds.y + ds.z * ds.z);
    f[15] = ds.w > 0.0f ? clampf(2.0f * __fdividef(sl, ds.w) - 1.0f, -1.0f, 1.0f) : -1.0f;
}

__device__ __forceinline__ void store_features(__nv_bfloat16* row, const float* f) {
    uint4 q0, q1;
    uint32_t* u0 = reinterpret_cast<uint32_t*>(&q0);
    uint32_t* u1 = reinterpret_cast<uint32_t*>(&q1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 a = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
        const __nv_bfloat162 b = __floats2bfloat162_rn(f[8 + 2 * i], f[8 + 2 * i + 1]);
        u0[i] = *reinterpret_cast<const uint32_t*>(&a);
        u1[i] = *reinterpret_cast<const uint32_t*>(&b);
    }
    reinterpret_cast<uint4*>(row)[0] = q0;
    reinterpret_cast<uint4*>(row)[1] = q1;
}

__device__ __forceinline__ int child_index(int c, int n) { return c >= 0 ? c : n - (c + 1); }

// ---------------------------------------------------------------------------------------
// learned selection
// ---------------------------------------------------------------------------------------
struct LevelArgs {
    int n;
    int tiles;
    const float4* bounds;
    const float4* records;
    const float4* dirstat;
    const float4* info;     // tile records, field-major (load_tile_info_t)
    const float4* extra;    // NodeExtra per inner node
    BoundParams bp;
    const int2* in;         // {tile, node | depth << 26}
    const int* in_count;
    int2* out;              // next level
    int* out_count;
    int capacity;           // entries per frontier
    int* work;              // chunks of kLevelThreads entries handed out
    unsigned long long* rows_scored;
    const unsigned char* weight_image;  // network, in the shared-memory layout (weight_image)
    float thr_logit;        // refine iff logit >= thr_logit
    int2* accepted;         // {tile, node}
    int* acc_count;
    int acc_capacity;
    int* tile_counts;
    float band;             // M > band * tau: refine without the network
    float clamp2, cos_thr;
    uint32_t* err;
};

constexpr int kDepthShift = 26;  // node ids < 2^26 (trees of up to 32M leaves), depth < 32

__device__ __forceinline__ int2 entry(int tile, int node, int depth) {
    return make_int2(tile, node | (min(depth, 31) << kDepthShift));
}

// A frontier entry names a tile of the frame and a node of the tree; anything else (a slot that an
// overflowing level could not fill) is skipped and reported.
__device__ __forceinline__ bool valid_entry(int2 en, int tiles, int n) {
    const int node = en.y & ((1 << kDepthShift) - 1);
    return en.x >= 0 && en.x < tiles && en.y >= 0 && node < 2 * n - 1;
}

enum Action : int { kNone = 0, kAccept = 1, kRefine = 2, kScore = 3 };

constexpr int kLevelThreads = 256;

// Accepts (tile, node) or pushes (tile, lc), (tile, rc) at depth + 1, per the thread's action;
// one atomic per CTA and kind (the two global counters are shared by every CTA of the level, so
// reservations are aggregated over the CTA's 8 warps).  The CTA's left children are written in
// thread order, then its right children in the same order: a run of entries that share a node
// (the same node for consecutive tiles) becomes two runs that share its children.  The initial
// frontier holds the root for every tile, so every level stays grouped by node, and a warp's
// loads of node data mostly touch one or two nodes.  Every thread of the CTA calls it (it holds
// barriers); se: 2 * warps + 3 shared ints, not touched by anything else.
__device__ __forceinline__ void emit(const LevelArgs& a, int* se, int action, int tile, int node, int lc, int rc,
                                     int depth) {
    constexpr int kW = kLevelThreads / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const unsigned am = __ballot_sync(0xffffffffu, action == kAccept);
    const unsigned pm = __ballot_sync(0xffffffffu, action == kRefine);
    if (lane == 0) {
        se[w] = __popc(am);
        se[kW + w] = __popc(pm);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int sa = 0, sp = 0;
        for (int i = 0; i < kW; ++i) {
            const int x = se[i], y = se[kW + i];
            se[i] = sa;
            se[kW + i] = sp;
            sa += x;
            sp += y;
        }
        const int ba = sa ? atomicAdd(a.acc_count, sa) : 0;
        const int bp = sp ? atomicAdd(a.out_count, 2 * sp) : 0;
        se[2 * kW] = ba;
        se[2 * kW + 1] = bp;
        se[2 * kW + 2] = sp;
    }
    __syncthreads();
    if (action == kAccept) {
        // unsigned: the shared counter keeps counting past the capacity and may wrap past 2^31
        const int pos = se[2 * kW] + se[w] + __popc(am & lt);
        const bool ok = (unsigned)pos < (unsigned)a.acc_capacity;
        if (ok)
            a.accepted[pos] = make_int2(tile, node);
        else
            set_error(a.err, ARC_DEVERR_CUT_OVERFLOW);
        // one per-tile count update per group of lanes with the same tile
        const unsigned grp = __match_any_sync(am, ok ? tile : -1 - lane);
        if (ok && lane == __ffs(grp) - 1) atomicAdd(&a.tile_counts[tile], __popc(grp));
    } else if (action == kRefine) {
        // every reserved slot below the capacity is written; the rest do not exist (the next level
        // reads min(count, capacity) entries)
        const int rank = se[kW + w] + __popc(pm & lt);
        const int pl = se[2 * kW + 1] + rank, pr = pl + se[2 * kW + 2];
        const bool okl = (unsigned)pl < (unsigned)a.capacity, okr = (unsigned)pr < (unsigned)a.capacity;
        if (okl) a.out[pl] = entry(tile, lc, depth + 1);
        if (okr) a.out[pr] = entry(tile, rc, depth + 1);
        if (!okl || !okr) set_error(a.err, ARC_DEVERR_CUT_OVERFLOW);
    }
}

// learned_level: 256 threads, one pair per thread per chunk, rows scored two 128-row tiles at a
// time.  Shared memory: weights and vectors (the image built by weight_image) | staged feature
// rows (512, K-major, K = 16: fewer than 256 left over plus one chunk) | hidden rows (256 x 64)
// | staged pairs {tile, node | depth}
constexpr int kLevelTiles = kLevelThreads / 128, kStageRows = 2 * kLevelThreads;
constexpr uint32_t fW = 0, fVec = mlp::kWeightBytes, fX = ((mlp::kImageBytes + 127) / 128) * 128,
                   fH = fX + kStageRows * 32, fMeta = fH + kLevelThreads * 128, kLevelSmem = fMeta + kStageRows * 8;
constexpr uint32_t kLevelTmemCols = 64 * kLevelTiles;

// BF16 core-matrix weights + FP32 vectors, once per selection
template <int ACT>
__global__ void weight_image(const float* params, unsigned char* img) {
    mlp::load_weights<ACT>(img, reinterpret_cast<float*>(img + mlp::kWeightBytes), params, threadIdx.x, blockDim.x);
}

template <int ACT>
__global__ void __launch_bounds__(kLevelThreads) learned_level(LevelArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar, wbar;
    __shared__ uint32_t tmem_base;
    __shared__ int s_chunk, s_staged;
    __shared__ int s_emit[2 * (kLevelThreads / 32) + 3];
    const int t = threadIdx.x, w = t >> 5;
    const int count = min(*a.in_count, a.capacity);
    if ((int64_t)blockIdx.x * kLevelThreads >= count) return;  // no chunk can be left for this CTA
    float* vec = reinterpret_cast<float*>(sm + fVec);
    int2* meta = reinterpret_cast<int2*>(sm + fMeta);
    if (t == 0) {
        mbar_init(&bar, 1);
        mbar_init(&wbar, 1);
        fence_mbar_init();
        mbar_arrive_expect_tx(&wbar, mlp::kImageBytes);
        bulk_g2s(sm + fW, a.weight_image, mlp::kImageBytes, &wbar);
        s_staged = 0;
    }
    for (int i = t; i < kStageRows * 2; i += kLevelThreads)  // rows past the staged ones stay finite
        reinterpret_cast<uint4*>(sm + fX)[i] = make_uint4(0, 0, 0, 0);
    if (w == 0) tc::alloc(&tmem_base, kLevelTmemCols);
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    bool ok = __syncthreads_and(mbar_wait_bounded(&wbar, 0, a.err)) != 0;
    bool mma_gave_up = false;  // a tensor-core wait gave up: its commit may still be in flight
    mlp::InferCta c{smem_u32(sm), fW, fH, sm, vec, tmem_base, &bar, 0u, a.err};
    unsigned long long scored = 0;
    // The next chunk's index and entries are fetched one chunk ahead, so that neither the work
    // counter's round trip nor the entry load sits on the chain of dependent loads of a chunk.
    if (t == 0) s_chunk = atomicAdd(a.work, 1);
    __syncthreads();
    int chunk = s_chunk;
    int2 en_next = make_int2(0, 0);
    if ((int64_t)chunk * kLevelThreads + t < count) en_next = a.in[(int64_t)chunk * kLevelThreads + t];
    while (ok) {
        // every thread has read s_chunk and s_staged before they change again
        __syncthreads();
        const int64_t first = (int64_t)chunk * kLevelThreads;
        const bool done = first >= count;
        const int64_t e = first + t;
        int next = 0;
        if (t == 0 && !done) next = atomicAdd(a.work, 1);
        int action = kNone, tile = 0, node = 0, lc = 0, rc = 0, depth = 0;
        if (!done && e < count) {
            const int2 en = en_next;
            const bool good = valid_entry(en, a.tiles, a.n);
            if (!good) set_error(a.err, en.x == -1 ? ARC_DEVERR_CUT_OVERFLOW : ARC_DEVERR_BAD_NODE);
            tile = good ? en.x : 0;
            node = good ? en.y & ((1 << kDepthShift) - 1) : 0;
            depth = good ? en.y >> kDepthShift : 0;
            action = good ? kAccept : kNone;
            if (good && node >= a.n) {
                const int k = node - a.n;
                float mean;
                const TileInfo ti = load_tile_info_t(a.info, a.tiles, tile, &mean);
                const float4 b0 = a.bounds[4 * (size_t)k], b1 = a.bounds[4 * (size_t)k + 1];
                const float4 nc = a.bounds[4 * (size_t)k + 2], wc = a.bounds[4 * (size_t)k + 3];
                const float4* rec = a.records + 4 * (size_t)node;
                const NodeExtra ne = load_node_extra(a.extra, k);
                const NodeGeom g = node_geom(ti, b0, b1, nc, wc, ne, a.bp);
                const float M = node_bound(ti, g, ne.Ls, ne.As, a.bp);
                lc = child_index(__float_as_int(b0.w), a.n);
                rc = child_index(__float_as_int(b1.w), a.n);
                if (M > ti.tau) action = M > a.band * ti.tau ? kRefine : kScore;
                if (action == kScore) {
                    float f[kFeat];
                    node_features(ti, mean, g, M, nc, wc, rec[0], rec[1], rec[2].x, ne.Ls, ne.As, a.records + 4 * (size_t)lc,
                                  a.records + 4 * (size_t)rc, a.dirstat[node], depth, a.clamp2, a.cos_thr, f);
                    // < kStageRows: fewer than kLevelThreads rows are left over from the last round.
                    // Slots in thread order within each group of converged lanes, so the staged rows
                    // (and the children they push) keep the frontier's grouping by node.
                    const unsigned sm_ = __activemask();
                    const int ldr = __ffs(sm_) - 1, ln = threadIdx.x & 31;
                    int slot = 0;
                    if (ln == ldr) slot = atomicAdd(&s_staged, __popc(sm_));
                    slot = __shfl_sync(sm_, slot, ldr) + __popc(sm_ & ((1u << ln) - 1u));
                    uint4 x0, x1;
                    x0.x = mlp::pack2(f[0], f[1]);
                    x0.y = mlp::pack2(f[2], f[3]);
                    x0.z = mlp::pack2(f[4], f[5]);
                    x0.w = mlp::pack2(f[6], f[7]);
                    x1.x = mlp::pack2(f[8], f[9]);
                    x1.y = mlp::pack2(f[10], f[11]);
                    x1.z = mlp::pack2(f[12], f[13]);
                    x1.w = mlp::pack2(f[14], f[15]);
                    *reinterpret_cast<uint4*>(sm + fX + tc::kmajor_offset(slot, 0, kFeat)) = x0;
                    *reinterpret_cast<uint4*>(sm + fX + tc::kmajor_offset(slot, 8, kFeat)) = x1;
                    meta[slot] = make_int2(tile, node | (depth << kDepthShift));
                }
            }
        }
        if (t == 0 && !done) s_chunk = next;
        // emit's barriers also order every staging of this chunk before s_staged is read
        emit(a, s_emit, action, tile, node, lc, rc, depth);
        if (!done) {
            chunk = s_chunk;
            const int64_t en = (int64_t)chunk * kLevelThreads + t;
            if (en < count) en_next = a.in[en];
        }
        int staged = s_staged;
        // score full tiles now, and whatever is left once the level is exhausted
        while (staged >= kLevelThreads || (done && staged > 0)) {
            const int n_rows = min(staged, kLevelThreads);
            // the children of every staged (inner) node are fetched while the network runs
            int2 m = make_int2(0, 0);
            int cl = 0, cr = 0;
            if (t < n_rows) {
                m = meta[t];
                const int mn = m.y & ((1 << kDepthShift) - 1);
                if (mn >= a.n) {
                    const size_t k = (size_t)(mn - a.n);
                    cl = __float_as_int(a.bounds[4 * k].w);
                    cr = __float_as_int(a.bounds[4 * k + 1].w);
                }
            }
            float y = 0.0f;
            if (!mlp::infer_tiles<kLevelTiles, ACT>(c, fX, t, &y)) {
                ok = false;
                mma_gave_up = true;
                break;
            }
            scored += n_rows;
            const int act = t < n_rows ? (y >= a.thr_logit ? kRefine : kAccept) : kNone;
            const int mnode = m.y & ((1 << kDepthShift) - 1), mdepth = m.y >> kDepthShift;
            const int mlc = child_index(cl, a.n), mrc = child_index(cr, a.n);
            // after emit's barriers every thread has read its pair: the rows can be moved
            emit(a, s_emit, act, m.x, mnode, mlc, mrc, mdepth);
            const int rest = staged - n_rows;
            if (t < rest) {
                const int r = kLevelThreads + t;
                *reinterpret_cast<uint4*>(sm + fX + tc::kmajor_offset(t, 0, kFeat)) =
                    *reinterpret_cast<const uint4*>(sm + fX + tc::kmajor_offset(r, 0, kFeat));
                *reinterpret_cast<uint4*>(sm + fX + tc::kmajor_offset(t, 8, kFeat)) =
                    *reinterpret_cast<const uint4*>(sm + fX + tc::kmajor_offset(r, 8, kFeat));
                meta[t] = meta[r];
            }
            if (t == 0) s_staged = rest;
            // the next round's first barrier (in infer_tiles) or the next chunk's orders these moves
            staged = rest;
        }
        if (!ok || done) break;
    }
    if (t == 0 && scored) atomicAdd(a.rows_scored, scored);
    if (!ok && t == 0) {
        // a bounded wait gave up (the error word says so): before this CTA's shared memory and
        // TMEM are released, give its weight copy and its last tensor-core commit a second
        // bounded wait (the failed wait has already flipped the phase)
        mbar_wait_bounded(&wbar, 0, a.err);
        if (mma_gave_up) mbar_wait_bounded(&bar, c.phase ^ 1u, a.err);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (w == 0) tc::dealloc(tmem_base, kLevelTmemCols);
}

// Past the last level the host runs: every pair still in the frontier is accepted.
__global__ void accept_frontier(LevelArgs a) {
    const int count = min(*a.in_count, a.capacity);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        const int2 en = a.in[e];
        if (!valid_entry(en, a.tiles, a.n)) {
            set_error(a.err, en.x == -1 ? ARC_DEVERR_CUT_OVERFLOW : ARC_DEVERR_BAD_NODE);
            continue;
        }
        const int pos = atomicAdd(a.acc_count, 1);
        if ((unsigned)pos < (unsigned)a.acc_capacity) {
            a.accepted[pos] = make_int2(en.x, en.y & ((1 << kDepthShift) - 1));
            atomicAdd(&a.tile_counts[en.x], 1);
        } else {
            set_error(a.err, ARC_DEVERR_CUT_OVERFLOW);
        }
    }
}

__global__ void init_frontier(int2* fr, int* count, const float4* info, int tiles, int root) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles) return;
    if (__float_as_int(info[4 * (size_t)t + 3].x) == 0) return;  // no valid pixel
    const int pos = atomicAdd(count, 1);
    fr[pos] = entry(t, root, 0);
}

// exclusive scan of per-tile chunk counts (single block) -> chunk base per tile, total chunks
__global__ void tile_chunk_scan(const int* counts, int tiles, int* base, int* total, int max_chunks, uint32_t* err) {
    __shared__ int carry;
    __shared__ int warp_sums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int start = 0; start < tiles; start += blockDim.x) {
        const int t = start + threadIdx.x;
        int c = 0;
        if (t < tiles) {
            c = (counts[t] + kChunk - 1) / kChunk;
            if (c > max_chunks) {
                set_error(err, ARC_DEVERR_CUT_OVERFLOW);
                c = max_chunks;
            }
        }
        // block exclusive scan
        int v = c;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        if (lane == 31) warp_sums[w] = v;
        __syncthreads();
        if (w == 0) {
            int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += u;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        const int excl = carry + (w > 0 ? warp_sums[w - 1] : 0) + v - c;
        if (t < tiles) base[t] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + c;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

struct ScatterArgs {
    const int2* accepted;
    const int* acc_count;
    int acc_capacity;
    const int* tile_counts;
    const int* chunk_base;
    int* fill;
    CutPool pool;
    const int* total_chunks;
    uint32_t* err;
};

__global__ void scatter_tables(ScatterArgs s, int tiles) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles) return;
    const int total = *s.total_chunks;
    int c = (s.tile_counts[t] + kChunk - 1) / kChunk;
    c = min(c, s.pool.max_chunks);
    int cnt = min(s.tile_counts[t], c * kChunk);
    for (int j = 0; j < c; ++j) {
        const int id = s.chunk_base[t] + j;
        if (id < s.pool.num_chunks && id < total) s.pool.tables[(size_t)t * s.pool.max_chunks + j] = id;
        if (id >= s.pool.num_chunks) {
            set_error(s.err, ARC_DEVERR_CUT_OVERFLOW);
            cnt = min(cnt, j * kChunk);
        }
    }
    s.pool.counts[t] = cnt;
}

// Each thread takes kScatterIlp pairs per trip (a warp reads 32 consecutive pairs for each), and
// all their loads, then all their slot reservations, are issued before any result is used, so
// that several global atomics per thread are in flight.  (blockDim a multiple of 32: every lane
// of a warp takes the same loop trips.)
constexpr int kScatterIlp = 4;

__global__ void scatter_nodes(ScatterArgs s) {
    // every reserved slot below the capacity was written; the counter may have wrapped past 2^31
    const int count = (int)min((unsigned)*s.acc_count, (unsigned)s.acc_capacity);
    const int lane = threadIdx.x & 31;
    const int64_t trip = (int64_t)blockDim.x * kScatterIlp;
    for (int64_t b = (int64_t)blockIdx.x * trip; b < count; b += (int64_t)gridDim.x * trip) {
        int2 p[kScatterIlp];
        bool valid[kScatterIlp];
#pragma unroll
        for (int u = 0; u < kScatterIlp; ++u) {
            const int64_t e = b + (int64_t)u * blockDim.x + threadIdx.x;
            valid[u] = e < count;
            p[u] = valid[u] ? s.accepted[e] : make_int2(-1 - lane, 0);
        }
        // lanes with the same tile take consecutive slots with one atomic
        unsigned grp[kScatterIlp];
        int base[kScatterIlp];
#pragma unroll
        for (int u = 0; u < kScatterIlp; ++u) {
            grp[u] = __match_any_sync(0xffffffffu, p[u].x);
            base[u] = 0;
            if (valid[u] && lane == __ffs(grp[u]) - 1) base[u] = atomicAdd(&s.fill[p[u].x], __popc(grp[u]));
        }
#pragma unroll
        for (int u = 0; u < kScatterIlp; ++u) {
            base[u] = __shfl_sync(0xffffffffu, base[u], __ffs(grp[u]) - 1);
            if (!valid[u]) continue;
            const int pos = base[u] + __popc(grp[u] & ((1u << lane) - 1u));
            const int id = s.chunk_base[p[u].x] + pos / kChunk;
            if (pos / kChunk < s.pool.max_chunks && id < s.pool.num_chunks && pos < s.pool.counts[p[u].x])
                s.pool.entries[(size_t)id * kChunk + pos % kChunk] = p[u].y;
        }
    }
}

// ---------------------------------------------------------------------------------------
// training samples
// ---------------------------------------------------------------------------------------
struct LabelArgs {
    const float4* gpos;
    const float4* gnrm;
    int64_t gpitch;
    int width, height;
    const MaterialRecord* mats;
    int num_mats;
    int n;
    const float4* bounds;
    const float4* records;
    const float4* dirstat;
    const float4* info;
    const float4* extra;
    BoundParams bp;
    PairConsts pc;
    float disk_scale;
    int ar_kind;
    int tiles_x;
    int tile0, batch;
    double* prefix;  // [batch][n + 1][64]
    float delta;
    float band;
    __nv_bfloat16* feats;
    float* labels;
    float* errs;
    int* keys;  // optional: (tile, node) of each sample
    int* count;
    int capacity;
    uint32_t* err;
};

__device__ __forceinline__ void pixel_of(const LabelArgs& a, int tile, int p, int& x, int& y) {
    x = (tile % a.tiles_x) * kTile + p % kTile;
    y = (tile / a.tiles_x) * kTile + p / kTile;
}

// luminance of one record's signed contribution at a pixel (receiver albedo applied)
template <int AR>
__device__ __forceinline__ float record_lum(const float4* rec, const Pixel<float>& px, const float* kd,
                                            const PairConsts& pc, float disk_scale) {
    float4 q3 = rec[3];
    if (AR == ARC_AR_DISK) {
        const float ww = rec[1].z * rec[1].z + rec[1].w * rec[1].w + rec[2].x * rec[2].x;
        q3.w = ww > 0.0f ? rsqrtf(ww) : 0.0f;
    }
    float g, ga;
    pair_terms<AR, float>(rec[0], rec[1], rec[2], q3, px, pc, g, ga);
    const float as = AR == ARC_AR_DISK ? disk_scale : 1.0f;
    const float c0 = kd[0] * (rec[2].y * g - as * q3.x * ga), c1 = kd[1] * (rec[2].z * g - as * q3.y * ga),
                c2 = kd[2] * (rec[2].w * g - as * q3.z * ga);
    return 0.2126f * c0 + 0.7152f * c1 + 0.0722f * c2;
}

__device__ __forceinline__ bool load_pixel(const LabelArgs& a, int tile, int p, Pixel<float>& px, float* kd) {
    int x, y;
    pixel_of(a, tile, p, x, y);
    px.px = px.py = px.pz = px.nx = px.ny = px.nz = 0.0f;
    kd[0] = kd[1] = kd[2] = 0.0f;
    if (x >= a.width || y >= a.height) return false;
    const float4 gp = a.gpos[(int64_t)y * a.gpitch + x], gn = a.gnrm[(int64_t)y * a.gpitch + x];
    const int m = (int)gn.w;
    if (m <= 0 || m >= a.num_mats) return false;
    const float l = rsqrtf(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z);
    px.px = gp.x;
    px.py = gp.y;
    px.pz = gp.z;
    px.nx = gn.x * l;
    px.ny = gn.y * l;
    px.nz = gn.z * l;
    const float4 d = a.mats[m].diffuse_exp;
    kd[0] = kOneOverPi * d.x;
    kd[1] = kOneOverPi * d.y;
    kd[2] = kOneOverPi * d.z;
    return true;
}

// The prefix sums are built in segments of seg_len leaves so that every (tile, segment) pair is
// its own CTA: label_segment_sums totals each segment, label_segment_scan turns the totals into
// each segment's starting value (per tile and pixel, in segment order), and label_prefix writes
// the running sums from there.
template <int AR>
__global__ void __launch_bounds__(64) label_segment_sums(LabelArgs a, int seg_len, double* seg) {
    const int b = blockIdx.x, s = blockIdx.y, p = threadIdx.x;
    Pixel<float> px;
    float kd[3];
    const bool valid = load_pixel(a, a.tile0 + b, p, px, kd);
    double run = 0.0;
    const int i1 = min(a.n, (s + 1) * seg_len);
    if (valid)
        for (int i = s * seg_len; i < i1; ++i)
            run += (double)record_lum<AR>(a.records + 4 * (size_t)i, px, kd, a.pc, a.disk_scale);
    seg[((size_t)b * gridDim.y + s) * 64 + p] = run;
}

__global__ void label_segment_scan(double* seg, int nseg) {
    const int b = blockIdx.x, p = threadIdx.x;
    double run = 0.0;
    for (int s = 0; s < nseg; ++s) {
        double* v = seg + ((size_t)b * nseg + s) * 64 + p;
        const double t = *v;
        *v = run;
        run += t;
    }
}

template <int AR>
__global__ void __launch_bounds__(64) label_prefix(LabelArgs a, int seg_len, const double* seg) {
    const int b = blockIdx.x, s = blockIdx.y, p = threadIdx.x;
    Pixel<float> px;
    float kd[3];
    const bool valid = load_pixel(a, a.tile0 + b, p, px, kd);
    double* P = a.prefix + (size_t)b * (a.n + 1) * 64;
    double run = seg[((size_t)b * gridDim.y + s) * 64 + p];
    if (s == 0) P[p] = 0.0;
    const int i1 = min(a.n, (s + 1) * seg_len);
    for (int i = s * seg_len; i < i1; ++i) {
        if (valid) run += (double)record_lum<AR>(a.records + 4 * (size_t)i, px, kd, a.pc, a.disk_scale);
        P[(size_t)(i + 1) * 64 + p] = run;
    }
}

template <int AR>
__global__ void __launch_bounds__(32) label_traverse(LabelArgs a, const int* ranges) {
    const int b = blockIdx.x, lane = threadIdx.x;
    const int tile = a.tile0 + b;
    float mean;
    const TileInfo t = load_tile_info(a.info, tile, &mean);
    if (t.valid == 0) return;
    const double* P = a.prefix + (size_t)b * (a.n + 1) * 64;
    Pixel<float> px[2];
    float kd[2][3];
    bool valid[2];
    for (int h = 0; h < 2; ++h) valid[h] = load_pixel(a, tile, lane + 32 * h, px[h], kd[h]);
    // exact tile scale: mean |T_p| over the valid pixels
    float s = 0.0f, nv = 0.0f;
    for (int h = 0; h < 2; ++h)
        if (valid[h]) {
            s += fabsf((float)P[(size_t)a.n * 64 + lane + 32 * h]);
            nv += 1.0f;
        }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        nv += __shfl_xor_sync(0xffffffffu, nv, o);
    }
    const float Eexact = nv > 0.0f ? s / nv : 0.0f;
    const float thr = a.delta * Eexact;
    // DFS with one node per step: stack entries node | (depth << 24) with bit 31 = "extra"
    int stack[128];
    int sp = 0;
    stack[sp++] = a.n;
    int budget = 4 * a.n;
    while (sp > 0 && --budget > 0) {
        const int e = stack[--sp];
        const bool extra = e < 0;
        const int node = (e & 0x7fffffff) & 0x00ffffff;
        const int depth = ((e & 0x7fffffff) >> 24) & 0x7f;
        if (node < a.n) continue;
        const int k = node - a.n;
        const float4 b0 = a.bounds[4 * (size_t)k], b1 = a.bounds[4 * (size_t)k + 1];
        const float4 nc = a.bounds[4 * (size_t)k + 2], wc = a.bounds[4 * (size_t)k + 3];
        const float4* rec = a.records + 4 * (size_t)node;
        const NodeExtra ne = load_node_extra(a.extra, k);
        const NodeGeom g = node_geom(t, b0, b1, nc, wc, ne, a.bp);
        const float M = node_bound(t, g, ne.Ls, ne.As, a.bp);
        if (!(M > t.tau)) continue;  // the analytic bound accepts it: no decision to learn
        const int c0 = child_index(__float_as_int(b0.w), a.n), c1 = child_index(__float_as_int(b1.w), a.n);
        const int d1 = min(depth + 1, 127) << 24;
        if (M > a.band * t.tau) {  // outside the network's band: selection always refines it
            if (!extra) {
                if (sp + 2 > 128) {
                    set_error(a.err, ARC_DEVERR_STACK_OVERFLOW);
                    break;
                }
                stack[sp++] = c1 | d1;
                stack[sp++] = c0 | d1;
            }
            continue;
        }
        // RMS over the tile's valid pixels of |exact node contribution - node estimate|
        const int f0 = ranges[2 * k], l0 = ranges[2 * k + 1];
        float e2 = 0.0f;
        for (int h = 0; h < 2; ++h) {
            if (!valid[h]) continue;
            const int p = lane + 32 * h;
            const float exact = (float)(P[(size_t)(l0 + 1) * 64 + p] - P[(size_t)f0 * 64 + p]);
            const float approx = record_lum<AR>(rec, px[h], kd[h], a.pc, a.disk_scale);
            e2 += (exact - approx) * (exact - approx);
        }
        for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
        const float erms = sqrtf(e2 / fmaxf(nv, 1.0f));
        const bool refine = erms > thr;
        if (lane == 0) {
            const int r = atomicAdd(a.count, 1);
            if (r < a.capacity) {
                float f[kFeat];
                node_features(t, mean, g, M, nc, wc, rec[0], rec[1], rec[2].x, ne.Ls, ne.As, a.records + 4 * (size_t)c0,
                              a.records + 4 * (size_t)c1,
                              a.dirstat[node], depth,
                              a.bp.clamp2, a.bp.cos_thr, f);
                store_features(a.feats + (size_t)r * kFeat, f);
                a.labels[r] = refine ? 1.0f : 0.0f;
                a.errs[r] = Eexact > 0.0f ? erms / Eexact : 0.0f;
                if (a.keys) {
                    a.keys[2 * (size_t)r] = tile;
                    a.keys[2 * (size_t)r + 1] = node;
                }
            }
        }
        if (extra) continue;
        if (sp + 2 > 128) {
            set_error(a.err, ARC_DEVERR_STACK_OVERFLOW);
            break;
        }
        const int flag = refine ? 0 : (int)0x80000000;  // below an accepted node: one level only
        stack[sp++] = (c1 | d1) | flag;
        stack[sp++] = (c0 | d1) | flag;
    }
}

template <typename T>
arc_status arena_get(arc_context* ctx, const char* name, size_t count, T** out) {
    return ctx->arena.get(name, sizeof(T) * (count > 0 ? count : 1), reinterpret_cast<void**>(out));
}

BoundParams bound_params(const ArcGatherParams* gp, const ArcCutParams* cp) {
    BoundParams bp;
    bp.clamp2 = gp->dist_clamp > 0.0f ? gp->dist_clamp * gp->dist_clamp : 0.0f;
    bp.ar_kind = gp->ar_kind;
    bp.eps_cone = 0.001f;
    bp.cos_thr = fmaxf(cosf(gp->cone_half_angle), 0.001f);
    bp.disk_scale = gp->disk_radius > 0.0f ? 1.0f / (kPi * gp->disk_radius * gp->disk_radius) : 0.0f;
    bp.ar_uncertain = cp->ar_uncertain_factor;
    return bp;
}

}  // namespace

arc_status launch_cut_select_learned(arc_context* ctx, const arc_lbvh* bvh, const ArcGatherParams* gp,
                                     const ArcCutParams* cp, const float4* info, const float4* extra, int tiles_x,
                                     int tiles_y, const CutPool& pool) {
    cudaStream_t st = ctx->stream;
    const int tiles = tiles_x * tiles_y;
    const int n = bvh->n;
    // capacities: frontier / rows per level and accepted pairs over the whole walk
    ARC_CHECK_ARG(2 * n - 1 < (1 << 26), "learned cut supports trees of up to 2^25 leaves");
    // frontier capacity per level
    const int cap = (int)std::min<int64_t>((int64_t)tiles * 16384 + (1 << 20), 1 << 30);
    const int acc_cap = (int)std::min<int64_t>((int64_t)pool.num_chunks * kChunk, (int64_t)INT32_MAX);
    int2 *fa, *fb;
    int2* accepted;
    int *counters, *tile_counts, *chunk_base, *fill;
    ARC_TRY(arena_get(ctx, "lc_front_a", cap, &fa));
    ARC_TRY(arena_get(ctx, "lc_front_b", cap, &fb));
    ARC_TRY(arena_get(ctx, "lc_accepted", acc_cap, &accepted));
    // counters: [3] accepted, [4] total chunks, then per level l at 8 + 4 l: [0] entries, [2] work
    constexpr int kMaxLevels = 96;
    constexpr int kSlots = 8 + 4 * (kMaxLevels + 1);
    ARC_TRY(arena_get(ctx, "lc_counters", kSlots, &counters));
    ARC_TRY(arena_get(ctx, "lc_tile_counts", tiles, &tile_counts));
    ARC_TRY(arena_get(ctx, "lc_chunk_base", tiles, &chunk_base));
    ARC_TRY(arena_get(ctx, "lc_fill", tiles, &fill));
    ARC_TRY_CUDA(cudaMemsetAsync(counters, 0, sizeof(int) * kSlots, st));
    ARC_TRY_CUDA(cudaMemsetAsync(tile_counts, 0, sizeof(int) * tiles, st));
    ARC_TRY_CUDA(cudaMemsetAsync(fill, 0, sizeof(int) * tiles, st));

    const float p = cp->mlp_threshold;
    LevelArgs la{};
    la.n = n;
    la.tiles = tiles;
    la.bounds = reinterpret_cast<const float4*>(bvh->view.bounds);
    la.records = reinterpret_cast<const float4*>(bvh->view.records);
    la.dirstat = reinterpret_cast<const float4*>(bvh->view.dirstat);
    float4* info_t;
    ARC_TRY(arena_get(ctx, "lc_info_t", 4 * (size_t)tiles, &info_t));
    la.info = info_t;
    la.extra = extra;
    la.bp = bound_params(gp, cp);
    la.capacity = cap;
    la.rows_scored = ctx->d_learned_rows;
    unsigned char* img;
    ARC_TRY(arena_get(ctx, "lc_weight_image", mlp::kImageBytes, &img));
    la.weight_image = img;
    if (mlp_loss_kind(cp->model) == ARC_MLP_LOSS_SQUARED)  // output: log2 of the relative node error
        la.thr_logit = p <= 0.0f ? -INFINITY : log2f(p);
    else  // output: logit of the refine probability
        la.thr_logit = p <= 0.0f ? -INFINITY : (p >= 1.0f ? INFINITY : logf(p / (1.0f - p)));
    la.accepted = accepted;
    la.acc_count = counters + 3;
    la.acc_capacity = acc_cap;
    la.tile_counts = tile_counts;
    la.band = cp->mlp_band > 0.0f ? cp->mlp_band : INFINITY;
    la.clamp2 = gp->dist_clamp > 0.0f ? gp->dist_clamp * gp->dist_clamp : 0.0f;
    la.cos_thr = fmaxf(cosf(gp->cone_half_angle), 0.001f);
    la.err = ctx->d_error;

    // resident CTAs per SM, from shared memory (the runtime's occupancy query assumes a smaller
    // shared-memory carve-out than the launch gets) and TMEM (kLevelTmemCols of 512 columns each)
    int smem_sm = 0;
    ARC_TRY_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
    // (1 KB per CTA reserved by the system, plus the kernel's static shared variables)
    const int per_sm = std::max(1, std::min(512 / (int)kLevelTmemCols, smem_sm / (int)(kLevelSmem + 1280)));
    const bool relu = mlp_activation(cp->model) == ARC_MLP_ACT_RELU;
    auto* level_kernel = relu ? learned_level<mlp::kActRelu> : learned_level<mlp::kActGelu>;
    ARC_TRY_CUDA(cudaFuncSetAttribute(level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLevelSmem));
    ARC_TRY_CUDA(cudaFuncSetAttribute(level_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
    stage_begin(ctx, "cut_learned");
    int kernels = 0;
    const int grid = ctx->sm_count * 8;
    if (relu)
        weight_image<mlp::kActRelu><<<1, 256, 0, st>>>(mlp_params(cp->model), img);
    else
        weight_image<mlp::kActGelu><<<1, 256, 0, st>>>(mlp_params(cp->model), img);
    init_frontier<<<(tiles + 255) / 256, 256, 0, st>>>(fa, counters + 8, info, tiles, n);
    tile_info_transpose<<<(tiles + 255) / 256, 256, 0, st>>>(info, info_t, tiles);
    kernels += 3;
    int2 *cur = fa, *nxt = fb;
    // Every level up to kMaxLevels is launched without reading anything back: a launch past the
    // tree's last level finds an empty frontier and returns at once, so the selection holds no
    // host synchronisation and can be recorded into a CUDA graph.  Pairs still in the frontier
    // after the last launch (a tree deeper than kMaxLevels) are accepted.
    for (int level = 0; level < kMaxLevels; ++level) {
        la.in = cur;
        la.in_count = counters + 8 + 4 * level;
        la.work = counters + 8 + 4 * level + 2;
        la.out = nxt;
        la.out_count = counters + 8 + 4 * (level + 1);
        level_kernel<<<ctx->sm_count * per_sm, kLevelThreads, kLevelSmem, st>>>(la);
        ++kernels;
        std::swap(cur, nxt);
    }
    la.in = cur;
    la.in_count = counters + 8 + 4 * kMaxLevels;
    accept_frontier<<<grid, 256, 0, st>>>(la);
    ++kernels;
    stage_end(ctx, kernels);
    // the accepted pairs grouped by tile into the cut pool, timed as a stage of its own
    stage_begin(ctx, "cut_lists");
    kernels = 0;
    ScatterArgs sa;
    sa.accepted = accepted;
    sa.acc_count = counters + 3;
    sa.acc_capacity = acc_cap;
    sa.tile_counts = tile_counts;
    sa.chunk_base = chunk_base;
    sa.fill = fill;
    sa.pool = pool;
    sa.total_chunks = counters + 4;
    sa.err = ctx->d_error;
    tile_chunk_scan<<<1, 1024, 0, st>>>(tile_counts, tiles, chunk_base, counters + 4, pool.max_chunks, ctx->d_error);
    scatter_tables<<<(tiles + 255) / 256, 256, 0, st>>>(sa, tiles);
    scatter_nodes<<<grid, 256, 0, st>>>(sa);
    kernels += 3;
    ARC_TRY_CUDA(cudaMemcpyAsync(pool.next, counters + 4, sizeof(int), cudaMemcpyDeviceToDevice, st));
    stage_end(ctx, kernels);
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

}  // namespace arc

using namespace arc;

// Training samples of the learned cut (see the file comment).  No counterpart in the reference.
extern "C" arc_status arc_cut_training_samples(arc_context* ctx, const arc_lbvh* bvh, const ArcGBufferView* gb,
                                               ArcFloat3 camera_position, const ArcGatherParams* gp,
                                               const ArcCutParams* cp, float delta, void* features_bf16,
                                               float* labels, float* errors, int32_t* keys, int32_t capacity,
                                               int32_t* count) {
    ARC_CHECK_ARG(ctx && bvh && gb && gp && cp && features_bf16 && labels && errors && count, "NULL argument");
    ARC_CHECK_ARG(bvh->n >= 2, "LBVH not built");
    ARC_CHECK_ARG(gp->ar_kind >= 0 && gp->ar_kind <= 2, "ar_kind out of range");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    (void)camera_position;
    cudaStream_t st = ctx->stream;
    const int W = gb->width, H = gb->height;
    const int tiles_x = (W + kTile - 1) / kTile, tiles = tiles_x * ((H + kTile - 1) / kTile);
    const int n = bvh->n;
    float4* info = nullptr;
    float4* extra = nullptr;
    ARC_TRY(launch_tile_setup(ctx, bvh, gb, gp, cp, &info, &extra));
    // batch of tiles whose FP64 prefixes fit in ~8 GB
    const size_t per_tile = (size_t)(n + 1) * 64 * sizeof(double);
    const int batch = (int)std::max<size_t>(1, std::min<size_t>((size_t)tiles, ((size_t)8 << 30) / per_tile));
    const int seg_len = 4096, nseg = (n + seg_len - 1) / seg_len;
    double* seg = nullptr;
    ARC_TRY(ctx->arena.get("label_segments", (size_t)batch * nseg * 64 * sizeof(double),
                           reinterpret_cast<void**>(&seg)));
    double* prefix = nullptr;
    ARC_TRY(ctx->arena.get("label_prefix", per_tile * batch, reinterpret_cast<void**>(&prefix)));
    int* dcount = nullptr;
    ARC_TRY(ctx->arena.get("label_count", sizeof(int), reinterpret_cast<void**>(&dcount)));
    ARC_TRY_CUDA(cudaMemsetAsync(dcount, 0, sizeof(int), st));
    LabelArgs a{};
    a.gpos = reinterpret_cast<const float4*>(gb->position);
    a.gnrm = reinterpret_cast<const float4*>(gb->normal);
    a.gpitch = gb->pitch;
    a.width = W;
    a.height = H;
    a.mats = ctx->d_materials;
    a.num_mats = ctx->num_materials;
    a.n = n;
    a.bounds = reinterpret_cast<const float4*>(bvh->view.bounds);
    a.records = reinterpret_cast<const float4*>(bvh->view.records);
    a.dirstat = reinterpret_cast<const float4*>(bvh->view.dirstat);
    a.info = info;
    a.extra = extra;
    a.bp = bound_params(gp, cp);
    a.pc.cos_thr = fmaxf(cosf(gp->cone_half_angle), 0.001f);
    a.pc.eps = 0.001f;
    a.pc.inv_clamp2 = gp->dist_clamp > 0.0f ? 1.0f / (gp->dist_clamp * gp->dist_clamp) : INFINITY;
    a.pc.disk_r2 = gp->disk_radius * gp->disk_radius;
    a.disk_scale = gp->disk_radius > 0.0f ? 1.0f / (kPi * gp->disk_radius * gp->disk_radius) : 0.0f;
    a.ar_kind = gp->ar_kind;
    a.tiles_x = tiles_x;
    a.prefix = prefix;
    a.delta = delta;
    a.band = cp->mlp_band > 0.0f ? cp->mlp_band : INFINITY;
    a.feats = static_cast<__nv_bfloat16*>(features_bf16);
    a.labels = labels;
    a.errs = errors;
    a.keys = keys;
    a.count = dcount;
    a.capacity = capacity;
    a.err = ctx->d_error;
    for (int t0 = 0; t0 < tiles; t0 += batch) {
        a.tile0 = t0;
        a.batch = std::min(batch, tiles - t0);
        const dim3 g2(a.batch, nseg);
        switch (gp->ar_kind) {
            case 0:
                label_segment_sums<0><<<g2, 64, 0, st>>>(a, seg_len, seg);
                label_segment_scan<<<a.batch, 64, 0, st>>>(seg, nseg);
                label_prefix<0><<<g2, 64, 0, st>>>(a, seg_len, seg);
                label_traverse<0><<<a.batch, 32, 0, st>>>(a, bvh->view.range);
                break;
            case 1:
                label_segment_sums<1><<<g2, 64, 0, st>>>(a, seg_len, seg);
                label_segment_scan<<<a.batch, 64, 0, st>>>(seg, nseg);
                label_prefix<1><<<g2, 64, 0, st>>>(a, seg_len, seg);
                label_traverse<1><<<a.batch, 32, 0, st>>>(a, bvh->view.range);
                break;
            default:
                label_segment_sums<2><<<g2, 64, 0, st>>>(a, seg_len, seg);
                label_segment_scan<<<a.batch, 64, 0, st>>>(seg, nseg);
                label_prefix<2><<<g2, 64, 0, st>>>(a, seg_len, seg);
                label_traverse<2><<<a.batch, 32, 0, st>>>(a, bvh->view.range);
                break;
        }
        ARC_TRY_CUDA(cudaGetLastError());
    }
    int h = 0;
    ARC_TRY_CUDA(cudaMemcpyAsync(&h, dcount, sizeof(int), cudaMemcpyDeviceToHost, st));
    ARC_TRY_CUDA(cudaStreamSynchronize(st));
    *count = std::min(h, capacity);
    return ARC_OK;
}
