// Clustered deferred antiradiance (scope rows a21-a23), the reference's accelerator for the disk
// antiradiance:
//   cluster_tiles    screen clusters (VisiblePointsBvh, bvh.cu:986-1179): 16 x 16 pixel tiles split
//                    by exponential depth slice k = floor(log(d / zNear) / log(1 + 2 tan(theta) / 16))
//                    (kernel_initBuffers, bvh.cu:986-1018), one cluster per (tile, k) with the
//                    bounding box of its pixels.  The reference's key k + tile * max_k collides
//                    across tiles (it needs max_k + 1) and its clusters take in background pixels
//                    at the origin; here a cluster is exactly a (tile, k) pair of surface pixels,
//                    found by a sort within the tile's block (no global sort), in slot
//                    tile * 256 + rank of k within the tile.
//   cluster_lights   per cluster, the AVPLs whose ray p_a + t w_a (t >= 0) meets the cluster box
//                    grown by twice the disk radius (kernel_gather_cluster_lights and intersectBB,
//                    cudaGather.cu:663-748), in AVPL order: a counting pass, a scan over the slots,
//                    and a writing pass, instead of the reference's num_clusters x num_avpls array.
//   clustered_ar     per pixel, the disk antiradiance of its cluster's AVPLs
//                    (kernel_antiradiance_clusterred, cudaGather.cu:605-659) with the brute-force
//                    gather's terms (pair_math.cuh) and Kahan sums.  A contributing AVPL's ray passes
//                    within the disk radius of the pixel, so it is in the list: the result is the
//                    brute-force disk antiradiance up to the order of the sum.
#include <cfloat>
#include <climits>

#include "arc_internal.h"
#include "device_common.cuh"
#include "pair_math.cuh"
#include "scan.cuh"

namespace arc {
namespace {

constexpr int kCT = 16;               // tile edge
constexpr int kCThreads = kCT * kCT;  // one thread per pixel of a tile; also cluster slots per tile

__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

struct TileArgsC {
    const float4* gpos;
    const float4* gnrm;
    int64_t gpitch;
    int width, height, tiles_x;
    float3 cam;
    float inv_z_near;
    float inv_log_step;  // 1 / log(1 + 2 tan(theta) / 16)
    int* pixel_cluster;  // [height * width]: slot, or -1 (no surface)
    float4* box;         // [slots][2]: {min, 0}, {max, 0}
    int* tile_count;     // clusters per tile
};

__global__ void __launch_bounds__(kCThreads) cluster_tiles(TileArgsC a) {
    __shared__ int key[kCThreads];
    __shared__ int who[kCThreads];
    __shared__ float sp[3][kCThreads];
    __shared__ uint32_t bmin[3][kCThreads], bmax[3][kCThreads];
    __shared__ int warp_flags[kCThreads / 32];
    const int tile = blockIdx.x, t = threadIdx.x;
    const int x = (tile % a.tiles_x) * kCT + t % kCT, y = (tile / a.tiles_x) * kCT + t / kCT;
    const bool inside = x < a.width && y < a.height;
    bool surface = false;
    float4 p = make_float4(0, 0, 0, 0);
    if (inside) {
        p = a.gpos[(int64_t)y * a.gpitch + x];
        surface = a.gnrm[(int64_t)y * a.gpitch + x].w > 0.0f;
    }
    int k = INT_MAX;  // no surface: sorts last, no cluster
    if (surface) {
        const float dx = a.cam.x - p.x, dy = a.cam.y - p.y, dz = a.cam.z - p.z;
        const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
        const float kf = floorf(logf(dist * a.inv_z_near) * a.inv_log_step);
        k = (int)fminf(fmaxf(kf, -1048576.0f), 1048576.0f);
    }
    key[t] = k;
    who[t] = t;
    sp[0][t] = p.x;
    sp[1][t] = p.y;
    sp[2][t] = p.z;
    bmin[0][t] = bmin[1][t] = bmin[2][t] = ordered(FLT_MAX);
    bmax[0][t] = bmax[1][t] = bmax[2][t] = ordered(-FLT_MAX);
    __syncthreads();
    // bitonic sort of (key, pixel) over the tile
    for (int size = 2; size <= kCThreads; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const int j = t ^ stride;
            if (j > t) {
                const bool up = (t & size) == 0;
                const int ka = key[t], kb = key[j];
                if ((ka > kb) == up && ka != kb) {
                    key[t] = kb;
                    key[j] = ka;
                    const int w = who[t];
                    who[t] = who[j];
                    who[j] = w;
                }
            }
            __syncthreads();
        }
    }
    // cluster rank of sorted entry t: the number of distinct keys up to it
    const int kt = key[t];
    const bool first = kt != INT_MAX && (t == 0 || key[t - 1] != kt);
    const unsigned m = __ballot_sync(0xffffffffu, first);
    const int lane = t & 31, w = t >> 5;
    if (lane == 0) warp_flags[w] = __popc(m);
    __syncthreads();
    int rank = __popc(m & ((2u << lane) - 1u));  // inclusive within the warp
    int count = 0;
    for (int q = 0; q < kCThreads / 32; ++q) {
        if (q < w) rank += warp_flags[q];
        count += warp_flags[q];
    }
    const int c = rank - 1;  // cluster of sorted entry t (valid when kt != INT_MAX)
    const int pix = who[t];
    const int px = (tile % a.tiles_x) * kCT + pix % kCT, py = (tile / a.tiles_x) * kCT + pix / kCT;
    if (kt != INT_MAX) {
        for (int d = 0; d < 3; ++d) {
            atomicMin(&bmin[d][c], ordered(sp[d][pix]));
            atomicMax(&bmax[d][c], ordered(sp[d][pix]));
        }
        a.pixel_cluster[(int64_t)py * a.width + px] = tile * kCThreads + c;
    } else if (px < a.width && py < a.height) {
        a.pixel_cluster[(int64_t)py * a.width + px] = -1;
    }
    __syncthreads();
    if (t < count) {
        const int64_t s = (int64_t)tile * kCThreads + t;
        a.box[2 * s] = make_float4(unordered(bmin[0][t]), unordered(bmin[1][t]), unordered(bmin[2][t]), 0.0f);
        a.box[2 * s + 1] = make_float4(unordered(bmax[0][t]), unordered(bmax[1][t]), unordered(bmax[2][t]), 0.0f);
    }
    if (t == 0) a.tile_count[tile] = count;
}

// intersectBB (cudaGather.cu:663-684): the slab test of the ray o + t d against [lo, hi], hit
// when the exit parameter is >= 0 and not before the entry.
__device__ __forceinline__ bool ray_box(float3 lo, float3 hi, float3 o, float3 d) {
    const float fx = 1.0f / d.x, fy = 1.0f / d.y, fz = 1.0f / d.z;
    const float t1 = (lo.x - o.x) * fx, t2 = (hi.x - o.x) * fx;
    const float t3 = (lo.y - o.y) * fy, t4 = (hi.y - o.y) * fy;
    const float t5 = (lo.z - o.z) * fz, t6 = (hi.z - o.z) * fz;
    const float tmin = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
    const float tmax = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
    return !(tmax < 0.0f || tmin > tmax);
}

struct LightArgsC {
    ArcAvplsGpuParam av;
    const float4* box;
    const int* tile_count;
    float grow;             // twice the disk radius
    int* counts;            // [slots] (pass 0)
    const int* offsets;     // block-local offsets of the slots' lists (pass 1)
    const int* block_sums;  // exclusive, per scan::kScanItems slots (pass 1)
    int* lists;             // (pass 1)
    int64_t list_cap;
    uint32_t* err;
};

// One block per tile; PASS 0 counts each cluster's AVPLs, PASS 1 writes them in AVPL order.
template <int PASS>
__global__ void __launch_bounds__(kCThreads) cluster_lights(LightArgsC a) {
    __shared__ float3 lo[kCThreads], hi[kCThreads];
    __shared__ int acc[kCThreads];  // PASS 0: counts; PASS 1: entries written so far
    __shared__ int wsum[2][kCThreads / 32];
    const int tile = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int count = a.tile_count[tile];
    if (count <= 0) return;  // uniform over the block
    for (int c = t; c < count; c += kCThreads) {
        const int64_t s = (int64_t)tile * kCThreads + c;
        const float4 b0 = a.box[2 * s], b1 = a.box[2 * s + 1];
        lo[c] = make_float3(b0.x - a.grow, b0.y - a.grow, b0.z - a.grow);
        hi[c] = make_float3(b1.x + a.grow, b1.y + a.grow, b1.z + a.grow);
        acc[c] = 0;
    }
    __syncthreads();
    const int n = a.av.numAvpls;
    const unsigned lt = (1u << lane) - 1u;
    for (int base = 0; base < n; base += kCThreads) {
        const int j = base + t;
        const bool have = j < n;
        const float3 o = have ? ld3(a.av.position, j) : make_float3(0, 0, 0);
        const float3 d = have ? ld3(a.av.incDirection, j) : make_float3(0, 0, 1);
        for (int c = 0; c < count; ++c) {
            const bool hit = have && ray_box(lo[c], hi[c], o, d);
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (PASS == 0) {
                if (lane == 0 && m) atomicAdd(&acc[c], __popc(m));
            } else {
                int* ws = wsum[c & 1];
                if (lane == 0) ws[w] = __popc(m);
                __syncthreads();
                int pos = acc[c] + __popc(m & lt), tot = 0;
                for (int q = 0; q < kCThreads / 32; ++q) {
                    if (q < w) pos += ws[q];
                    tot += ws[q];
                }
                if (hit) {
                    const int64_t s = (int64_t)tile * kCThreads + c;
                    const int64_t dst = (int64_t)a.block_sums[s / scan::kScanItems] + a.offsets[s] + pos;
                    if (dst < a.list_cap)
                        a.lists[dst] = j;
                    else
                        set_error(a.err, ARC_DEVERR_CUT_OVERFLOW);
                }
                __syncthreads();  // every thread has read acc[c] and ws
                if (t == 0) acc[c] += tot;
            }
        }
    }
    if (PASS == 0) {
        __syncthreads();
        for (int c = t; c < count; c += kCThreads) a.counts[(int64_t)tile * kCThreads + c] = acc[c];
    }
}

struct ArArgsC {
    const float4* gpos;
    const float4* gnrm;
    int64_t gpitch;
    int width, height, tiles_x;
    const MaterialRecord* mats;
    int num_mats;
    const float4* records;
    int num_avpls;
    const int* pixel_cluster;
    const int* counts;
    const int* offsets;
    const int* block_sums;
    const int* lists;
    int64_t list_cap;
    PairConsts pc;
    float disk_scale;
    float4* out_ar;
    double* out_ar64;  // 3 doubles per pixel, or NULL
    int64_t opitch;
    uint32_t* err;
};

__global__ void __launch_bounds__(kCThreads) clustered_ar(ArArgsC a) {
    const int tile = blockIdx.x, t = threadIdx.x;
    const int x = (tile % a.tiles_x) * kCT + t % kCT, y = (tile / a.tiles_x) * kCT + t / kCT;
    if (x >= a.width || y >= a.height) return;
    const int cid = a.pixel_cluster[(int64_t)y * a.width + x];
    double ar[3] = {0.0, 0.0, 0.0};
    if (cid >= 0) {
        const float4 gp = a.gpos[(int64_t)y * a.gpitch + x], gn = a.gnrm[(int64_t)y * a.gpitch + x];
        int mat = (int)gn.w;
        if (mat <= 0 || mat >= a.num_mats) {
            set_error(a.err, ARC_DEVERR_BAD_MATERIAL);
            mat = 0;
        }
        Pixel<float> s;
        const float l = rsqrtf(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z);
        s.px = gp.x;
        s.py = gp.y;
        s.pz = gp.z;
        s.nx = gn.x * l;
        s.ny = gn.y * l;
        s.nz = gn.z * l;
        float sum[3] = {0, 0, 0}, comp[3] = {0, 0, 0};
        const int n = a.counts[cid];
        const int64_t off = (int64_t)a.block_sums[cid / scan::kScanItems] + a.offsets[cid];
        for (int i = 0; i < n; ++i) {
            if (off + i >= a.list_cap) break;
            const int j = a.lists[off + i];
            if ((unsigned)j >= (unsigned)a.num_avpls) {  // not an AVPL: a list the lights pass left short
                set_error(a.err, ARC_DEVERR_BAD_NODE);
                break;
            }
            const float4* q = a.records + 4 * (int64_t)j;
            const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
            float g, ga;
            pair_terms<ARC_AR_DISK, float>(q0, q1, q2, q3, s, a.pc, g, ga);
            if (ga != 0.0f) {
                kahan_add(sum[0], comp[0], q3.x * ga);
                kahan_add(sum[1], comp[1], q3.y * ga);
                kahan_add(sum[2], comp[2], q3.z * ga);
            }
        }
        if (mat > 0) {
            const float4 dif = a.mats[mat].diffuse_exp;
            const float kd[3] = {kOneOverPi * dif.x, kOneOverPi * dif.y, kOneOverPi * dif.z};
            for (int c = 0; c < 3; ++c) ar[c] = (double)kd[c] * (double)a.disk_scale * ((double)sum[c] - (double)comp[c]);
        }
    }
    const int64_t o = (int64_t)y * a.opitch + x;
    if (a.out_ar) a.out_ar[o] = make_float4((float)ar[0], (float)ar[1], (float)ar[2], 1.0f);
    if (a.out_ar64)
        for (int c = 0; c < 3; ++c) a.out_ar64[3 * o + c] = ar[c];
}

// result = radiance - antiradiance after the clustered pass: in FP64 when the caller keeps the
// FP64 result (it then holds the radiance), else in FP32 from the float result plane
__global__ void subtract_antiradiance(float4* result, double* result64, const double* ar64, int width, int height,
                                      int64_t pitch) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)width * height) return;
    const int64_t o = (int64_t)(i / width) * pitch + i % width;
    double r[3];
    for (int c = 0; c < 3; ++c) {
        const double rad = result64 ? result64[3 * o + c] : (double)(&result[o].x)[c];
        r[c] = rad - ar64[3 * o + c];
        if (result64) result64[3 * o + c] = r[c];
    }
    if (result) result[o] = make_float4((float)r[0], (float)r[1], (float)r[2], 1.0f);
}

}  // namespace

arc_status launch_run_clustered_antiradiance(arc_context* ctx, const ArcAvplsGpuParam* avpls,
                                             const ArcGBufferView* gbuffer, ArcFloat3 camera_position,
                                             const ArcClusterParams* cl, const ArcGatherParams* gp,
                                             const ArcOutputView* out) {
    const int W = gbuffer->width, H = gbuffer->height;
    double* ar64 = nullptr;
    ARC_TRY(ctx->arena.get("run_ar64", (size_t)H * out->pitch * 3 * sizeof(double), reinterpret_cast<void**>(&ar64)));
    ArcOutputView ao{nullptr, nullptr, out->antiradiance, ar64, out->pitch};
    ARC_TRY(arc_antiradiance_clustered(ctx, avpls, gbuffer, camera_position, cl, gp, &ao, nullptr));
    const int64_t px = (int64_t)W * H;
    stage_begin(ctx, "combine");
    subtract_antiradiance<<<(unsigned)((px + 255) / 256), 256, 0, ctx->stream>>>(
        reinterpret_cast<float4*>(out->result), out->result_fp64, ar64, W, H, out->pitch);
    stage_end(ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

}  // namespace arc

using namespace arc;

extern "C" arc_status arc_antiradiance_clustered(arc_context* ctx, const ArcAvplsGpuParam* avpls,
                                                 const ArcGBufferView* gbuffer, ArcFloat3 camera_position,
                                                 const ArcClusterParams* cparams, const ArcGatherParams* params,
                                                 const ArcOutputView* out, ArcClusterInfo* info) {
    ARC_CHECK_ARG(ctx && avpls && gbuffer && cparams && params && out, "NULL argument");
    ARC_CHECK_ARG(params->ar_kind == ARC_AR_DISK && params->disk_radius > 0.0f,
                  "clustered antiradiance is the disk variant (ar_kind DISK, disk_radius > 0)");
    ARC_CHECK_ARG(cparams->z_near > 0.0f && cparams->theta > 0.0f && cparams->theta < 1.5707f, "bad cluster parameters");
    ARC_CHECK_ARG(gbuffer->width > 0 && gbuffer->height > 0 && gbuffer->pitch >= gbuffer->width && gbuffer->position &&
                      gbuffer->normal,
                  "bad G-buffer view");
    ARC_CHECK_ARG(out->pitch >= gbuffer->width && (out->antiradiance || out->result_fp64), "bad output view");
    ARC_CHECK_ARG(avpls->numAvpls >= 0, "negative AVPL count");
    ARC_CHECK_ARG(ctx->num_materials > 0, "materials not uploaded");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int W = gbuffer->width, H = gbuffer->height;
    const int tiles_x = (W + kCT - 1) / kCT, tiles = tiles_x * ((H + kCT - 1) / kCT);
    const int64_t slots = (int64_t)tiles * kCThreads;
    ARC_CHECK_ARG(slots < INT32_MAX, "image too large for the cluster slots");
    int *pixel_cluster, *tile_count, *counts, *offsets, *block_sums, *total;
    float4* box;
    ARC_TRY(ctx->arena.get("cl_pixel", (size_t)W * H * sizeof(int), reinterpret_cast<void**>(&pixel_cluster)));
    ARC_TRY(ctx->arena.get("cl_tile_count", (size_t)tiles * sizeof(int), reinterpret_cast<void**>(&tile_count)));
    ARC_TRY(ctx->arena.get("cl_box", (size_t)slots * 2 * sizeof(float4), reinterpret_cast<void**>(&box)));
    ARC_TRY(ctx->arena.get("cl_counts", (size_t)slots * sizeof(int), reinterpret_cast<void**>(&counts)));
    ARC_TRY(ctx->arena.get("cl_offsets", (size_t)slots * sizeof(int), reinterpret_cast<void**>(&offsets)));
    ARC_TRY(ctx->arena.get("cl_block_sums", (size_t)(scan::num_blocks(slots) + 1) * sizeof(int),
                           reinterpret_cast<void**>(&block_sums)));
    ARC_TRY(ctx->arena.get("cl_total", sizeof(int), reinterpret_cast<void**>(&total)));

    TileArgsC ta;
    ta.gpos = reinterpret_cast<const float4*>(gbuffer->position);
    ta.gnrm = reinterpret_cast<const float4*>(gbuffer->normal);
    ta.gpitch = gbuffer->pitch;
    ta.width = W;
    ta.height = H;
    ta.tiles_x = tiles_x;
    ta.cam = make_float3(camera_position.x, camera_position.y, camera_position.z);
    ta.inv_z_near = 1.0f / cparams->z_near;
    ta.inv_log_step = 1.0f / logf(1.0f + 2.0f * tanf(cparams->theta) / (float)kCT);
    ta.pixel_cluster = pixel_cluster;
    ta.box = box;
    ta.tile_count = tile_count;
    LightArgsC la;
    la.av = *avpls;
    la.box = box;
    la.tile_count = tile_count;
    la.grow = 2.0f * params->disk_radius;
    la.counts = counts;
    la.offsets = offsets;
    la.block_sums = block_sums;
    la.err = ctx->d_error;

    stage_begin(ctx, "cluster_build");
    cluster_tiles<<<tiles, kCThreads, 0, st>>>(ta);
    ARC_TRY_CUDA(cudaMemsetAsync(counts, 0, (size_t)slots * sizeof(int), st));
    la.lists = nullptr;
    la.list_cap = 0;
    cluster_lights<0><<<tiles, kCThreads, 0, st>>>(la);
    scan::exclusive_scan(counts, slots, offsets, block_sums, total, st);
    stage_end(ctx, 4);
    ARC_TRY_CUDA(cudaGetLastError());
    int entries = 0;
    ARC_TRY_CUDA(cudaMemcpyAsync(&entries, total, sizeof(int), cudaMemcpyDeviceToHost, st));
    ARC_TRY_CUDA(cudaStreamSynchronize(st));
    if (entries < 0) {  // the int scan wrapped: more than 2^31 list entries
        set_last_error("clustered antiradiance: more than 2^31 cluster-list entries");
        return ARC_ERR_UNSUPPORTED;
    }
    int* lists = nullptr;
    ARC_TRY(ctx->arena.get("cl_lists", (size_t)(entries > 0 ? entries : 1) * sizeof(int),
                           reinterpret_cast<void**>(&lists)));
    la.lists = lists;
    la.list_cap = entries;
    const float4* records = nullptr;
    ARC_TRY(launch_pack_records(ctx, avpls, &records));
    stage_begin(ctx, "cluster_lights");
    cluster_lights<1><<<tiles, kCThreads, 0, st>>>(la);
    stage_end(ctx, 1);
    ArArgsC aa;
    aa.gpos = ta.gpos;
    aa.gnrm = ta.gnrm;
    aa.gpitch = gbuffer->pitch;
    aa.width = W;
    aa.height = H;
    aa.tiles_x = tiles_x;
    aa.mats = ctx->d_materials;
    aa.num_mats = ctx->num_materials;
    aa.records = records;
    aa.num_avpls = avpls->numAvpls;
    aa.pixel_cluster = pixel_cluster;
    aa.counts = counts;
    aa.offsets = offsets;
    aa.block_sums = block_sums;
    aa.lists = lists;
    aa.list_cap = entries;
    aa.pc.cos_thr = 0.0f;
    aa.pc.eps = 0.001f;
    aa.pc.inv_clamp2 = params->dist_clamp > 0.0f ? 1.0f / (params->dist_clamp * params->dist_clamp) : INFINITY;
    aa.pc.disk_r2 = params->disk_radius * params->disk_radius;
    aa.disk_scale = 1.0f / (kPi * params->disk_radius * params->disk_radius);
    aa.out_ar = reinterpret_cast<float4*>(out->antiradiance);
    aa.out_ar64 = out->result_fp64;
    aa.opitch = out->pitch;
    aa.err = ctx->d_error;
    stage_begin(ctx, "clustered_ar");
    clustered_ar<<<tiles, kCThreads, 0, st>>>(aa);
    stage_end(ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());
    if (info) {
        info->pixel_cluster = pixel_cluster;
        info->box = reinterpret_cast<const float*>(box);
        info->tile_count = tile_count;
        info->counts = counts;
        info->lists = lists;
        info->num_tiles = tiles;
        info->slots_per_tile = kCThreads;
        info->list_entries = entries;
    }
    return ARC_OK;
}
