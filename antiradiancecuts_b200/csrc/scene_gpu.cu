// Synthetic scenes on the GPU: the primary-ray G-buffer and the AVPL light tracer of
// scene_gen.cpp, from the same source (scene_math.h).  This file is compiled with -fmad=false, so
// every add, multiply, divide and square root rounds as on the CPU: the G-buffer is the same bits;
// the AVPLs differ only through the azimuth's cosf / sinf (and a specular lobe's powf), which the
// device library computes independently of the host's.
//
// Tracer: one thread per light path traces into a per-path slot of max_bounces AVPLs and
// records its count; a scan of the counts gives every path its output offset, and a scatter
// writes the AVPLs in path order into the caller's SoA arrays (AvplsGpuParam) until num_avpls are
// written, exactly the order of the CPU tracer.  Paths go in batches until the count is reached.
#include <algorithm>

#include "arc_internal.h"
#include "scan.cuh"
#include "scene_math.h"

namespace arc {
namespace {

using namespace scene;

// The scene and its rectangles in device memory (one copy per call).
struct SceneDev {
    ArcSceneDesc desc;
    Rect rects[kMaxRects];
    int nrects;
};

constexpr int kSceneThreads = 256;

// Stages the rectangles in shared memory; returns their count.
__device__ __forceinline__ int stage_rects(const SceneDev* sd, Rect* srect) {
    const int n = sd->nrects;
    for (int i = threadIdx.x; i < n; i += blockDim.x) srect[i] = sd->rects[i];
    __syncthreads();
    return n;
}

__global__ void __launch_bounds__(kSceneThreads) scene_gbuffer_kernel(const SceneDev* sd, Camera cam, int width,
                                                                      int height, float4* pos, float4* nrm,
                                                                      int64_t pitch) {
    __shared__ Rect srect[kMaxRects];
    const int n = stage_rects(sd, srect);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)width * height) return;
    const int x = (int)(i % width), y = (int)(i / width);
    float P[4], N[4];
    gbuffer_texel(cam, srect, n, width, height, x, y, P, N);
    pos[(int64_t)y * pitch + x] = make_float4(P[0], P[1], P[2], P[3]);
    nrm[(int64_t)y * pitch + x] = make_float4(N[0], N[1], N[2], N[3]);
}

// Paths path0 .. path0 + npaths - 1: AVPLs into slots [i * max_bounces, ...), counts[i].
__global__ void __launch_bounds__(kSceneThreads) scene_trace_kernel(const SceneDev* sd, uint64_t seed,
                                                                    int64_t path0, int npaths, int max_bounces,
                                                                    int explicit_direct, ArcAvplHost* slots,
                                                                    int* counts) {
    __shared__ Rect srect[kMaxRects];
    const int n = stage_rects(sd, srect);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npaths) return;
    ArcAvplHost* dst = slots + (size_t)i * max_bounces;
    int c = 0;
    trace_path(sd->desc, srect, n, seed, (uint64_t)(path0 + i), max_bounces, explicit_direct != 0,
               [&](const ArcAvplHost& a) {
                   if (c < max_bounces) dst[c] = a;
                   ++c;
               });
    counts[i] = min(c, max_bounces);
}

constexpr int kScanItems = scan::kScanItems;

struct ScatterArgs {
    const ArcAvplHost* slots;
    const int* counts;
    const int* offsets;     // block-local
    const int* block_sums;  // exclusive, per kScanItems block
    int npaths;
    int max_bounces;
    int64_t path0;
    int* produced;     // AVPLs written by earlier batches; advanced by this batch's total
    int64_t* paths;    // paths needed for num_avpls AVPLs (set by the batch that reaches it)
    ArcAvplsGpuParam out;
};

__global__ void __launch_bounds__(kSceneThreads) scatter_avpls(ScatterArgs s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.npaths) return;
    const int base = *s.produced;
    const int c = s.counts[i];
    const int64_t first = (int64_t)base + s.block_sums[i / kScanItems] + s.offsets[i];
    const int64_t need = s.out.numAvpls;
    for (int j = 0; j < c; ++j) {
        const int64_t d = first + j;
        if (d >= need) break;
        const ArcAvplHost& a = s.slots[(size_t)i * s.max_bounces + j];
        s.out.position[d] = a.position;
        s.out.normal[d] = a.normal;
        s.out.incDirection[d] = a.incDirection;
        s.out.incRadiance[d] = a.incRadiance;
        s.out.antiradiance[d] = a.antiradiance;
        s.out.materialIndex[d] = a.materialIndex;
        s.out.bounce[d] = a.bounce;
    }
    if (c > 0 && first < need && first + c >= need) *s.paths = s.path0 + i + 1;  // this path completes the set
}

// produced += this batch's total, saturated at the count asked for
__global__ void advance_produced(int* produced, const int* total, int need) {
    *produced = (int)min((int64_t)*produced + *total, (int64_t)need);
}

arc_status upload_scene(arc_context* ctx, const ArcSceneDesc* scene, SceneDev** out) {
    SceneDev h;
    memset(&h, 0, sizeof(h));
    h.desc = *scene;
    h.nrects = build_rects(*scene, h.rects);
    // the tracer indexes the material table with every surface's material
    for (int i = 0; i < h.nrects; ++i)
        ARC_CHECK_ARG(h.rects[i].material >= 0 && h.rects[i].material < ARC_MAX_MATERIALS, "material out of range");
    ARC_CHECK_ARG(scene->light_material >= 0 && scene->light_material < ARC_MAX_MATERIALS, "material out of range");
    SceneDev* d = nullptr;
    ARC_TRY(ctx->arena.get("scene_desc", sizeof(SceneDev), reinterpret_cast<void**>(&d)));
    // pageable source: the call returns once the bytes are staged, so h may go out of scope
    ARC_TRY_CUDA(cudaMemcpyAsync(d, &h, sizeof(SceneDev), cudaMemcpyHostToDevice, ctx->stream));
    *out = d;
    return ARC_OK;
}

}  // namespace
}  // namespace arc

using namespace arc;

extern "C" arc_status arc_scene_gbuffer_device(arc_context* ctx, const ArcSceneDesc* scene, const ArcGBufferView* out) {
    ARC_CHECK_ARG(ctx && scene && out && out->position && out->normal, "NULL argument");
    ARC_CHECK_ARG(out->width > 0 && out->height > 0 && out->pitch >= out->width, "bad G-buffer view");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    SceneDev* sd = nullptr;
    ARC_TRY(upload_scene(ctx, scene, &sd));
    const scene::Camera cam = scene::make_camera(*scene, out->width, out->height);
    const int64_t px = (int64_t)out->width * out->height;
    stage_begin(ctx, "scene_gbuffer");
    scene_gbuffer_kernel<<<(unsigned)((px + kSceneThreads - 1) / kSceneThreads), kSceneThreads, 0, ctx->stream>>>(
        sd, cam, out->width, out->height, reinterpret_cast<float4*>(const_cast<float*>(out->position)),
        reinterpret_cast<float4*>(const_cast<float*>(out->normal)), out->pitch);
    stage_end(ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

extern "C" arc_status arc_scene_trace_avpls_device(arc_context* ctx, const ArcSceneDesc* scene, uint64_t seed,
                                                   int32_t max_bounces, int32_t explicit_direct_illum,
                                                   const ArcAvplsGpuParam* out, int64_t* num_paths) {
    ARC_CHECK_ARG(ctx && scene && out, "NULL argument");
    ARC_CHECK_ARG(max_bounces >= 1 && max_bounces <= 64, "max_bounces out of range (1..64)");
    ARC_CHECK_ARG(out->numAvpls >= 0, "negative AVPL count");
    ARC_CHECK_ARG(out->numAvpls == 0 || (out->position && out->normal && out->incDirection && out->incRadiance &&
                                         out->antiradiance && out->materialIndex && out->bounce),
                  "NULL AVPL array");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int need = out->numAvpls;
    if (need == 0) {
        if (num_paths) *num_paths = 0;
        return ARC_OK;
    }
    SceneDev* sd = nullptr;
    ARC_TRY(upload_scene(ctx, scene, &sd));
    // about 1.8 AVPLs per path in the preset scenes: one batch of `need` paths usually suffices;
    // the per-path slots stay within 4 GB (which also keeps every count sum within an int)
    const int64_t slot_cap = ((int64_t)4 << 30) / ((int64_t)max_bounces * (int64_t)sizeof(ArcAvplHost));
    const int batch = (int)std::min<int64_t>(std::max(4096, need), slot_cap);
    const int nblocks = scan::num_blocks(batch);
    ArcAvplHost* slots = nullptr;
    int *counts = nullptr, *offsets = nullptr, *block_sums = nullptr, *state = nullptr;
    int64_t* paths = nullptr;
    ARC_TRY(ctx->arena.get("scene_slots", (size_t)batch * max_bounces * sizeof(ArcAvplHost),
                           reinterpret_cast<void**>(&slots)));
    ARC_TRY(ctx->arena.get("scene_counts", (size_t)batch * sizeof(int), reinterpret_cast<void**>(&counts)));
    ARC_TRY(ctx->arena.get("scene_offsets", (size_t)batch * sizeof(int), reinterpret_cast<void**>(&offsets)));
    ARC_TRY(ctx->arena.get("scene_block_sums", (size_t)nblocks * sizeof(int), reinterpret_cast<void**>(&block_sums)));
    ARC_TRY(ctx->arena.get("scene_state", 4 * sizeof(int), reinterpret_cast<void**>(&state)));  // produced, total
    ARC_TRY(ctx->arena.get("scene_paths", sizeof(int64_t), reinterpret_cast<void**>(&paths)));
    ARC_TRY_CUDA(cudaMemsetAsync(state, 0, 4 * sizeof(int), st));
    ARC_TRY_CUDA(cudaMemsetAsync(paths, 0, sizeof(int64_t), st));
    stage_begin(ctx, "scene_trace");
    int kernels = 0;
    int produced = 0;
    int64_t path0 = 0;
    while (produced < need) {
        if (path0 > (int64_t)need * 1000 + 100000) {  // the light sees nothing (as the CPU tracer)
            stage_end(ctx, kernels);
            return ARC_ERR_INVALID_ARG;
        }
        const unsigned grid = (unsigned)((batch + kSceneThreads - 1) / kSceneThreads);
        scene_trace_kernel<<<grid, kSceneThreads, 0, st>>>(sd, seed, path0, batch, max_bounces, explicit_direct_illum,
                                                          slots, counts);
        scan::exclusive_scan(counts, batch, offsets, block_sums, state + 1, st);
        ScatterArgs sa{slots, counts, offsets, block_sums, batch, max_bounces, path0, state, paths, *out};
        scatter_avpls<<<grid, kSceneThreads, 0, st>>>(sa);
        advance_produced<<<1, 1, 0, st>>>(state, state + 1, need);
        kernels += 5;
        ARC_TRY_CUDA(cudaGetLastError());
        ARC_TRY_CUDA(cudaMemcpyAsync(&produced, state, sizeof(int), cudaMemcpyDeviceToHost, st));
        ARC_TRY_CUDA(cudaStreamSynchronize(st));
        path0 += batch;
    }
    stage_end(ctx, kernels);
    if (num_paths) {
        ARC_TRY_CUDA(cudaMemcpyAsync(num_paths, paths, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        ARC_TRY_CUDA(cudaStreamSynchronize(st));
    }
    return ARC_OK;
}
