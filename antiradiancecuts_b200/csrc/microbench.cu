// FP32 FMA throughput microbenchmark: the roofline denominator of the gather kernels (the
// measured machine peaks list HBM bandwidth and BF16 tensor throughput only).  Each thread runs
// 8 independent FMA chains, scalar (FFMA) or packed (fma.rn.f32x2, two lanes per instruction).
#include <cstdint>

#include "arc_internal.h"

namespace arc {
namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) fma_scalar(float* out, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + c;
    for (int i = 0; i < kIters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 1234.5f) out[threadIdx.x] = s;  // keeps the chains alive
}

__global__ void __launch_bounds__(256) fma_packed(float* out, float a, float b) {
    uint64_t x[kChains / 2];
    const float2 av = make_float2(a, a), bv = make_float2(b, b);
    const uint64_t A = *reinterpret_cast<const uint64_t*>(&av), B = *reinterpret_cast<const uint64_t*>(&bv);
#pragma unroll
    for (int c = 0; c < kChains / 2; ++c) {
        const float2 v = make_float2(threadIdx.x * 1e-3f + c, c + 0.5f);
        x[c] = *reinterpret_cast<const uint64_t*>(&v);
    }
    for (int i = 0; i < kIters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains / 2; ++c) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[c]) : "l"(A), "l"(B));
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains / 2; ++c) {
        const float2 v = *reinterpret_cast<const float2*>(&x[c]);
        s += v.x + v.y;
    }
    if (s == 1234.5f) out[threadIdx.x] = s;
}

}  // namespace
}  // namespace arc

using namespace arc;

extern "C" arc_status arc_measure_fp32_peak(arc_context* ctx, double* scalar_tflops, double* packed_tflops) {
    ARC_CHECK_ARG(ctx && scalar_tflops && packed_tflops, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    float* out = nullptr;
    ARC_TRY(ctx->arena.get("fma_sink", 1024 * sizeof(float), reinterpret_cast<void**>(&out)));
    const int blocks = ctx->sm_count * 8;
    const double flops = 2.0 * kChains * (double)kIters * blocks * 256;
    ScopedEvents<2> ev;
    ARC_TRY_CUDA(ev.create());
    const cudaEvent_t e0 = ev[0], e1 = ev[1];
    float best[2] = {1e30f, 1e30f};
    for (int rep = 0; rep < 6; ++rep) {
        for (int v = 0; v < 2; ++v) {
            ARC_TRY_CUDA(cudaEventRecord(e0, ctx->stream));
            if (v == 0)
                fma_scalar<<<blocks, 256, 0, ctx->stream>>>(out, 0.999f, 1e-4f);
            else
                fma_packed<<<blocks, 256, 0, ctx->stream>>>(out, 0.999f, 1e-4f);
            ARC_TRY_CUDA(cudaEventRecord(e1, ctx->stream));
            ARC_TRY_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            ARC_TRY_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0 && ms < best[v]) best[v] = ms;  // rep 0 warms up
        }
    }
    *scalar_tflops = flops / (best[0] * 1e-3) / 1e12;
    *packed_tflops = flops / (best[1] * 1e-3) / 1e12;
    return ARC_OK;
}
