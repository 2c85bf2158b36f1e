// The cut-refinement MLP (16 -> 64 -> 64 -> 64 -> 1, GELU or ReLU, BF16 weights, FP32 accumulation) on
// the 5th-generation tensor cores.  No counterpart in the reference: it predicts, for an 8x8 pixel
// tile and a tree node, whether the cut must refine the node.
//
// Two kernels.  Each 128-thread CTA walks 128-row tiles of the input (thread t owns row t):
//   forward   X[128x16] -> tcgen05.mma -> TMEM -> +b, activation -> BF16 core-matrix smem -> next layer;
//             the 64 -> 1 output layer runs on the CUDA cores from registers (mlp_tile.cuh, shared
//             with the fused level kernel of the learned cut).
//   training  the forward pass, then BCE gradient, and the backward pass:
//             dH_l = dZ_{l+1} W_{l+1}                       (M = 128 rows, B read MN-major)
//             dW_l += dZ_l^T H_{l-1}   (accumulated in TMEM over every tile the CTA owns;
//                                       M padded to 128 = out features, A and B read MN-major)
//             bias / output-layer gradients are warp-reduced into shared memory.
// Weights are kept as an FP32 master copy (Adam updates it) and rounded to BF16 into shared
// memory by every CTA.  Every tensor-core result waits on an mbarrier with a bounded wait; the CTA
// stops (and still frees its TMEM) if a wait gives up.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "arc_internal.h"
#include "device_common.cuh"
#include "mlp_tile.cuh"
#include "pcg32.h"
#include "tcgen05.cuh"

namespace arc {
namespace mlp {

// shared-memory carve-up (bytes); dZ is followed by 2 KB because the M-padded weight-gradient
// MMA reads up to that far past it (the extra rows land in D rows 64..127, which are ignored)
constexpr uint32_t sW1 = 0, sW2 = sW1 + 2048, sW3 = sW2 + 8192, sX = sW3 + 8192, sH1 = sX + 4096,
                   sH2 = sH1 + 16384, sZ1 = sH2 + 16384, sZ2 = sZ1 + 16384, sDZ = sZ2 + 16384,
                   sVecTrain = sDZ + 16384 + 2048;
constexpr uint32_t kVecBytes = (4 * 64 + 4 * 64 + 4) * 4;
constexpr uint32_t kSmemTrain = sVecTrain + kVecBytes;
// inference: weights | X tile (4 KB) | hidden (16 KB) | vectors
constexpr uint32_t sInX = kWeightBytes, sInH = sInX + 4096, sInVec = sInH + 16384,
                   kSmemInfer = sInVec + kVecBytesInfer;

struct Args {
    const float* params;
    const __nv_bfloat16* x;  // [rows][16]
    int64_t rows;
    float* logits;            // [rows] (forward mode)
    const float* labels;      // [rows] (training)
    const float* weights;     // [rows] sample weights or NULL
    float loss_scale;         // 1 / sum of weights
    float* grads;             // [kParams] (atomicAdd)
    float* loss;              // [1]
    int loss_kind;            // arc_mlp_loss
    uint32_t* err;
};

// store 64 values of row t as BF16 into a K-major (K = 64) core-matrix buffer
__device__ __forceinline__ void store_row64(unsigned char* buf, int t, const float* v) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint4 q;
        q.x = pack2(v[8 * c + 0], v[8 * c + 1]);
        q.y = pack2(v[8 * c + 2], v[8 * c + 3]);
        q.z = pack2(v[8 * c + 4], v[8 * c + 5]);
        q.w = pack2(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(buf + tc::kmajor_offset(t, 8 * c, 64)) = q;
    }
}

__device__ __forceinline__ void load_row64(const unsigned char* buf, int t, float* v) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint4 q = *reinterpret_cast<const uint4*>(buf + tc::kmajor_offset(t, 8 * c, 64));
        const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 f = __bfloat1622float2(p[e]);
            v[8 * c + 2 * e] = f.x;
            v[8 * c + 2 * e + 1] = f.y;
        }
    }
}

__device__ __forceinline__ void load_tmem64(uint32_t taddr, float* v) {
#pragma unroll
    for (int c = 0; c < 4; ++c) tc::ld16(taddr + 16 * c, v + 16 * c);
}

// one 32-lane sum, result in every lane
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// column sums of a 128 x 64 block held one row per thread -> shared accumulator g[64]
__device__ __forceinline__ void accumulate_columns(const float* v, float* g, int lane) {
#pragma unroll
    for (int j = 0; j < 64; ++j) {
        const float s = warp_sum(v[j]);
        if (lane == 0) atomicAdd(&g[j], s);
    }
}

// Forward over every row of the input: persistent CTAs, one 128-row tile at a time.
template <int ACT>
__global__ void __launch_bounds__(128) mlp_infer_kernel(Args a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int t = threadIdx.x, w = t >> 5;
    float* vec = reinterpret_cast<float*>(sm + sInVec);
    load_weights<ACT>(sm, vec, a.params, t, 128);
    if (w == 0) tc::alloc(&tmem_base, 64);
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    InferCta c{smem_u32(sm), 0, sInH, sm, vec, tmem_base, &bar, 0u, a.err};
    const int64_t ntiles = (a.rows + kRows - 1) / kRows;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t row = tile * kRows + t;
        const bool valid = row < a.rows;
        uint4 x0 = make_uint4(0, 0, 0, 0), x1 = make_uint4(0, 0, 0, 0);
        if (valid) {
            const uint4* xp = reinterpret_cast<const uint4*>(a.x + row * kIn);
            x0 = xp[0];
            x1 = xp[1];
        }
        *reinterpret_cast<uint4*>(sm + sInX + tc::kmajor_offset(t, 0, kIn)) = x0;
        *reinterpret_cast<uint4*>(sm + sInX + tc::kmajor_offset(t, 8, kIn)) = x1;
        float y;
        if (!infer_tile<ACT>(c, sInX, t, &y)) {
            // the wait gave up (the error word says so): its commit gets a second bounded wait
            // before the TMEM and shared memory are released (the failed wait flipped the phase)
            if (t == 0) mbar_wait_bounded(&bar, c.phase ^ 1u, a.err);
            break;
        }
        if (valid) a.logits[row] = y;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (w == 0) tc::dealloc(tmem_base, 64);
}

// Forward + backward with weight-gradient accumulation in TMEM (training).
template <int ACT>
__global__ void __launch_bounds__(128) mlp_train_kernel(Args a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    float* vec = reinterpret_cast<float*>(sm + sVecTrain);
    float* b1 = vec;
    float* b2 = vec + 64;
    float* b3 = vec + 128;
    float* w4 = vec + 192;
    float* gb1 = vec + 256;  // training: bias / output-layer gradient accumulators
    float* gb2 = vec + 320;
    float* gb3 = vec + 384;
    float* gw4 = vec + 448;
    float* gb4 = vec + 512;
    constexpr uint32_t kCols = 256;  // D | dW3 | dW2 | dW1

    // weights -> BF16 core-matrix layouts, vectors -> FP32
    for (int i = t; i < kHid * kIn; i += 128)
        *reinterpret_cast<__nv_bfloat16*>(sm + sW1 + tc::kmajor_offset(i / kIn, i % kIn, kIn)) =
            __float2bfloat16_rn(a.params[oW1 + i]);
    for (int i = t; i < kHid * kHid; i += 128) {
        *reinterpret_cast<__nv_bfloat16*>(sm + sW2 + tc::kmajor_offset(i / kHid, i % kHid, kHid)) =
            __float2bfloat16_rn(a.params[oW2 + i]);
        *reinterpret_cast<__nv_bfloat16*>(sm + sW3 + tc::kmajor_offset(i / kHid, i % kHid, kHid)) =
            __float2bfloat16_rn(a.params[oW3 + i]);
    }
    if (t < 64) {
        b1[t] = a.params[oB1 + t];
        b2[t] = a.params[oB2 + t];
        b3[t] = a.params[oB3 + t];
        w4[t] = a.params[oW4 + t];
    }
    const float b4 = a.params[oB4];
    for (int i = t; i < 4 * 64 + 4; i += 128) gb1[i] = 0.0f;
    if (w == 0) tc::alloc(&tmem_base, kCols);
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t lane_off = (uint32_t)(w * 32) << 16;
    const uint32_t base = smem_u32(sm);
    uint32_t phase = 0;
    bool any_tile = false;
    bool gave_up = false;  // a tensor-core wait gave up: its commit may still be in flight

    constexpr uint32_t idKK64 = tc::idesc_bf16(128, 64, false, false);
    constexpr uint32_t idKM64 = tc::idesc_bf16(128, 64, false, true);
    constexpr uint32_t idMM64 = tc::idesc_bf16(128, 64, true, true);
    constexpr uint32_t idMM16 = tc::idesc_bf16(128, 16, true, true);

    // wait for the MMAs committed on `bar`; every thread learns whether all threads got there
    auto wait_mma = [&]() -> bool {
        const bool ok = mbar_wait_bounded(&bar, phase, a.err);
        phase ^= 1u;
        tc::fence_after_sync();
        const bool all = __syncthreads_and(ok) != 0;
        if (!all) gave_up = true;
        return all;
    };
    // make this thread's generic-proxy smem writes visible to the tensor cores, then barrier
    auto publish_smem = [&]() {
        fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
    };
    // forward layer with K = 64: D = A[128 x 64] B^T
    auto layer64 = [&](uint32_t A, uint32_t B) {
        if (t == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int s = 0; s < 4; ++s)
                tc::mma(tmem, tc::smem_desc(base + A + 256 * s, 128, 1024), tc::smem_desc(base + B + 256 * s, 128, 1024),
                        idKK64, s > 0);
            tc::commit(&bar);
        }
    };

    const int64_t ntiles = (a.rows + kRows - 1) / kRows;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t row = tile * kRows + t;
        const bool valid = row < a.rows;
        uint4 x0 = make_uint4(0, 0, 0, 0), x1 = make_uint4(0, 0, 0, 0);
        if (valid) {
            const uint4* xp = reinterpret_cast<const uint4*>(a.x + row * kIn);
            x0 = xp[0];
            x1 = xp[1];
        }
        *reinterpret_cast<uint4*>(sm + sX + tc::kmajor_offset(t, 0, kIn)) = x0;
        *reinterpret_cast<uint4*>(sm + sX + tc::kmajor_offset(t, 8, kIn)) = x1;

        float z[64], h[64];
        // ---- layer 1 (K = 16) ----
        publish_smem();
        if (t == 0) {
            tc::fence_after_sync();
            tc::mma(tmem, tc::smem_desc(base + sX, 128, 256), tc::smem_desc(base + sW1, 128, 256), idKK64, false);
            tc::commit(&bar);
        }
        if (!wait_mma()) break;
        load_tmem64(tmem + lane_off, z);
#pragma unroll
        for (int j = 0; j < 64; ++j) {
            z[j] += b1[j];
            h[j] = act<ACT>(z[j]);
        }
        store_row64(sm + sH1, t, h);
        store_row64(sm + sZ1, t, z);
        // ---- layer 2 ----
        publish_smem();
        layer64(sH1, sW2);
        if (!wait_mma()) break;
        load_tmem64(tmem + lane_off, z);
#pragma unroll
        for (int j = 0; j < 64; ++j) {
            z[j] += b2[j];
            h[j] = act<ACT>(z[j]);
        }
        store_row64(sm + sH2, t, h);
        store_row64(sm + sZ2, t, z);
        // ---- layer 3 (kept in registers) ----
        publish_smem();
        layer64(sH2, sW3);
        if (!wait_mma()) break;
        load_tmem64(tmem + lane_off, z);
#pragma unroll
        for (int j = 0; j < 64; ++j) {
            z[j] += b3[j];
            h[j] = act<ACT>(z[j]);
        }
        // ---- output layer on the CUDA cores ----
        float y = b4;
#pragma unroll
        for (int j = 0; j < 64; ++j) y = fmaf(h[j], w4[j], y);

        // ---- loss, output-layer gradients, dZ3 ----
        float dy = 0.0f, l = 0.0f;
        if (valid) {
            const float lab = a.labels[row];
            const float wgt = a.weights ? a.weights[row] : 1.0f;
            if (a.loss_kind == ARC_MLP_LOSS_SQUARED) {
                const float d = y - lab;
                dy = wgt * 2.0f * d * a.loss_scale;
                l = wgt * d * d * a.loss_scale;
            } else {
                const float p = 1.0f / (1.0f + expf(-y));
                dy = wgt * (p - lab) * a.loss_scale;
                l = wgt * (fmaxf(y, 0.0f) - y * lab + log1pf(expf(-fabsf(y)))) * a.loss_scale;
            }
        }
        {
            const float ls = warp_sum(l), ds = warp_sum(dy);
            if (lane == 0) {
                atomicAdd(a.loss, ls);
                atomicAdd(gb4, ds);
            }
        }
        float g[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) g[j] = dy * h[j];
        accumulate_columns(g, gw4, lane);
#pragma unroll
        for (int j = 0; j < 64; ++j) g[j] = dy * w4[j] * act_grad<ACT>(z[j]);  // dZ3
        accumulate_columns(g, gb3, lane);
        store_row64(sm + sDZ, t, g);
        // dW3 += dZ3^T H2 ; dH2 = dZ3 W3
        publish_smem();
        if (t == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int s = 0; s < 8; ++s)
                tc::mma(tmem + 64, tc::smem_desc(base + sDZ + 2048 * s, 1024, 128),
                        tc::smem_desc(base + sH2 + 2048 * s, 1024, 128), idMM64, any_tile || s > 0);
#pragma unroll
            for (int s = 0; s < 4; ++s)
                tc::mma(tmem, tc::smem_desc(base + sDZ + 256 * s, 128, 1024), tc::smem_desc(base + sW3 + 2048 * s, 1024, 128),
                        idKM64, s > 0);
            tc::commit(&bar);
        }
        if (!wait_mma()) break;
        load_tmem64(tmem + lane_off, g);  // dH2
        load_row64(sm + sZ2, t, z);
#pragma unroll
        for (int j = 0; j < 64; ++j) g[j] *= act_grad<ACT>(z[j]);  // dZ2
        accumulate_columns(g, gb2, lane);
        store_row64(sm + sDZ, t, g);
        // dW2 += dZ2^T H1 ; dH1 = dZ2 W2
        publish_smem();
        if (t == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int s = 0; s < 8; ++s)
                tc::mma(tmem + 128, tc::smem_desc(base + sDZ + 2048 * s, 1024, 128),
                        tc::smem_desc(base + sH1 + 2048 * s, 1024, 128), idMM64, any_tile || s > 0);
#pragma unroll
            for (int s = 0; s < 4; ++s)
                tc::mma(tmem, tc::smem_desc(base + sDZ + 256 * s, 128, 1024), tc::smem_desc(base + sW2 + 2048 * s, 1024, 128),
                        idKM64, s > 0);
            tc::commit(&bar);
        }
        if (!wait_mma()) break;
        load_tmem64(tmem + lane_off, g);  // dH1
        load_row64(sm + sZ1, t, z);
#pragma unroll
        for (int j = 0; j < 64; ++j) g[j] *= act_grad<ACT>(z[j]);  // dZ1
        accumulate_columns(g, gb1, lane);
        store_row64(sm + sDZ, t, g);
        // dW1 += dZ1^T X  (N = 16)
        publish_smem();
        if (t == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int s = 0; s < 8; ++s)
                tc::mma(tmem + 192, tc::smem_desc(base + sDZ + 2048 * s, 1024, 128),
                        tc::smem_desc(base + sX + 512 * s, 256, 128), idMM16, any_tile || s > 0);
            tc::commit(&bar);
        }
        if (!wait_mma()) break;
        any_tile = true;
    }

    if (any_tile && !gave_up) {
        // weight gradients: D rows 0..63 (= output features) live in TMEM lanes 0..63
        if (w < 2) {
            float v[64];
            load_tmem64(tmem + lane_off + 64, v);
#pragma unroll
            for (int j = 0; j < 64; ++j) atomicAdd(&a.grads[oW3 + t * 64 + j], v[j]);
            load_tmem64(tmem + lane_off + 128, v);
#pragma unroll
            for (int j = 0; j < 64; ++j) atomicAdd(&a.grads[oW2 + t * 64 + j], v[j]);
            tc::ld16(tmem + lane_off + 192, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) atomicAdd(&a.grads[oW1 + t * 16 + j], v[j]);
        }
        __syncthreads();
        if (t < 64) {
            atomicAdd(&a.grads[oB1 + t], gb1[t]);
            atomicAdd(&a.grads[oB2 + t], gb2[t]);
            atomicAdd(&a.grads[oB3 + t], gb3[t]);
            atomicAdd(&a.grads[oW4 + t], gw4[t]);
        }
        if (t == 0) atomicAdd(&a.grads[oB4], gb4[0]);
    }
    // after a wait that gave up (the error word says so), the last commit gets a second bounded
    // wait before the TMEM and shared memory are released (the failed wait flipped the phase)
    if (gave_up && t == 0) mbar_wait_bounded(&bar, phase ^ 1u, a.err);
    tc::fence_before_sync();
    __syncthreads();
    if (w == 0) tc::dealloc(tmem, kCols);
}

__global__ void adam_kernel(float* params, float* grads, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grads[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    grads[i] = 0.0f;
}

}  // namespace mlp
}  // namespace arc

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
using namespace arc;

struct arc_mlp {
    arc_context* ctx = nullptr;
    float* params = nullptr;  // device FP32 master copy
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    float* loss = nullptr;
    int64_t step = 0;
    int32_t loss_kind = ARC_MLP_LOSS_BCE;
    int32_t activation = ARC_MLP_ACT_GELU;
};

namespace {

arc_status mlp_launch(arc_mlp* m, bool train, const void* x, int64_t rows, float* logits, const float* labels,
                      const float* weights, float loss_scale) {
    arc_context* ctx = m->ctx;
    mlp::Args a{};
    a.params = m->params;
    a.x = static_cast<const __nv_bfloat16*>(x);
    a.rows = rows;
    a.logits = logits;
    a.labels = labels;
    a.weights = weights;
    a.loss_scale = loss_scale;
    a.grads = m->grads;
    a.loss = m->loss;
    a.loss_kind = m->loss_kind;
    a.err = ctx->d_error;
    const int64_t tiles = (rows + mlp::kRows - 1) / mlp::kRows;
    if (tiles == 0) return ARC_OK;
    // the shared-memory limit is a per-device attribute of the kernel: set it on every call (a
    // host-side call), not once per process, so contexts on other devices get it too
    const bool relu = m->activation == ARC_MLP_ACT_RELU;
    if (train) {
        auto* k = relu ? mlp::mlp_train_kernel<mlp::kActRelu> : mlp::mlp_train_kernel<mlp::kActGelu>;
        ARC_TRY_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::kSmemTrain));
        const int grid = (int)std::min<int64_t>(tiles, ctx->sm_count);
        stage_begin(ctx, "mlp_train");
        k<<<grid, 128, mlp::kSmemTrain, ctx->stream>>>(a);
        stage_end(ctx, 1);
    } else {
        auto* k = relu ? mlp::mlp_infer_kernel<mlp::kActRelu> : mlp::mlp_infer_kernel<mlp::kActGelu>;
        ARC_TRY_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::kSmemInfer));
        const int grid = (int)std::min<int64_t>(tiles, (int64_t)ctx->sm_count * 4);
        stage_begin(ctx, "mlp_forward");
        k<<<grid, 128, mlp::kSmemInfer, ctx->stream>>>(a);
        stage_end(ctx, 1);
    }
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

}  // namespace

namespace arc {
const float* mlp_params(const arc_mlp* m) { return m->params; }
int32_t mlp_loss_kind(const arc_mlp* m) { return m->loss_kind; }
int32_t mlp_activation(const arc_mlp* m) { return m->activation; }
arc_status mlp_forward_device(arc_mlp* m, const void* x, int64_t rows, float* logits) {
    return mlp_launch(m, false, x, rows, logits, nullptr, nullptr, 0.0f);
}
}  // namespace arc

extern "C" {

int32_t arc_mlp_num_params(void) { return mlp::kParams; }

arc_status arc_mlp_create(arc_context* ctx, uint64_t seed, arc_mlp** out) {
    ARC_CHECK_ARG(ctx && out, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    arc_mlp* m = new arc_mlp();
    m->ctx = ctx;
    const size_t bytes = sizeof(float) * mlp::kParams;
    cudaError_t e = cudaMalloc(&m->params, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->grads, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->adam_m, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->adam_v, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(float));
    if (e != cudaSuccess) {
        set_last_error(std::string("arc_mlp_create: ") + cudaGetErrorString(e));
        arc_mlp_destroy(m);
        return ARC_ERR_OUT_OF_MEMORY;
    }
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a PCG32 stream
    std::vector<float> p(mlp::kParams, 0.0f);
    arc_pcg32 r;
    arc_pcg32_seed(&r, seed, 0x6d6c70ULL);
    auto fill = [&](int off, int count, int fan_in) {
        const float b = 1.0f / std::sqrt((float)fan_in);
        for (int i = 0; i < count; ++i) p[off + i] = (2.0f * arc_pcg32_float(&r) - 1.0f) * b;
    };
    fill(mlp::oW1, 64 * 16, 16);
    fill(mlp::oB1, 64, 16);
    fill(mlp::oW2, 64 * 64, 64);
    fill(mlp::oB2, 64, 64);
    fill(mlp::oW3, 64 * 64, 64);
    fill(mlp::oB3, 64, 64);
    fill(mlp::oW4, 64, 64);
    fill(mlp::oB4, 1, 64);
    e = cudaMemcpy(m->params, p.data(), bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->grads, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(m->adam_m, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(m->adam_v, 0, bytes);
    if (e != cudaSuccess) {
        set_last_error(std::string("arc_mlp_create: ") + cudaGetErrorString(e));
        arc_mlp_destroy(m);
        return ARC_ERR_CUDA;
    }
    *out = m;
    return ARC_OK;
}

arc_status arc_mlp_destroy(arc_mlp* m) {
    if (!m) return ARC_OK;
    if (m->ctx) {
        cudaSetDevice(m->ctx->device);
        cudaStreamSynchronize(m->ctx->stream);
    }
    cudaFree(m->params);
    cudaFree(m->grads);
    cudaFree(m->adam_m);
    cudaFree(m->adam_v);
    cudaFree(m->loss);
    delete m;
    return ARC_OK;
}

arc_status arc_mlp_set_params(arc_mlp* m, const float* host, int32_t n) {
    ARC_CHECK_ARG(m && host && n == mlp::kParams, "parameter count mismatch");
    ARC_TRY_CUDA(cudaSetDevice(m->ctx->device));
    ARC_TRY_CUDA(cudaMemcpyAsync(m->params, host, sizeof(float) * n, cudaMemcpyHostToDevice, m->ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return ARC_OK;
}

arc_status arc_mlp_get_params(arc_mlp* m, float* host, int32_t n) {
    ARC_CHECK_ARG(m && host && n == mlp::kParams, "parameter count mismatch");
    ARC_TRY_CUDA(cudaSetDevice(m->ctx->device));
    ARC_TRY_CUDA(cudaMemcpyAsync(host, m->params, sizeof(float) * n, cudaMemcpyDeviceToHost, m->ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return ARC_OK;
}

arc_status arc_mlp_forward(arc_mlp* m, const void* features_bf16, int64_t rows, float* logits) {
    ARC_CHECK_ARG(m && (rows == 0 || (features_bf16 && logits)), "NULL argument");
    ARC_CHECK_ARG(reinterpret_cast<uintptr_t>(features_bf16) % 16 == 0, "features must be 16-byte aligned");
    ARC_TRY_CUDA(cudaSetDevice(m->ctx->device));
    return mlp_launch(m, false, features_bf16, rows, logits, nullptr, nullptr, 0.0f);
}

arc_status arc_mlp_gradients(arc_mlp* m, const void* features_bf16, const float* labels, const float* weights,
                             int64_t rows, float weight_sum, float* host_grads, float* host_loss) {
    ARC_CHECK_ARG(m && features_bf16 && labels && rows > 0 && weight_sum > 0.0f, "bad argument");
    ARC_TRY_CUDA(cudaSetDevice(m->ctx->device));
    ARC_TRY_CUDA(cudaMemsetAsync(m->grads, 0, sizeof(float) * mlp::kParams, m->ctx->stream));
    ARC_TRY_CUDA(cudaMemsetAsync(m->loss, 0, sizeof(float), m->ctx->stream));
    ARC_TRY(mlp_launch(m, true, features_bf16, rows, nullptr, labels, weights, 1.0f / weight_sum));
    if (host_grads)
        ARC_TRY_CUDA(cudaMemcpyAsync(host_grads, m->grads, sizeof(float) * mlp::kParams, cudaMemcpyDeviceToHost,
                                     m->ctx->stream));
    if (host_loss) ARC_TRY_CUDA(cudaMemcpyAsync(host_loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(m->ctx->stream));
    ARC_TRY_CUDA(cudaMemsetAsync(m->grads, 0, sizeof(float) * mlp::kParams, m->ctx->stream));
    return ARC_OK;
}

arc_status arc_mlp_set_loss(arc_mlp* m, int32_t kind) {
    ARC_CHECK_ARG(m, "NULL model");
    ARC_CHECK_ARG(kind == ARC_MLP_LOSS_BCE || kind == ARC_MLP_LOSS_SQUARED, "unknown loss");
    m->loss_kind = kind;
    return ARC_OK;
}

int32_t arc_mlp_get_loss(const arc_mlp* m) { return m ? m->loss_kind : -1; }

arc_status arc_mlp_set_activation(arc_mlp* m, int32_t kind) {
    ARC_CHECK_ARG(m, "NULL model");
    ARC_CHECK_ARG(kind == ARC_MLP_ACT_GELU || kind == ARC_MLP_ACT_RELU, "unknown activation");
    m->activation = kind;
    return ARC_OK;
}

int32_t arc_mlp_get_activation(const arc_mlp* m) { return m ? m->activation : -1; }

arc_status arc_mlp_train_step(arc_mlp* m, const void* features_bf16, const float* labels, const float* weights,
                              int64_t rows, float weight_sum, float lr, float* device_loss_accum) {
    ARC_CHECK_ARG(m && features_bf16 && labels && rows > 0 && weight_sum > 0.0f, "bad argument");
    ARC_TRY_CUDA(cudaSetDevice(m->ctx->device));
    float* saved = m->loss;
    if (device_loss_accum) m->loss = device_loss_accum;
    arc_status s = mlp_launch(m, true, features_bf16, rows, nullptr, labels, weights, 1.0f / weight_sum);
    m->loss = saved;
    ARC_TRY(s);
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - std::pow(b1, (float)m->step), bc2 = 1.0f - std::pow(b2, (float)m->step);
    mlp::adam_kernel<<<(mlp::kParams + 255) / 256, 256, 0, m->ctx->stream>>>(m->params, m->grads, m->adam_m, m->adam_v,
                                                                             mlp::kParams, lr, b1, b2, 1e-8f, bc1, bc2);
    m->ctx->launches += 1;
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

}  // extern "C"
