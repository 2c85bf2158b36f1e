// Shared pieces of the cut-refinement MLP (16 -> 64 -> 64 -> 64 -> 1): parameter layout, the
// activations, and the inference of one 128-row tile on the tensor cores, used by the stand-alone
// forward kernel (mlp.cu) and by the fused level kernel of the learned cut (learned.cu).  The
// activation is a property of the model and a template parameter of every kernel (kActGelu,
// kActRelu).
//
// ReLU: max(x, 0).  Inference takes the parameters as they are; a hidden value costs one add
// (bias), and the rounding to BF16 applies the ReLU for free (cvt.rn.relu.bf16x2.f32).
//
// GELU, in its sigmoid form (Hendrycks & Gimpel 2016, x sigma(1.702 x)), written with
// the hardware tanh (tanh.approx.f32):
//     gelu(x) = x/2 (1 + tanh(s x)),   s = 1.702 / 2.
// Training and the FP64 oracle use this function.  Inference folds its constants into the
// parameters (load_weights): with z' = s z the activation is (1 / (2 s)) g(z'), g(z) = z + z tanh(z),
// so layer 1 takes s W1, s b1, the next layers (s / (2 s)) W = W / 2 and s b, and the output layer
// w4 / (2 s); the epilogue is then one add (bias), one tanh and one multiply-add per value.
// (Two forms were measured and dropped: the tanh form of GELU, whose cubic argument costs three
// more operations per value, and a BF16-pair tanh, tanh.approx.bf16x2, whose packing cost more
// issue slots than the special-function work it saved.)
#ifndef ARC_MLP_TILE_CUH_
#define ARC_MLP_TILE_CUH_

#include <cuda_bf16.h>
#include <stdint.h>

#include "device_common.cuh"
#include "tcgen05.cuh"

namespace arc {
namespace mlp {

constexpr int kIn = 16, kHid = 64, kRows = 128;
// parameter layout of the FP32 master copy
constexpr int oW1 = 0, oB1 = oW1 + kHid * kIn, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid,
              oB3 = oW3 + kHid * kHid, oW4 = oB3 + kHid, oB4 = oW4 + kHid, kParams = oB4 + 1;  // 9473

constexpr int kActGelu = 0, kActRelu = 1;  // arc_mlp_activation
constexpr float kGeluS = 0.851f;                   // 1.702 / 2
constexpr float kGeluOut = 0.5f / 0.851f;          // 1 / (2 s): the folded activation's scale

__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float gelu(float x) {
    const float th = tanh_hw(kGeluS * x);
    const float hx = 0.5f * x;
    return fmaf(hx, th, hx);
}

// d gelu / dx = (1 + th) / 2 + (x / 2) s (1 - th^2)
__device__ __forceinline__ float gelu_grad(float x) {
    const float th = tanh_hw(kGeluS * x);
    return fmaf(0.5f, th, 0.5f) + 0.5f * x * kGeluS * (1.0f - th * th);
}

// activation and its derivative in unfolded form (training)
template <int ACT>
__device__ __forceinline__ float act(float x) {
    if constexpr (ACT == kActRelu) return fmaxf(x, 0.0f);
    else return gelu(x);
}

template <int ACT>
__device__ __forceinline__ float act_grad(float x) {
    if constexpr (ACT == kActRelu) return x > 0.0f ? 1.0f : 0.0f;
    else return gelu_grad(x);
}

// The folded activation of inference for a pair: x = z + b (both already scaled by s), g(x) =
// x + x tanh(x); the result is 2 s gelu of the unscaled value.
__device__ __forceinline__ uint64_t act2(uint64_t z, uint64_t b) {
    const uint64_t x = f2_add(z, b);
    float x0, x1;
    f2_split(x, x0, x1);
    return f2_fma(x, f2(tanh_hw(x0), tanh_hw(x1)), x);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// {bf16(max(a, 0)), bf16(max(b, 0))}, a in the low half like pack2 (cvt puts its first source in
// the high half)
__device__ __forceinline__ uint32_t pack2_relu(float a, float b) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
    return d;
}

// One inference hidden value pair: z + b through the activation, rounded to a BF16 pair.
template <int ACT>
__device__ __forceinline__ uint32_t hidden_pair(uint64_t z, uint64_t b) {
    float g0, g1;
    if constexpr (ACT == kActRelu) {
        f2_split(f2_add(z, b), g0, g1);
        return pack2_relu(g0, g1);
    } else {
        f2_split(act2(z, b), g0, g1);
        return pack2(g0, g1);
    }
}

// y + w (activation of z + b) for a pair, FP32 (the output layer)
template <int ACT>
__device__ __forceinline__ uint64_t output_pair(uint64_t z, uint64_t b, uint64_t w, uint64_t y) {
    if constexpr (ACT == kActRelu) {
        float x0, x1;
        f2_split(f2_add(z, b), x0, x1);
        return f2_fma(f2(fmaxf(x0, 0.0f), fmaxf(x1, 0.0f)), w, y);
    } else {
        return f2_fma(act2(z, b), w, y);
    }
}

// Weights of one CTA for inference: W1 | W2 | W3 as BF16 K-major core matrices, then b1, b2,
// b3, w4, b4 as FP32.
constexpr uint32_t kW1 = 0, kW2 = kW1 + 2048, kW3 = kW2 + 8192, kWeightBytes = kW3 + 8192;
constexpr uint32_t kVecBytesInfer = (4 * 64 + 4) * 4;
// weights followed by the vectors: the image a CTA copies into shared memory in one bulk copy
constexpr uint32_t kImageBytes = kWeightBytes + kVecBytesInfer;
static_assert(kImageBytes % 16 == 0, "bulk copies move multiples of 16 bytes");

// Every thread of the CTA (nthreads of them) helps load the weights (into shared memory, or into
// a global image in the same layout): W1 | W2 | W3 in BF16, then b1 | b2 | b3 | w4 | b4 in FP32.
// GELU folds its constants in (see the top of this file): s W1 | W2 / 2 | W3 / 2, then
// s b1 | s b2 | s b3 | w4 / (2 s) | b4; ReLU takes the parameters as they are.
template <int ACT>
__device__ __forceinline__ void load_weights(unsigned char* w, float* vec, const float* params, int t, int nthreads) {
    const float s1 = ACT == kActGelu ? kGeluS : 1.0f, sh = ACT == kActGelu ? 0.5f : 1.0f,
                sb = ACT == kActGelu ? kGeluS : 1.0f, so = ACT == kActGelu ? kGeluOut : 1.0f;
    for (int i = t; i < kHid * kIn; i += nthreads)
        *reinterpret_cast<__nv_bfloat16*>(w + kW1 + tc::kmajor_offset(i / kIn, i % kIn, kIn)) =
            __float2bfloat16_rn(s1 * params[oW1 + i]);
    for (int i = t; i < kHid * kHid; i += nthreads) {
        *reinterpret_cast<__nv_bfloat16*>(w + kW2 + tc::kmajor_offset(i / kHid, i % kHid, kHid)) =
            __float2bfloat16_rn(sh * params[oW2 + i]);
        *reinterpret_cast<__nv_bfloat16*>(w + kW3 + tc::kmajor_offset(i / kHid, i % kHid, kHid)) =
            __float2bfloat16_rn(sh * params[oW3 + i]);
    }
    for (int i = t; i < 64; i += nthreads) {
        vec[i] = sb * params[oB1 + i];
        vec[64 + i] = sb * params[oB2 + i];
        vec[128 + i] = sb * params[oB3 + i];
        vec[192 + i] = so * params[oW4 + i];
    }
    if (t == 0) vec[256] = params[oB4];
}

// Inference state of one 128-thread CTA: the smem base address (shared window), the weight block,
// the 128-row hidden buffer, the FP32 vectors, 64 TMEM columns and one mbarrier.
struct InferCta {
    uint32_t base;     // smem_u32 of the dynamic shared memory
    uint32_t w;        // byte offsets within it
    uint32_t h;        // 16 KB, K-major [128][64]
    unsigned char* sm;
    const float* vec;  // b1 | b2 | b3 | w4 | b4
    uint32_t tmem;
    uint64_t* bar;
    uint32_t phase;  // parity of the next barrier completion
    uint32_t* err;
};

// Waits for the MMAs committed on the barrier; every thread learns whether all threads got there.
__device__ __forceinline__ bool wait_mma(InferCta& c) {
    const bool ok = mbar_wait_bounded(c.bar, c.phase, c.err);
    c.phase ^= 1u;
    tc::fence_after_sync();
    return __syncthreads_and(ok) != 0;
}

// Makes this thread's generic-proxy smem writes visible to the tensor cores, then barrier.
__device__ __forceinline__ void publish_smem() {
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
}

// TMEM address of thread t's row: tile t / 128 owns accumulator columns 64 (t / 128) ..+63, and a
// warp may only read its lane quarter, 32 ((t / 32) % 4) .. +31.
__device__ __forceinline__ uint32_t row_tmem(const InferCta& c, int t) {
    return c.tmem + ((uint32_t)(((t >> 5) & 3) * 32) << 16) + 64u * (uint32_t)(t >> 7);
}

// Hidden layer epilogue for this thread's row: 16 columns at a time from TMEM, + bias, the
// activation, BF16 into the K-major hidden buffer (rows of all tiles, 64 columns).
template <int ACT>
__device__ __forceinline__ void hidden_epilogue(const InferCta& c, int t, const float* bias) {
    const uint32_t taddr = row_tmem(c, t);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float z[16];
        tc::ld16(taddr + 16 * q, z);
        uint32_t u[8];
#pragma unroll
        for (int j = 0; j < 8; j += 2) {  // biases four at a time (one broadcast 16-byte load)
            const float4 bb = *reinterpret_cast<const float4*>(bias + 16 * q + 2 * j);
            u[j] = hidden_pair<ACT>(f2(z[2 * j], z[2 * j + 1]), f2(bb.x, bb.y));
            u[j + 1] = hidden_pair<ACT>(f2(z[2 * j + 2], z[2 * j + 3]), f2(bb.z, bb.w));
        }
        *reinterpret_cast<uint4*>(c.sm + c.h + tc::kmajor_offset(t, 16 * q, 64)) = make_uint4(u[0], u[1], u[2], u[3]);
        *reinterpret_cast<uint4*>(c.sm + c.h + tc::kmajor_offset(t, 16 * q + 8, 64)) =
            make_uint4(u[4], u[5], u[6], u[7]);
    }
}

// Logits of NT 128-row tiles: row t (of 128 NT, one per thread of the CTA) of the K-major input
// rows at smem offset x (stride between 8-row groups: 256 bytes), hidden rows at c.h (1024 bytes
// between 8-row groups), tile u's accumulator in TMEM columns 64 u .. 64 u + 63.  Called by all
// 128 NT threads; returns false (every thread) if a tensor-core wait gave up, after which the
// caller frees its TMEM and stops.
template <int NT, int ACT>
__device__ __forceinline__ bool infer_tiles(InferCta& c, uint32_t x, int t, float* logit) {
    constexpr uint32_t id = tc::idesc_bf16(128, 64, false, false);
    // layer 1 (K = 16)
    publish_smem();
    if (t == 0) {
        tc::fence_after_sync();
#pragma unroll
        for (int u = 0; u < NT; ++u)
            tc::mma(c.tmem + 64 * u, tc::smem_desc(c.base + x + 4096 * u, 128, 256),
                    tc::smem_desc(c.base + c.w + kW1, 128, 256), id, false);
        tc::commit(c.bar);
    }
    if (!wait_mma(c)) return false;
    hidden_epilogue<ACT>(c, t, c.vec);
    // layers 2 and 3 (K = 64); layer 2 overwrites the hidden buffer it read once its MMAs are done
#pragma unroll 1
    for (int l = 0; l < 2; ++l) {
        publish_smem();
        if (t == 0) {
            tc::fence_after_sync();
            const uint32_t wb = c.w + (l == 0 ? kW2 : kW3);
#pragma unroll
            for (int u = 0; u < NT; ++u)
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    tc::mma(c.tmem + 64 * u, tc::smem_desc(c.base + c.h + 16384 * u + 256 * s, 128, 1024),
                            tc::smem_desc(c.base + wb + 256 * s, 128, 1024), id, s > 0);
            tc::commit(c.bar);
        }
        if (!wait_mma(c)) return false;
        if (l == 0) hidden_epilogue<ACT>(c, t, c.vec + 64);
    }
    // layer 3 epilogue and the 64 -> 1 output layer on the CUDA cores
    const uint32_t taddr = row_tmem(c, t);
    const float* b3 = c.vec + 128;
    const float* w4 = c.vec + 192;
    uint64_t y2 = f2(c.vec[256], 0.0f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float z[16];
        tc::ld16(taddr + 16 * q, z);
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            const float4 bb = *reinterpret_cast<const float4*>(b3 + 16 * q + 2 * j);
            const float4 ww = *reinterpret_cast<const float4*>(w4 + 16 * q + 2 * j);
            y2 = output_pair<ACT>(f2(z[2 * j], z[2 * j + 1]), f2(bb.x, bb.y), f2(ww.x, ww.y), y2);
            y2 = output_pair<ACT>(f2(z[2 * j + 2], z[2 * j + 3]), f2(bb.z, bb.w), f2(ww.z, ww.w), y2);
        }
    }
    float y0, y1;
    f2_split(y2, y0, y1);
    const float y = y0 + y1;
    // every thread's TMEM reads are done before the next round's MMAs overwrite the accumulators
    tc::fence_before_sync();
    *logit = y;
    return true;
}

template <int ACT>
__device__ __forceinline__ bool infer_tile(InferCta& c, uint32_t x, int t, float* logit) {
    return infer_tiles<1, ACT>(c, x, t, logit);
}

}  // namespace mlp
}  // namespace arc

#endif  // ARC_MLP_TILE_CUH_
