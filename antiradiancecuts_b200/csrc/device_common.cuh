// Device helpers shared by the kernels: vector math, explicitly rounded float ops (for results
// that must match the CPU build bit for bit), error reporting, and the mbarrier + bulk-copy
// (TMA, non-multicast) primitives used to stage AVPL chunks in shared memory.
#ifndef ARC_DEVICE_COMMON_CUH_
#define ARC_DEVICE_COMMON_CUH_

#include <cuda_runtime.h>
#include <stdint.h>

#include "arc_api.h"

namespace arc {

// ---------------------------------------------------------------------------------------
// Explicitly rounded FP32 operations.  nvcc contracts a*b+c into FMA by default; results that
// are compared bit for bit with the CPU oracle (Morton normalisation, tree bounds, cones,
// cut decisions) use these so that every operation rounds as written.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float rn_sqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float rn_dot(float ax, float ay, float az, float bx, float by, float bz) {
    return rn_add(rn_add(rn_mul(ax, bx), rn_mul(ay, by)), rn_mul(az, bz));
}

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ float3 ld3(const ArcFloat3* p, int64_t i) {
    const float* q = reinterpret_cast<const float*>(p) + 3 * i;
    return f3(q[0], q[1], q[2]);
}

__device__ __forceinline__ void set_error(uint32_t* err, uint32_t bit) {
    if (err) atomicOr(err, bit);
}

// ---------------------------------------------------------------------------------------
// mbarrier + cp.async.bulk (global -> shared, one CTA, no multicast)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) into shared memory,
// completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`.  Gives up after `limit` polls (each poll may
// suspend the thread for a short hardware-defined time), records ARC_DEVERR_TIMEOUT and
// returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t* err,
                                                  uint32_t limit = (1u << 24)) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    set_error(err, ARC_DEVERR_TIMEOUT);
    return false;
}

// cp.async (global -> shared, 4 bytes, through L1): one thread's copies complete as a group.
__device__ __forceinline__ void cp_async4(void* dst_smem, const void* src_gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst_smem)), "l"(src_gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// waits until at most N of this thread's most recent groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A CTA whose bounded wait on its ring of `stages` bulk-copy buffers gave up at chunk `fail_c`
// may still have the copies of chunks fail_c .. fail_c + stages - 1 in flight (the issuing thread
// refills a buffer only after its own wait succeeded).  The issuing thread calls this before the
// CTA exits, so that no copy still writes shared memory that the next CTA on the SM may own: one
// more bounded wait per such copy (the phase a copy completes is the one its chunk waits for).
__device__ __forceinline__ void drain_ring_bounded(uint64_t* bars, int stages, int fail_c, int nchunks,
                                                   uint32_t* err) {
    for (int c = fail_c; c < fail_c + stages && c < nchunks; ++c)
        mbar_wait_bounded(&bars[c % stages], (uint32_t)((c / stages) & 1), err);
}

// Packed FP32 pairs (sm_100 f32x2 instructions: two IEEE round-to-nearest operations each, the
// same results as the scalar forms).
__device__ __forceinline__ uint64_t f2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_split(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

constexpr float kOneOverPi = 0.318309886f;  // CUDA_ONE_OVER_PI (cudaUtil.hpp:46-49)
constexpr float kPi = 3.14159265f;          // CUDA_PI

}  // namespace arc

#endif  // ARC_DEVICE_COMMON_CUH_
