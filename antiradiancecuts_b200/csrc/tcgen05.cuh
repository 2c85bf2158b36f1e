// Minimal tcgen05 (5th-generation tensor core) helpers for sm_100a: shared-memory matrix
// descriptors for the no-swizzle core-matrix layouts, the kind::f16 instruction descriptor, MMA
// issue / commit, TMEM allocation and TMEM -> register loads.
//
// Core-matrix layout used by every operand here ("interleaved", no swizzle): an 8-row x 16-byte
// core matrix is 128 contiguous bytes, row r at byte 16 r.  For a K-major operand with R rows
// and K bf16 columns, core matrix (row group g = r / 8, k chunk c = k / 8) sits at
//     g * (K / 8) * 128 + c * 128,
// so LBO (between the two k chunks of one K = 16 step) = 128 B and SBO (between row groups) =
// K / 8 * 128 B.  The same bytes read as an MN-major operand (MN = the row index's partner) use
// LBO' = K / 8 * 128 B between k groups and SBO' = 128 B between MN chunks.
#ifndef ARC_TCGEN05_CUH_
#define ARC_TCGEN05_CUH_

#include <stdint.h>

#include "device_common.cuh"

namespace arc {
namespace tc {

// Shared-memory matrix descriptor (sm_100 "version 1"): start address, leading / stride byte
// offsets (16-byte units), no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;  // descriptor version for sm_100
    return d;                 // base offset 0, legacy LBO mode, layout type 0 = no swizzle
}

// Instruction descriptor of tcgen05.mma.kind::f16 with BF16 A and B and an FP32 accumulator.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn_major, bool b_mn_major) {
    return (1u << 4)                         // D format: F32
           | (1u << 7)                       // A format: BF16
           | (1u << 10)                      // B format: BF16
           | ((a_mn_major ? 1u : 0u) << 15)  // A major-ness
           | ((b_mn_major ? 1u : 0u) << 16)  // B major-ness
           | ((uint32_t)(N >> 3) << 17)      // N / 8
           | ((uint32_t)(M >> 4) << 24);     // M / 16
}

// D[tmem] (=|+=) A[smem] * B[smem]; issued by one thread.
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrive on `bar` once every previously issued MMA of this thread has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by one full warp; the base address is written to *dst (shared memory).
__device__ __forceinline__ void alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w .. 32w + 31).
__device__ __forceinline__ void ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) in a K-major core-matrix layout with K bf16 columns.
__host__ __device__ constexpr uint32_t kmajor_offset(int row, int k, int K) {
    return (uint32_t)((row >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

}  // namespace tc
}  // namespace arc

#endif  // ARC_TCGEN05_CUH_
