// Exclusive prefix sum of int counts on the device, in two launches: block-local offsets with one
// total per block of kScanItems counts (scan_blocks), then an in-place exclusive scan of the block
// totals by one block (scan_totals).  The offset of element i is block_sums[i / kScanItems] +
// offsets[i].  Sums must fit an int.
#ifndef ARC_SCAN_CUH_
#define ARC_SCAN_CUH_

namespace arc {
namespace scan {
namespace {  // internal linkage: every including file gets its own kernels

constexpr int kThreads = 256;
constexpr int kScanItems = 4 * kThreads;

inline int num_blocks(int64_t n) { return (int)((n + kScanItems - 1) / kScanItems); }

__global__ void __launch_bounds__(kThreads) scan_blocks(const int* counts, int64_t n, int* offsets, int* block_sums) {
    __shared__ int warp_sums[kThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanItems + 4 * threadIdx.x;
    int v[4], s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = base + k < n ? counts[base + k] : 0;
        s += v[k];
    }
    // inclusive scan of the thread sums over the block
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        int ws = lane < kThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        if (lane < kThreads / 32) warp_sums[lane] = ws;
    }
    __syncthreads();
    int run = x - s + (w > 0 ? warp_sums[w - 1] : 0);  // exclusive prefix of this thread
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (base + k < n) offsets[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kThreads - 1) block_sums[blockIdx.x] = run;
}

// Exclusive scan of the block totals in place (one block of 1024 threads, any count); *total gets
// their sum.
__global__ void __launch_bounds__(1024) scan_totals(int* block_sums, int nblocks, int* total) {
    __shared__ int carry;
    __shared__ int warp_sums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblocks; b0 += 1024) {
        const int i = b0 + threadIdx.x;
        const int v = i < nblocks ? block_sums[i] : 0;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[w] = x;
        __syncthreads();
        if (w == 0) {
            int ws = warp_sums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += y;
            }
            warp_sums[lane] = ws;
        }
        __syncthreads();
        const int incl = x + (w > 0 ? warp_sums[w - 1] : 0);
        if (i < nblocks) block_sums[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// Launches both kernels on `st`: offsets[n], block_sums[num_blocks(n)], *total (device).
inline void exclusive_scan(const int* counts, int64_t n, int* offsets, int* block_sums, int* total, cudaStream_t st) {
    const int nb = num_blocks(n);
    scan_blocks<<<nb > 0 ? nb : 1, kThreads, 0, st>>>(counts, n, offsets, block_sums);
    scan_totals<<<1, 1024, 0, st>>>(block_sums, nb, total);
}

}  // namespace
}  // namespace scan
}  // namespace arc

#endif  // ARC_SCAN_CUH_
