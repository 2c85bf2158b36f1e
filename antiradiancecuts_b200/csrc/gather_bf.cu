// Brute-force gather: radiance minus antiradiance of every AVPL at every pixel, fused into one
// kernel.  Replaces kernel_radiance_simple + kernel_antiradiance + kernel_combine
// (cudaGather.cu:269-314, 446-557, 782-803) and the cone antiradiance of Shaders/Gather.frag:149-188.
//
// Fast path (Lambertian materials, which every configured scene uses):
//   * AVPLs are first packed into 64-byte records {p, n}, {n, w}, {w, L'}, {A, 1/|w|} with
//     L' = L * (diffuse/pi) of the AVPL's own material (1 for light-source AVPLs), so the AVPL-side
//     BRDF of getRadiance (cudaGather.cu:84-90) is paid once per AVPL instead of once per pair.
//   * The receiver's Lambertian BRDF is constant per pixel and is applied once in the epilogue.
//   * A block owns a 16 x (16*PX) pixel tile; AVPL records are staged chunk by chunk into shared
//     memory with bulk asynchronous copies (cp.async.bulk, no multicast) on an mbarrier ring and
//     read back as broadcast 128-bit loads, each reused for PX pixels per thread.
//   * Radiance and antiradiance go to separate compensated sums (per-chunk FP32 partials folded
//     into Kahan sums, or per-term Kahan) and are combined in FP64.
// General path (specular materials or geometry-term limits): one thread per pixel evaluating the
// full f_r on both sides of every pair.
#include <cfloat>
#include <cmath>

#include "arc_internal.h"
#include "device_common.cuh"
#include "pair_math.cuh"

namespace arc {

namespace {

constexpr int kThreads = 256;
constexpr int kTileW = 16;
constexpr int kStages = 2;

struct BfArgs {
    const float4* records;  // 4 float4 per AVPL
    int32_t n;
    const float4* gpos;
    const float4* gnrm;
    int64_t gpitch;
    int32_t width, height;
    const MaterialRecord* mats;
    int32_t num_mats;
    float3 cam;
    PairConsts pc;       // per-pair constants (cone threshold, clamp, disk radius)
    float cos_thr;       // cone: max(cos(half angle), 0.001)
    float eps;           // cone: 0.001 (Gather.frag:10)
    float clamp2;        // dist_clamp^2, or 0
    float disk_r2;       // disk radius^2
    float disk_scale;    // 1 / (pi r^2)
    float lim_rad;       // GeoTermLimitRadiance or +inf
    float lim_ar;        // GeoTermLimitAntiradiance or +inf
    int32_t chunk;       // AVPL records per stage
    float4* out_res;
    float4* out_rad;
    float4* out_ar;
    double* out_res64;
    double* out_ar64;    // antiradiance in FP64 (3 per pixel), used by the cut path
    int64_t opitch;
    uint32_t* err;
    // general path (raw SoA)
    ArcAvplsGpuParam soa;
    // packed path over a compacted pixel list (nullptr: rectangular tiles)
    const int* pixel_list;
    const int* pixel_count;
};

// ---------------------------------------------------------------------------------------
// pack: SoA -> 64-byte records
// ---------------------------------------------------------------------------------------
// One AVPL's 64-byte record (fields 0..15: p, n, w, L', A, 1/|w|).
__device__ __forceinline__ void bf_record(const ArcAvplsGpuParam& a, const MaterialRecord* mats, int32_t num_mats,
                                          int64_t i, uint32_t* err, float4* r) {
    const float3 p = ld3(a.position, i), nr = ld3(a.normal, i), w = ld3(a.incDirection, i);
    const float3 L = ld3(a.incRadiance, i), A = ld3(a.antiradiance, i);
    int m = a.materialIndex[i];
    if (m < 0 || m >= num_mats) {
        set_error(err, ARC_DEVERR_BAD_MATERIAL);
        m = 0;
    }
    const float4 dif = mats[m].diffuse_exp;
    const float inv_n = rn_div(1.0f, rn_sqrt(rn_dot(nr.x, nr.y, nr.z, nr.x, nr.y, nr.z)));
    const float3 n = f3(rn_mul(nr.x, inv_n), rn_mul(nr.y, inv_n), rn_mul(nr.z, inv_n));
    const float ww = rn_dot(w.x, w.y, w.z, w.x, w.y, w.z);
    const bool light = (ww == 0.0f);
    float3 Lp;
    Lp.x = light ? L.x : rn_mul(L.x, rn_mul(kOneOverPi, dif.x));
    Lp.y = light ? L.y : rn_mul(L.y, rn_mul(kOneOverPi, dif.y));
    Lp.z = light ? L.z : rn_mul(L.z, rn_mul(kOneOverPi, dif.z));
    const float inv_w = light ? 0.0f : rn_div(1.0f, rn_sqrt(ww));
    r[0] = make_float4(p.x, p.y, p.z, n.x);
    r[1] = make_float4(n.y, n.z, w.x, w.y);
    r[2] = make_float4(w.z, Lp.x, Lp.y, Lp.z);
    r[3] = make_float4(A.x, A.y, A.z, inv_w);
}

__global__ void pack_bf_records(ArcAvplsGpuParam a, const MaterialRecord* mats, int32_t num_mats, float4* rec,
                                uint32_t* err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.numAvpls) return;
    float4 r[4];
    bf_record(a, mats, num_mats, i, err, r);
    float4* d = rec + 4 * i;
    d[0] = r[0];
    d[1] = r[1];
    d[2] = r[2];
    d[3] = r[3];
}

// The same records interleaved by AVPL pair: float pair * 32 + 2 f + h holds field f of AVPL
// 2 pair + h; an odd count is padded with a zero record (it contributes exactly 0).
__global__ void pack_bf_pairs(ArcAvplsGpuParam a, const MaterialRecord* mats, int32_t num_mats, float* rec,
                              uint32_t* err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.numAvpls + (a.numAvpls & 1)) return;
    float4 r[4] = {make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0),
                   make_float4(0, 0, 0, 0)};
    if (i < a.numAvpls) bf_record(a, mats, num_mats, i, err, r);
    const float* f = reinterpret_cast<const float*>(r);
    float* d = rec + (i >> 1) * 32 + (i & 1);
#pragma unroll
    for (int q = 0; q < 16; ++q) d[2 * q] = f[q];
}

// PREC: 0 = chunk partials folded into Kahan sums, 1 = per-term Kahan, 2 = naive FP32, 3 = FP64.
// RAD = false skips the radiance sums (antiradiance-only pass of the solid-angle cut path).
template <int AR, int PREC, int PX, bool RAD = true>
__global__ void __launch_bounds__(kThreads) gather_bf_kernel(BfArgs k) {
    using T = typename std::conditional<PREC == 3, double, float>::type;
    extern __shared__ __align__(128) unsigned char smem[];
    float4* stage = reinterpret_cast<float4*>(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)kStages * k.chunk * 64);

    const int tid = threadIdx.x;
    const int tx = tid % kTileW, ty = tid / kTileW;
    const int x = blockIdx.x * kTileW + tx;
    const int rows = kThreads / kTileW;  // 16
    const int ybase = blockIdx.y * rows * PX + ty;

    const int nchunks = (k.n + k.chunk - 1) / k.chunk;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int c = 0; c < kStages && c < nchunks; ++c) {
            const int cnt = min(k.chunk, k.n - c * k.chunk);
            mbar_arrive_expect_tx(&bars[c], (uint32_t)cnt * 64u);
            bulk_g2s(stage + (size_t)c * k.chunk * 4, k.records + (size_t)c * k.chunk * 4, (uint32_t)cnt * 64u,
                     &bars[c]);
        }
    }

    Pixel<T> pix[PX];
    float sc[PX][6];  // Kahan compensation (PREC 0/1)
    float ss[PX][6];  // Kahan running sums (PREC 0)
    bool valid[PX];
    int mat[PX];
#pragma unroll
    for (int j = 0; j < PX; ++j) {
        const int y = ybase + j * rows;
        valid[j] = (x < k.width && y < k.height);
        mat[j] = 0;
        float4 gp = make_float4(0, 0, 0, 0), gn = make_float4(0, 0, 0, 0);
        if (valid[j]) {
            gp = k.gpos[(int64_t)y * k.gpitch + x];
            gn = k.gnrm[(int64_t)y * k.gpitch + x];
            mat[j] = (int)gn.w;
            if (mat[j] <= 0 || mat[j] >= k.num_mats) {
                if (mat[j] != 0) set_error(k.err, ARC_DEVERR_BAD_MATERIAL);
                valid[j] = false;
            }
        }
        T nx = 0, ny = 0, nz = 0;
        if (valid[j]) {
            const T l = rsqrt_t<T>((T)gn.x * gn.x + (T)gn.y * gn.y + (T)gn.z * gn.z);
            nx = gn.x * l;
            ny = gn.y * l;
            nz = gn.z * l;
        }
        pix[j].px = gp.x;
        pix[j].py = gp.y;
        pix[j].pz = gp.z;
        pix[j].nx = nx;
        pix[j].ny = ny;
        pix[j].nz = nz;
        pix[j].r0 = pix[j].r1 = pix[j].r2 = pix[j].a0 = pix[j].a1 = pix[j].a2 = 0;
#pragma unroll
        for (int c = 0; c < 6; ++c) sc[j][c] = ss[j][c] = 0.0f;
    }

    bool ok = true;
    int fail_c = -1;  // first chunk whose wait gave up
    for (int c = 0; c < nchunks; ++c) {
        const int s = c % kStages;
        const uint32_t parity = (uint32_t)((c / kStages) & 1);
        if (ok) {
            ok = mbar_wait_bounded(&bars[s], parity, k.err);
            if (!ok) fail_c = c;
        }
        if (ok) {
            const int cnt = min(k.chunk, k.n - c * k.chunk);
            const float4* rec = stage + (size_t)s * k.chunk * 4;
#pragma unroll 2
            for (int i = 0; i < cnt; ++i) {
                const float4 q0 = rec[4 * i + 0], q1 = rec[4 * i + 1], q2 = rec[4 * i + 2], q3 = rec[4 * i + 3];
#pragma unroll
                for (int j = 0; j < PX; ++j) {
                    T g, ga;
                    pair_terms<AR, T>(q0, q1, q2, q3, pix[j], k.pc, g, ga);
                    if (PREC == 1) {
                        if (RAD) {
                            kahan_add(ss[j][0], sc[j][0], (float)(q2.y * g));
                            kahan_add(ss[j][1], sc[j][1], (float)(q2.z * g));
                            kahan_add(ss[j][2], sc[j][2], (float)(q2.w * g));
                        }
                        if (AR != ARC_AR_NONE) {
                            kahan_add(ss[j][3], sc[j][3], (float)(q3.x * ga));
                            kahan_add(ss[j][4], sc[j][4], (float)(q3.y * ga));
                            kahan_add(ss[j][5], sc[j][5], (float)(q3.z * ga));
                        }
                    } else {
                        if (RAD) {
                            pix[j].r0 += (T)q2.y * g;
                            pix[j].r1 += (T)q2.z * g;
                            pix[j].r2 += (T)q2.w * g;
                        }
                        if (AR != ARC_AR_NONE) {
                            pix[j].a0 += (T)q3.x * ga;
                            pix[j].a1 += (T)q3.y * ga;
                            pix[j].a2 += (T)q3.z * ga;
                        }
                    }
                }
            }
            if (PREC == 0) {
#pragma unroll
                for (int j = 0; j < PX; ++j) {
                    kahan_add(ss[j][0], sc[j][0], (float)pix[j].r0);
                    kahan_add(ss[j][1], sc[j][1], (float)pix[j].r1);
                    kahan_add(ss[j][2], sc[j][2], (float)pix[j].r2);
                    kahan_add(ss[j][3], sc[j][3], (float)pix[j].a0);
                    kahan_add(ss[j][4], sc[j][4], (float)pix[j].a1);
                    kahan_add(ss[j][5], sc[j][5], (float)pix[j].a2);
                    pix[j].r0 = pix[j].r1 = pix[j].r2 = pix[j].a0 = pix[j].a1 = pix[j].a2 = 0;
                }
            }
        }
        __syncthreads();  // every thread is done reading stage s before it is refilled
        if (tid == 0 && ok && c + kStages < nchunks) {
            fence_proxy_async_smem();
            const int cn = c + kStages;
            const int cnt = min(k.chunk, k.n - cn * k.chunk);
            mbar_arrive_expect_tx(&bars[s], (uint32_t)cnt * 64u);
            bulk_g2s(stage + (size_t)s * k.chunk * 4, k.records + (size_t)cn * k.chunk * 4, (uint32_t)cnt * 64u,
                     &bars[s]);
        }
    }
    // the copies the ring still has in flight after a wait gave up (only thread 0 issues them)
    if (tid == 0 && fail_c >= 0) drain_ring_bounded(bars, kStages, fail_c, nchunks, k.err);

    // epilogue: receiver BRDF, signed combine, stores
#pragma unroll
    for (int j = 0; j < PX; ++j) {
        const int y = ybase + j * rows;
        if (x >= k.width || y >= k.height) continue;
        double rad[3] = {0, 0, 0}, ar[3] = {0, 0, 0}, res[3] = {0, 0, 0};
        float radf[3] = {0, 0, 0}, arf[3] = {0, 0, 0}, resf[3] = {0, 0, 0};
        if (valid[j]) {
            const float4 d = k.mats[mat[j]].diffuse_exp;
            const float kd[3] = {kOneOverPi * d.x, kOneOverPi * d.y, kOneOverPi * d.z};
            const float arscale = (AR == ARC_AR_DISK) ? k.disk_scale : 1.0f;
            if (PREC == 2) {
                const float S[6] = {(float)pix[j].r0, (float)pix[j].r1, (float)pix[j].r2,
                                    (float)pix[j].a0, (float)pix[j].a1, (float)pix[j].a2};
                for (int c = 0; c < 3; ++c) {
                    radf[c] = kd[c] * S[c];
                    arf[c] = kd[c] * arscale * S[3 + c];
                    resf[c] = radf[c] - arf[c];
                    rad[c] = radf[c];
                    ar[c] = arf[c];
                    res[c] = resf[c];
                }
            } else {
                double S[6];
                if (PREC == 3) {
                    S[0] = (double)pix[j].r0; S[1] = (double)pix[j].r1; S[2] = (double)pix[j].r2;
                    S[3] = (double)pix[j].a0; S[4] = (double)pix[j].a1; S[5] = (double)pix[j].a2;
                } else {
                    for (int c = 0; c < 6; ++c) S[c] = (double)ss[j][c] - (double)sc[j][c];
                }
                for (int c = 0; c < 3; ++c) {
                    rad[c] = (double)kd[c] * S[c];
                    ar[c] = (double)kd[c] * (double)arscale * S[3 + c];
                    res[c] = rad[c] - ar[c];
                    radf[c] = (float)rad[c];
                    arf[c] = (float)ar[c];
                    resf[c] = (float)res[c];
                }
            }
        }
        const int64_t o = (int64_t)y * k.opitch + x;
        if (k.out_res) k.out_res[o] = make_float4(resf[0], resf[1], resf[2], 1.0f);
        if (k.out_rad) k.out_rad[o] = make_float4(radf[0], radf[1], radf[2], 1.0f);
        if (k.out_ar) k.out_ar[o] = make_float4(arf[0], arf[1], arf[2], 1.0f);
        if (k.out_res64) {
            k.out_res64[3 * o + 0] = res[0];
            k.out_res64[3 * o + 1] = res[1];
            k.out_res64[3 * o + 2] = res[2];
        }
        if (k.out_ar64) {
            k.out_ar64[3 * o + 0] = ar[0];
            k.out_ar64[3 * o + 1] = ar[1];
            k.out_ar64[3 * o + 2] = ar[2];
        }
    }
}

// Surface pixels of the G-buffer, compacted into a list (order within a warp arbitrary), for the
// list form of the packed kernel; every other pixel gets here the outputs the gather gives a pixel
// without a surface (0, w = 1).  Bad material indices are reported as the gather kernels do.
__global__ void bf_compact_pixels(BfArgs k, int* list, int* count) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    const int lane = threadIdx.x & 31;
    bool valid = x < k.width;
    if (valid) {
        const int m = (int)k.gnrm[(int64_t)y * k.gpitch + x].w;
        if (m <= 0 || m >= k.num_mats) {
            if (m != 0) set_error(k.err, ARC_DEVERR_BAD_MATERIAL);
            valid = false;
        }
    }
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    int base = 0;
    if (vm) {
        const int leader = __ffs(vm) - 1;
        if (lane == leader) base = atomicAdd(count, __popc(vm));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    if (valid) {
        list[base + __popc(vm & ((1u << lane) - 1u))] = y * k.width + x;
    } else if (x < k.width) {
        const int64_t o = (int64_t)y * k.opitch + x;
        const float4 z = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        if (k.out_res) k.out_res[o] = z;
        if (k.out_rad) k.out_rad[o] = z;
        if (k.out_ar) k.out_ar[o] = z;
        if (k.out_res64) k.out_res64[3 * o] = k.out_res64[3 * o + 1] = k.out_res64[3 * o + 2] = 0.0;
        if (k.out_ar64) k.out_ar64[3 * o] = k.out_ar64[3 * o + 1] = k.out_ar64[3 * o + 2] = 0.0;
    }
}

// ---------------------------------------------------------------------------------------
// Packed FP32x2 variant of the default path (per-chunk partials folded into Kahan sums, no or cone
// antiradiance).  Records come from pack_bf_pairs, so one 16-byte shared load brings two fields of
// two AVPLs, and each thread evaluates two AVPLs per step for each of its PX pixels with
// add/mul/fma.rn.f32x2 (sm_100).  Same terms as pair_terms; within a chunk the even and odd AVPLs
// are summed apart and added before the chunk's Kahan step.
// ---------------------------------------------------------------------------------------
// LIST: the block takes kThreads * PX consecutive entries of the compacted list of surface pixels
// (bf_compact_pixels) instead of a 16 x 16 PX rectangle.
template <int AR, int PX, bool LIST>
__global__ void __launch_bounds__(kThreads) gather_bf_packed_kernel(BfArgs k) {
    extern __shared__ __align__(128) unsigned char smem[];
    float* stage = reinterpret_cast<float*>(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)kStages * k.chunk * 64);

    const int tid = threadIdx.x;
    const int tx = tid % kTileW, ty = tid / kTileW;
    const int rows = kThreads / kTileW;  // 16
    const int64_t lbase = (int64_t)blockIdx.x * kThreads * PX;
    int list_n = 0;
    if (LIST) {
        list_n = *k.pixel_count;
        if (lbase >= list_n) return;  // uniform: before any barrier
    }
    // pixel j of this thread
    auto pixel_xy = [&](int j, int& px_, int& py_) {
        if (LIST) {
            const int64_t e = lbase + (int64_t)j * kThreads + tid;
            const int idx = e < list_n ? k.pixel_list[e] : -1;
            px_ = idx >= 0 ? idx % k.width : k.width;  // past the image: no pixel
            py_ = idx >= 0 ? idx / k.width : 0;
        } else {
            px_ = blockIdx.x * kTileW + tx;
            py_ = blockIdx.y * rows * PX + ty + j * rows;
        }
    };

    const int npad = k.n + (k.n & 1);  // records incl. the zero pad; k.chunk is even
    const int nchunks = (npad + k.chunk - 1) / k.chunk;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int c = 0; c < kStages && c < nchunks; ++c) {
            const int cnt = min(k.chunk, npad - c * k.chunk);
            mbar_arrive_expect_tx(&bars[c], (uint32_t)cnt * 64u);
            bulk_g2s(stage + (size_t)c * k.chunk * 16, k.records + (size_t)c * k.chunk * 4, (uint32_t)cnt * 64u,
                     &bars[c]);
        }
    }

    uint64_t PXc[PX], PYc[PX], PZc[PX], NXc[PX], NYc[PX], NZc[PX];
    float sc[PX][6], ss[PX][6];
    bool valid[PX];
    int mat[PX];
#pragma unroll
    for (int j = 0; j < PX; ++j) {
        int x, y;
        pixel_xy(j, x, y);
        valid[j] = (x < k.width && y < k.height);
        mat[j] = 0;
        float4 gp = make_float4(0, 0, 0, 0), gn = make_float4(0, 0, 0, 0);
        if (valid[j]) {
            gp = k.gpos[(int64_t)y * k.gpitch + x];
            gn = k.gnrm[(int64_t)y * k.gpitch + x];
            mat[j] = (int)gn.w;
            if (mat[j] <= 0 || mat[j] >= k.num_mats) {
                if (mat[j] != 0) set_error(k.err, ARC_DEVERR_BAD_MATERIAL);
                valid[j] = false;
            }
        }
        float nx = 0.0f, ny = 0.0f, nz = 0.0f;
        if (valid[j]) {
            const float l = rsqrtf(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z);
            nx = gn.x * l;
            ny = gn.y * l;
            nz = gn.z * l;
        }
        PXc[j] = f2(-gp.x, -gp.x);
        PYc[j] = f2(-gp.y, -gp.y);
        PZc[j] = f2(-gp.z, -gp.z);
        NXc[j] = f2(nx, nx);
        NYc[j] = f2(ny, ny);
        NZc[j] = f2(nz, nz);
#pragma unroll
        for (int c = 0; c < 6; ++c) sc[j][c] = ss[j][c] = 0.0f;
    }
    const float cos_thr = k.pc.cos_thr, eps = k.pc.eps, inv_clamp2 = k.pc.inv_clamp2;
    // distance floor folded into the FMA chain: l2 + 1e-30 equals max(l2, 1e-30) for l2 above ~1e-23
    const uint64_t kTiny2 = f2(1e-30f, 1e-30f);

    bool ok = true;
    int fail_c = -1;  // first chunk whose wait gave up
    for (int c = 0; c < nchunks; ++c) {
        const int s = c % kStages;
        const uint32_t parity = (uint32_t)((c / kStages) & 1);
        if (ok) {
            ok = mbar_wait_bounded(&bars[s], parity, k.err);
            if (!ok) fail_c = c;
        }
        if (ok) {
            const int pairs = min(k.chunk, npad - c * k.chunk) >> 1;
            const float* st = stage + (size_t)s * k.chunk * 16;
            uint64_t acc[PX][6];
#pragma unroll
            for (int j = 0; j < PX; ++j)
#pragma unroll
                for (int q = 0; q < 6; ++q) acc[j][q] = 0;  // packed zeros
#pragma unroll 2
            for (int pr = 0; pr < pairs; ++pr) {
                const ulonglong2* s2 = reinterpret_cast<const ulonglong2*>(st + pr * 32);
                const ulonglong2 f01 = s2[0], f23 = s2[1], f45 = s2[2], f89 = s2[4], f1011 = s2[5];
#pragma unroll
                for (int j = 0; j < PX; ++j) {
                    const uint64_t dx = f2_add(f01.x, PXc[j]), dy = f2_add(f01.y, PYc[j]), dz = f2_add(f23.x, PZc[j]);
                    const uint64_t l2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_fma(dx, dx, kTiny2)));  // >= 1e-30
                    float l2a, l2b;
                    f2_split(l2, l2a, l2b);
                    const uint64_t r = f2(rsqrtf(l2a), rsqrtf(l2b));
                    const uint64_t c1 = f2_mul(f2_fma(NZc[j], dz, f2_fma(NYc[j], dy, f2_mul(NXc[j], dx))), r);
                    const uint64_t c2n = f2_mul(f2_fma(f45.y, dz, f2_fma(f45.x, dy, f2_mul(f23.y, dx))), r);
                    float c1a, c1b, c2a, c2b, rra, rrb, ia, ib;
                    f2_split(c1, c1a, c1b);
                    f2_split(c2n, c2a, c2b);
                    f2_split(f2_mul(r, r), rra, rrb);
                    const uint64_t inv = f2(fminf(rra, inv_clamp2), fminf(rrb, inv_clamp2));
                    // c1 / max(d^2, clamp^2): the radiance term's receiver factor and the cone term itself
                    f2_split(f2_mul(c1, inv), ia, ib);
                    const uint64_t g = f2_mul(f2(fmaxf(ia, 0.0f), fmaxf(ib, 0.0f)), f2(fmaxf(-c2a, 0.0f), fmaxf(-c2b, 0.0f)));
                    acc[j][0] = f2_fma(f89.y, g, acc[j][0]);
                    acc[j][1] = f2_fma(f1011.x, g, acc[j][1]);
                    acc[j][2] = f2_fma(f1011.y, g, acc[j][2]);
                    if (AR == ARC_AR_CONE) {
                        const ulonglong2 f67 = s2[3], f1213 = s2[6], f1415 = s2[7];
                        const uint64_t wdr = f2_mul(f2_fma(f89.x, dz, f2_fma(f67.y, dy, f2_mul(f67.x, dx))), r);
                        float wa, wb;
                        f2_split(wdr, wa, wb);
                        const uint64_t ga = f2((-wa > cos_thr && c1a > eps) ? ia : 0.0f,
                                               (-wb > cos_thr && c1b > eps) ? ib : 0.0f);
                        acc[j][3] = f2_fma(f1213.x, ga, acc[j][3]);
                        acc[j][4] = f2_fma(f1213.y, ga, acc[j][4]);
                        acc[j][5] = f2_fma(f1415.x, ga, acc[j][5]);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < PX; ++j)
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    float lo, hi;
                    f2_split(acc[j][q], lo, hi);
                    kahan_add(ss[j][q], sc[j][q], lo + hi);
                }
        }
        __syncthreads();  // every thread is done reading stage s before it is refilled
        if (tid == 0 && ok && c + kStages < nchunks) {
            fence_proxy_async_smem();
            const int cn = c + kStages;
            const int cnt = min(k.chunk, npad - cn * k.chunk);
            mbar_arrive_expect_tx(&bars[s], (uint32_t)cnt * 64u);
            bulk_g2s(stage + (size_t)s * k.chunk * 16, k.records + (size_t)cn * k.chunk * 4, (uint32_t)cnt * 64u,
                     &bars[s]);
        }
    }
    // the copies the ring still has in flight after a wait gave up (only thread 0 issues them)
    if (tid == 0 && fail_c >= 0) drain_ring_bounded(bars, kStages, fail_c, nchunks, k.err);

    // epilogue: receiver BRDF, FP64 signed combine, stores
#pragma unroll
    for (int j = 0; j < PX; ++j) {
        int x, y;
        pixel_xy(j, x, y);
        if (x >= k.width || y >= k.height) continue;
        double rad[3] = {0, 0, 0}, ar[3] = {0, 0, 0}, res[3] = {0, 0, 0};
        if (valid[j]) {
            const float4 d = k.mats[mat[j]].diffuse_exp;
            const float kd[3] = {kOneOverPi * d.x, kOneOverPi * d.y, kOneOverPi * d.z};
            for (int c = 0; c < 3; ++c) {
                rad[c] = (double)kd[c] * ((double)ss[j][c] - (double)sc[j][c]);
                ar[c] = (double)kd[c] * ((double)ss[j][3 + c] - (double)sc[j][3 + c]);
                res[c] = rad[c] - ar[c];
            }
        }
        const int64_t o = (int64_t)y * k.opitch + x;
        if (k.out_res) k.out_res[o] = make_float4((float)res[0], (float)res[1], (float)res[2], 1.0f);
        if (k.out_rad) k.out_rad[o] = make_float4((float)rad[0], (float)rad[1], (float)rad[2], 1.0f);
        if (k.out_ar) k.out_ar[o] = make_float4((float)ar[0], (float)ar[1], (float)ar[2], 1.0f);
        if (k.out_res64) {
            k.out_res64[3 * o + 0] = res[0];
            k.out_res64[3 * o + 1] = res[1];
            k.out_res64[3 * o + 2] = res[2];
        }
        if (k.out_ar64) {
            k.out_ar64[3 * o + 0] = ar[0];
            k.out_ar64[3 * o + 1] = ar[1];
            k.out_ar64[3 * o + 2] = ar[2];
        }
    }
}

// ---------------------------------------------------------------------------------------
// General path: full f_r on both sides (cudaGather.cu:59-95), geometry-term limits
// (Gather.frag:182, 190-194); one thread per pixel over the raw SoA arrays.
// ---------------------------------------------------------------------------------------
template <typename T>
struct V {
    T x, y, z;
};
template <typename T>
__device__ __forceinline__ V<T> vsub(V<T> a, V<T> b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename T>
__device__ __forceinline__ V<T> vs(T s, V<T> a) {
    return {s * a.x, s * a.y, s * a.z};
}
template <typename T>
__device__ __forceinline__ T vdot(V<T> a, V<T> b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T>
__device__ __forceinline__ V<T> vnorm(V<T> a) {
    return vs(rsqrt_t<T>(vdot(a, a)), a);
}

// f_r(w_i, w_o, n, mat) = diffuse/pi + [|spec| > 0] (e+2)/(2 pi) max(0, reflect(-w_i, n).w_o)^e spec
template <typename T>
__device__ __forceinline__ V<T> brdf(V<T> w_i, V<T> w_o, V<T> n, const MaterialRecord& m) {
    V<T> d = {(T)kOneOverPi * m.diffuse_exp.x, (T)kOneOverPi * m.diffuse_exp.y, (T)kOneOverPi * m.diffuse_exp.z};
    if (m.specular_flag.w != 0.0f) {
        const V<T> I = vs((T)-1, w_i);
        const V<T> r = vsub(I, vs((T)2 * vdot(n, I), n));
        T c = vdot(r, w_o);
        c = c > (T)0 ? c : (T)0;
        const T e = m.diffuse_exp.w;
        const T f = (T)0.5 * (T)kOneOverPi * (e + (T)2) * (T)pow(c, e);
        d.x += f * m.specular_flag.x;
        d.y += f * m.specular_flag.y;
        d.z += f * m.specular_flag.z;
    }
    return d;
}

template <int AR, typename T>
__global__ void __launch_bounds__(kThreads) gather_general_kernel(BfArgs k) {
    __shared__ MaterialRecord smat[ARC_MAX_MATERIALS];
    for (int i = threadIdx.x; i < k.num_mats; i += blockDim.x) smat[i] = k.mats[i];
    __syncthreads();
    const int x = blockIdx.x * kTileW + threadIdx.x % kTileW;
    const int y = blockIdx.y * (kThreads / kTileW) + threadIdx.x / kTileW;
    if (x >= k.width || y >= k.height) return;
    const float4 gp = k.gpos[(int64_t)y * k.gpitch + x];
    const float4 gn = k.gnrm[(int64_t)y * k.gpitch + x];
    const int m = (int)gn.w;
    double rad[3] = {0, 0, 0}, ar[3] = {0, 0, 0};
    if (m > 0 && m < k.num_mats) {
        const V<T> p = {(T)gp.x, (T)gp.y, (T)gp.z};
        const V<T> n = vnorm(V<T>{(T)gn.x, (T)gn.y, (T)gn.z});
        const V<T> cam = {(T)k.cam.x, (T)k.cam.y, (T)k.cam.z};
        const V<T> w_o = vnorm(vsub(cam, p));
        T s[6] = {0, 0, 0, 0, 0, 0};
        float c[6] = {0, 0, 0, 0, 0, 0};
        const ArcAvplsGpuParam& a = k.soa;
        for (int i = 0; i < a.numAvpls; ++i) {
            const float3 fpa = ld3(a.position, i), fna = ld3(a.normal, i), fwa = ld3(a.incDirection, i);
            const V<T> pa = {(T)fpa.x, (T)fpa.y, (T)fpa.z};
            const V<T> na = vnorm(V<T>{(T)fna.x, (T)fna.y, (T)fna.z});
            const V<T> wa = {(T)fwa.x, (T)fwa.y, (T)fwa.z};
            int ma = a.materialIndex[i];
            if (ma < 0 || ma >= k.num_mats) ma = 0;
            const V<T> v = vsub(pa, p);
            T l2 = vdot(v, v);
            if (!(l2 > (T)0)) continue;
            const V<T> w = vs(rsqrt_t<T>(l2), v);  // pixel -> AVPL
            const V<T> fr = brdf<T>(w, w_o, n, smat[m]);
            // radiance
            V<T> fl = {1, 1, 1};
            if (vdot(wa, wa) != (T)0) fl = brdf<T>(vs((T)-1, wa), vs((T)-1, w), na, smat[ma]);
            T c1 = vdot(n, w), c2 = -vdot(na, w);
            c1 = c1 < (T)0 ? (T)0 : (c1 > (T)1 ? (T)1 : c1);
            c2 = c2 < (T)0 ? (T)0 : (c2 > (T)1 ? (T)1 : c2);
            const T l2c = l2 < (T)k.clamp2 ? (T)k.clamp2 : l2;
            T g = c1 * c2 / l2c;
            if (g > (T)k.lim_rad) g = (T)k.lim_rad;
            const float3 L = ld3(a.incRadiance, i), A = ld3(a.antiradiance, i);
            T term[6];
            term[0] = (T)L.x * fl.x * fr.x * g;
            term[1] = (T)L.y * fl.y * fr.y * g;
            term[2] = (T)L.z * fl.z * fr.z * g;
            T ga = 0;
            if (AR == ARC_AR_CONE) {
                const T cw = -vdot(w, wa);
                const T cn = vdot(n, w);
                if (cw > (T)k.eps && cn > (T)k.eps && cw > (T)k.cos_thr) {
                    ga = cn / l2c;
                    if (ga > (T)k.lim_ar) ga = (T)k.lim_ar;
                }
            } else if (AR == ARC_AR_DISK) {
                const T wn = vdot(wa, n);
                if (wn != (T)0) {
                    const T t = -vdot(v, n) / wn;
                    const V<T> wu = vnorm(wa);
                    const V<T> h = {pa.x + t * wu.x, pa.y + t * wu.y, pa.z + t * wu.z};
                    const V<T> hp = vsub(h, p);
                    if (t > (T)0 && vdot(hp, hp) < (T)k.disk_r2 && wn < (T)0 && -vdot(w, na) < (T)0) ga = (T)k.disk_scale;
                }
            }
            term[3] = (T)A.x * fr.x * ga;
            term[4] = (T)A.y * fr.y * ga;
            term[5] = (T)A.z * fr.z * ga;
            if (sizeof(T) == 8) {
                for (int q = 0; q < 6; ++q) s[q] += term[q];
            } else {
                for (int q = 0; q < 6; ++q) {
                    float ssq = (float)s[q];
                    kahan_add(ssq, c[q], (float)term[q]);
                    s[q] = (T)ssq;
                }
            }
        }
        for (int q = 0; q < 3; ++q) {
            rad[q] = (double)s[q] - (double)c[q];
            ar[q] = (double)s[3 + q] - (double)c[3 + q];
        }
    }
    const int64_t o = (int64_t)y * k.opitch + x;
    const double res[3] = {rad[0] - ar[0], rad[1] - ar[1], rad[2] - ar[2]};
    if (k.out_res) k.out_res[o] = make_float4((float)res[0], (float)res[1], (float)res[2], 1.0f);
    if (k.out_rad) k.out_rad[o] = make_float4((float)rad[0], (float)rad[1], (float)rad[2], 1.0f);
    if (k.out_ar) k.out_ar[o] = make_float4((float)ar[0], (float)ar[1], (float)ar[2], 1.0f);
    if (k.out_res64) {
        k.out_res64[3 * o + 0] = res[0];
        k.out_res64[3 * o + 1] = res[1];
        k.out_res64[3 * o + 2] = res[2];
    }
}

// Tile shapes selectable by ArcGatherParams::tile_config: pixels per thread x AVPLs per stage.
struct TileShape {
    int px;
    int chunk;
};
constexpr TileShape kTileShapes[] = {{1, 128}, {2, 128}, {2, 256}, {4, 128}, {4, 256}, {1, 256}, {2, 64},
                                     {4, 64},  {1, 512}, {2, 512}, {4, 512}, {1, 1024}, {2, 1024}};
constexpr int kNumTileShapes = sizeof(kTileShapes) / sizeof(kTileShapes[0]);
constexpr int kDefaultTileShape = 2;

template <int AR, int PREC, int PX, bool RAD = true>
arc_status launch_fast(const BfArgs& a, cudaStream_t st) {
    const size_t smem = (size_t)kStages * a.chunk * 64 + kStages * sizeof(uint64_t);
    auto fn = gather_bf_kernel<AR, PREC, PX, RAD>;
    if (smem > 48 * 1024) ARC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((a.width + kTileW - 1) / kTileW, (a.height + 16 * PX - 1) / (16 * PX));
    fn<<<grid, kThreads, smem, st>>>(a);
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

template <int AR, int PREC>
arc_status launch_fast_px(const BfArgs& a, int px, cudaStream_t st) {
    if (px == 1) return launch_fast<AR, PREC, 1>(a, st);
    if (px == 2) return launch_fast<AR, PREC, 2>(a, st);
    return launch_fast<AR, PREC, 4>(a, st);
}

template <int AR>
arc_status launch_fast_prec(const BfArgs& a, int prec, int px, cudaStream_t st) {
    switch (prec) {
        case 0: return launch_fast_px<AR, 0>(a, px, st);
        case 1: return launch_fast_px<AR, 1>(a, px, st);
        case 2: return launch_fast_px<AR, 2>(a, px, st);
        default: return launch_fast<AR, 3, 1>(a, st);
    }
}

// the packed kernel serves the default precision with no or cone antiradiance
bool use_packed(const ArcGatherParams& p) { return p.precision == ARC_PREC_KAHAN && p.ar_kind != ARC_AR_DISK; }

template <int AR, int PX>
arc_status launch_packed(const BfArgs& a, cudaStream_t st) {
    const size_t smem = (size_t)kStages * a.chunk * 64 + kStages * sizeof(uint64_t);
    if (a.pixel_list) {  // one block per kThreads * PX listed pixels; blocks past the count return
        auto fn = gather_bf_packed_kernel<AR, PX, true>;
        if (smem > 48 * 1024)
            ARC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int64_t pixels = (int64_t)a.width * a.height;
        fn<<<(unsigned)((pixels + kThreads * PX - 1) / (kThreads * PX)), kThreads, smem, st>>>(a);
    } else {
        auto fn = gather_bf_packed_kernel<AR, PX, false>;
        if (smem > 48 * 1024)
            ARC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        dim3 grid((a.width + kTileW - 1) / kTileW, (a.height + 16 * PX - 1) / (16 * PX));
        fn<<<grid, kThreads, smem, st>>>(a);
    }
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

template <int AR>
arc_status launch_packed_px(const BfArgs& a, int px, cudaStream_t st) {
    if (px == 1) return launch_packed<AR, 1>(a, st);
    if (px == 2) return launch_packed<AR, 2>(a, st);
    return launch_packed<AR, 4>(a, st);
}

// dispatch of the fast path (records packed by pack_bf_pairs when use_packed(p), else by
// pack_bf_records)
arc_status launch_fast_path(const BfArgs& a, const ArcGatherParams& p, int px, cudaStream_t st) {
    if (use_packed(p)) return p.ar_kind == ARC_AR_NONE ? launch_packed_px<0>(a, px, st) : launch_packed_px<2>(a, px, st);
    switch (p.ar_kind) {
        case 0: return launch_fast_prec<0>(a, p.precision, px, st);
        case 1: return launch_fast_prec<1>(a, p.precision, px, st);
        default: return launch_fast_prec<2>(a, p.precision, px, st);
    }
}

BfArgs make_args(arc_context* ctx, const GatherLaunch& g);
arc_status pack_records(arc_context* ctx, const GatherLaunch& g, BfArgs& a, bool pairs);

}  // namespace

int bf_num_tile_shapes() { return kNumTileShapes; }

arc_status launch_gather_bruteforce(arc_context* ctx, const GatherLaunch& g) {
    const ArcGatherParams& p = *g.params;
    const ArcGBufferView& gb = *g.gbuffer;
    const ArcOutputView& out = *g.out;
    ARC_CHECK_ARG(p.ar_kind >= 0 && p.ar_kind <= 2, "ar_kind out of range");
    ARC_CHECK_ARG(p.precision >= 0 && p.precision <= 3, "precision out of range");
    ARC_CHECK_ARG(p.tile_config >= -1 && p.tile_config < kNumTileShapes, "tile_config out of range");
    ARC_CHECK_ARG(gb.width > 0 && gb.height > 0 && gb.pitch >= gb.width && gb.position && gb.normal,
                  "bad G-buffer view");
    ARC_CHECK_ARG(out.pitch >= gb.width && (out.result || out.radiance || out.antiradiance || out.result_fp64),
                  "bad output view");
    ARC_CHECK_ARG(g.avpls->numAvpls >= 0, "negative AVPL count");
    ARC_CHECK_ARG(ctx->num_materials > 0, "materials not uploaded");
    ARC_CHECK_ARG(p.ar_kind != ARC_AR_DISK || p.disk_radius > 0.0f, "disk radius must be > 0");
    ARC_CHECK_ARG(reinterpret_cast<uintptr_t>(gb.position) % 16 == 0 && reinterpret_cast<uintptr_t>(gb.normal) % 16 == 0,
                  "G-buffer planes must be 16-byte aligned");

    BfArgs a = make_args(ctx, g);
    const bool general = ctx->any_specular || p.geo_limit_radiance > 0.0f || p.geo_limit_antiradiance > 0.0f;
    cudaStream_t st = ctx->stream;
    if (general) {
        dim3 grid((gb.width + kTileW - 1) / kTileW, (gb.height + 15) / 16);
        stage_begin(ctx, "bf_general");
        if (p.precision == ARC_PREC_FP64) {
            if (p.ar_kind == 0) gather_general_kernel<0, double><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 1) gather_general_kernel<1, double><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 2) gather_general_kernel<2, double><<<grid, kThreads, 0, st>>>(a);
        } else {
            if (p.ar_kind == 0) gather_general_kernel<0, float><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 1) gather_general_kernel<1, float><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 2) gather_general_kernel<2, float><<<grid, kThreads, 0, st>>>(a);
        }
        stage_end(ctx, 1);
        ARC_TRY_CUDA(cudaGetLastError());
        return ARC_OK;
    }
    ARC_TRY(pack_records(ctx, g, a, use_packed(p)));
    const int shape = p.tile_config >= 0 ? p.tile_config : (ctx->bf_tile_config >= 0 ? ctx->bf_tile_config : kDefaultTileShape);
    const TileShape ts = kTileShapes[shape];
    a.chunk = ts.chunk;
    if (use_packed(p)) {  // only surface pixels are gathered
        int *list = nullptr, *count = nullptr;
        ARC_TRY(ctx->arena.get("bf_pixel_list", sizeof(int) * (size_t)gb.width * gb.height,
                               reinterpret_cast<void**>(&list)));
        ARC_TRY(ctx->arena.get("bf_pixel_count", sizeof(int), reinterpret_cast<void**>(&count)));
        ARC_TRY_CUDA(cudaMemsetAsync(count, 0, sizeof(int), st));
        stage_begin(ctx, "bf_pixels");
        bf_compact_pixels<<<dim3((gb.width + 255) / 256, gb.height), 256, 0, st>>>(a, list, count);
        stage_end(ctx, 1);
        ARC_TRY_CUDA(cudaGetLastError());
        a.pixel_list = list;
        a.pixel_count = count;
    }
    stage_begin(ctx, "bf_gather");
    const arc_status s = launch_fast_path(a, p, ts.px, st);
    stage_end(ctx, 1);
    return s;
}

arc_status launch_pack_records(arc_context* ctx, const ArcAvplsGpuParam* avpls, const float4** records) {
    const int n = avpls->numAvpls;
    float4* rec = nullptr;
    ARC_TRY(ctx->arena.get("bf_records", (size_t)(n + 1) * 64, reinterpret_cast<void**>(&rec)));
    if (n > 0) {
        stage_begin(ctx, "bf_pack");
        pack_bf_records<<<(n + 255) / 256, 256, 0, ctx->stream>>>(*avpls, ctx->d_materials, ctx->num_materials, rec,
                                                                   ctx->d_error);
        stage_end(ctx, 1);
        ARC_TRY_CUDA(cudaGetLastError());
    }
    *records = rec;
    return ARC_OK;
}

arc_status launch_antiradiance_only(arc_context* ctx, const GatherLaunch& g, double* ar64) {
    const ArcGatherParams& p = *g.params;
    BfArgs a = make_args(ctx, g);
    a.out_res = nullptr;
    a.out_rad = nullptr;
    a.out_res64 = nullptr;
    a.out_ar64 = ar64;
    cudaStream_t st = ctx->stream;
    ARC_TRY(pack_records(ctx, g, a, false));
    a.chunk = kTileShapes[kDefaultTileShape].chunk;
    stage_begin(ctx, "bf_antiradiance");
    const arc_status s = p.ar_kind == ARC_AR_DISK ? launch_fast<ARC_AR_DISK, 0, 2, false>(a, st)
                                                  : launch_fast<ARC_AR_CONE, 0, 2, false>(a, st);
    stage_end(ctx, 1);
    return s;
}

}  // namespace arc

namespace arc {
namespace {

BfArgs make_args(arc_context* ctx, const GatherLaunch& g) {
    const ArcGatherParams& p = *g.params;
    const ArcGBufferView& gb = *g.gbuffer;
    const ArcOutputView& out = *g.out;
    BfArgs a{};
    a.n = g.avpls->numAvpls;
    a.gpos = reinterpret_cast<const float4*>(gb.position);
    a.gnrm = reinterpret_cast<const float4*>(gb.normal);
    a.gpitch = gb.pitch;
    a.width = gb.width;
    a.height = gb.height;
    a.mats = ctx->d_materials;
    a.num_mats = ctx->num_materials;
    a.cam = g.cam;
    a.eps = 0.001f;
    a.cos_thr = fmaxf(cosf(p.cone_half_angle), a.eps);
    a.clamp2 = p.dist_clamp > 0.0f ? p.dist_clamp * p.dist_clamp : 0.0f;
    a.disk_r2 = p.disk_radius * p.disk_radius;
    a.pc.cos_thr = a.cos_thr;
    a.pc.eps = a.eps;
    a.pc.inv_clamp2 = p.dist_clamp > 0.0f ? 1.0f / a.clamp2 : INFINITY;
    a.pc.disk_r2 = a.disk_r2;
    a.disk_scale = p.disk_radius > 0.0f ? 1.0f / (kPi * p.disk_radius * p.disk_radius) : 0.0f;
    a.lim_rad = p.geo_limit_radiance > 0.0f ? p.geo_limit_radiance : INFINITY;
    a.lim_ar = p.geo_limit_antiradiance > 0.0f ? p.geo_limit_antiradiance : INFINITY;
    a.out_res = reinterpret_cast<float4*>(out.result);
    a.out_rad = reinterpret_cast<float4*>(out.radiance);
    a.out_ar = reinterpret_cast<float4*>(out.antiradiance);
    a.out_res64 = out.result_fp64;
    a.opitch = out.pitch;
    a.err = ctx->d_error;
    a.soa = *g.avpls;
    return a;
}

// Pack the AVPL records into the context arena.
arc_status pack_records(arc_context* ctx, const GatherLaunch& g, BfArgs& a, bool pairs) {
    float4* rec = nullptr;
    ARC_TRY(ctx->arena.get("bf_records", (size_t)(a.n + 1) * 64, reinterpret_cast<void**>(&rec)));
    if (a.n > 0) {
        stage_begin(ctx, "bf_pack");
        if (pairs)
            pack_bf_pairs<<<(a.n + 1 + 255) / 256, 256, 0, ctx->stream>>>(
                *g.avpls, ctx->d_materials, ctx->num_materials, reinterpret_cast<float*>(rec), ctx->d_error);
        else
            pack_bf_records<<<(a.n + 255) / 256, 256, 0, ctx->stream>>>(*g.avpls, ctx->d_materials,
                                                                         ctx->num_materials, rec, ctx->d_error);
        stage_end(ctx, 1);
        ARC_TRY_CUDA(cudaGetLastError());
    }
    a.records = rec;
    return ARC_OK;
}

}  // namespace
}  // namespace arc

// ---------------------------------------------------------------------------------------
// Allocation-free brute-force gather (arc_gather_bruteforce_noalloc).
//
// For hosts that own every byte of device memory themselves and forbid the library from
// allocating: renderer plugins whose host pre-allocates a fixed device budget at start-up, and
// real-time frame loops that must not call cudaMalloc/cudaFree mid-frame (both can synchronise
// the device and stall the frame).  Such a caller cannot create an arc_context (which
// allocates), so this entry point takes a stream instead and keeps its only scratch -- the
// packed AVPL records, the material table and the device error word -- in one file-scope
// __device__ array of fixed size, which every GPU that loads libarc holds until the process
// exits.
// ---------------------------------------------------------------------------------------
#include <mutex>

static constexpr int kNoAllocMaxAvpls = 65536;  // AVPL records the static scratch holds
static constexpr size_t kNoAllocRecordBytes = (size_t)kNoAllocMaxAvpls * 64;
static constexpr size_t kNoAllocMaterialBytes = ARC_MAX_MATERIALS * sizeof(arc::MaterialRecord);
// [records: 64 B x kNoAllocMaxAvpls][materials: 32 B x 64][error word: 256 B]  (4.2 MB)
static constexpr size_t kNoAllocBytes = kNoAllocRecordBytes + kNoAllocMaterialBytes + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace arc {
namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
// per device: the context the address was looked up in, and the address
void* g_noalloc_ctx[kNoAllocMaxDevices] = {};
unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {};

using CtxGetCurrentFn = int (*)(void**);  // cuCtxGetCurrent(CUcontext*) -> CUresult

// The driver context current on this thread (NULL if the driver entry point is unavailable).
void* current_driver_context() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    void* c = nullptr;
    if (fn && fn(&c) != 0) c = nullptr;
    return c;
}

// Device address of g_noalloc_scratch in the current device's context, looked up with that
// device current the first time a call runs in that context (again after a device reset or in
// another driver context, where the module is loaded anew at another address).  The host-side
// name g_noalloc_scratch is only a stand-in for the symbol and must never be handed to a kernel.
arc_status noalloc_scratch(unsigned char** out) {
    int dev = 0;
    ARC_TRY_CUDA(cudaGetDevice(&dev));
    ARC_CHECK_ARG(dev >= 0 && dev < kNoAllocMaxDevices, "device index beyond the allocation-free path's table");
    // (NULL before the runtime has made the device's primary context current: looked up then)
    const void* c = current_driver_context();
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev] || !c || c != g_noalloc_ctx[dev]) {
        void* p = nullptr;
        ARC_TRY_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
        g_noalloc_ctx[dev] = current_driver_context();  // current now, after the lookup
    }
    *out = g_noalloc_addr[dev];
    return ARC_OK;
}

// The material table travels as a kernel argument (no host buffer is read after the call
// returns); the same launch clears the call's error word.
struct NoAllocMaterials {
    MaterialRecord rec[ARC_MAX_MATERIALS];
    int count;
};

__global__ void noalloc_write_materials(NoAllocMaterials t, MaterialRecord* mats, uint32_t* err) {
    const int i = threadIdx.x;
    if (i < t.count) mats[i] = t.rec[i];
    if (i == 0) *err = 0u;
}

}  // namespace
}  // namespace arc

extern "C" arc_status arc_gather_bruteforce_noalloc(void* cuda_stream, const ArcMaterial* materials,
                                                    int32_t num_materials, const ArcAvplsGpuParam* avpls,
                                                    const ArcGBufferView* gbuffer, ArcFloat3 camera_position,
                                                    const ArcGatherParams* params, const ArcOutputView* out,
                                                    uint32_t* device_error_word) {
    using namespace arc;
    ARC_CHECK_ARG(materials && avpls && gbuffer && params && out, "NULL argument");
    const ArcGatherParams& p = *params;
    const ArcGBufferView& gb = *gbuffer;
    ARC_CHECK_ARG(num_materials > 0 && num_materials <= ARC_MAX_MATERIALS,
                  "material count must be in [1, ARC_MAX_MATERIALS]");
    ARC_CHECK_ARG(avpls->numAvpls >= 0, "negative AVPL count");
    if (avpls->numAvpls > kNoAllocMaxAvpls) {
        set_last_error("arc_gather_bruteforce_noalloc: " + std::to_string(avpls->numAvpls) +
                       " AVPLs exceed the allocation-free path's maximum of " + std::to_string(kNoAllocMaxAvpls) +
                       " (use arc_gather_bruteforce)");
        return ARC_ERR_INVALID_ARG;
    }
    ARC_CHECK_ARG(p.ar_kind >= 0 && p.ar_kind <= 2, "ar_kind out of range");
    ARC_CHECK_ARG(p.precision >= 0 && p.precision <= 3, "precision out of range");
    ARC_CHECK_ARG(p.tile_config >= -1 && p.tile_config < kNumTileShapes, "tile_config out of range");
    ARC_CHECK_ARG(gb.width > 0 && gb.height > 0 && gb.pitch >= gb.width && gb.position && gb.normal,
                  "bad G-buffer view");
    ARC_CHECK_ARG(reinterpret_cast<uintptr_t>(gb.position) % 16 == 0 && reinterpret_cast<uintptr_t>(gb.normal) % 16 == 0,
                  "G-buffer planes must be 16-byte aligned");
    ARC_CHECK_ARG(out->pitch >= gb.width && (out->result || out->radiance || out->antiradiance || out->result_fp64),
                  "bad output view");
    ARC_CHECK_ARG(p.ar_kind != ARC_AR_DISK || p.disk_radius > 0.0f, "disk radius must be > 0");

    unsigned char* scratch = nullptr;
    ARC_TRY(noalloc_scratch(&scratch));
    float4* records = reinterpret_cast<float4*>(scratch);
    MaterialRecord* mats = reinterpret_cast<MaterialRecord*>(scratch + kNoAllocRecordBytes);
    uint32_t* err = reinterpret_cast<uint32_t*>(scratch + kNoAllocRecordBytes + kNoAllocMaterialBytes);
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);

    // material table and error word: the scratch keeps the previous call's contents, so both are
    // rewritten here (the records are rewritten by the pack kernel for every AVPL used)
    NoAllocMaterials tab;
    tab.count = num_materials;
    bool spec = false;
    for (int i = 0; i < num_materials; ++i) {
        const ArcMaterial& m = materials[i];
        const float sl = sqrtf(m.specular.x * m.specular.x + m.specular.y * m.specular.y + m.specular.z * m.specular.z);
        tab.rec[i].diffuse_exp = make_float4(m.diffuse.x, m.diffuse.y, m.diffuse.z, m.exponent);
        tab.rec[i].specular_flag = make_float4(m.specular.x, m.specular.y, m.specular.z, sl > 0.0f ? 1.0f : 0.0f);
        spec = spec || sl > 0.0f;
    }
    for (int i = num_materials; i < ARC_MAX_MATERIALS; ++i) {
        tab.rec[i].diffuse_exp = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        tab.rec[i].specular_flag = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    noalloc_write_materials<<<1, ARC_MAX_MATERIALS, 0, st>>>(tab, mats, err);
    ARC_TRY_CUDA(cudaGetLastError());

    BfArgs a{};
    a.n = avpls->numAvpls;
    a.gpos = reinterpret_cast<const float4*>(gb.position);
    a.gnrm = reinterpret_cast<const float4*>(gb.normal);
    a.gpitch = gb.pitch;
    a.width = gb.width;
    a.height = gb.height;
    a.mats = mats;
    a.num_mats = num_materials;
    a.cam = make_float3(camera_position.x, camera_position.y, camera_position.z);
    a.eps = 0.001f;
    a.cos_thr = fmaxf(cosf(p.cone_half_angle), a.eps);
    a.clamp2 = p.dist_clamp > 0.0f ? p.dist_clamp * p.dist_clamp : 0.0f;
    a.disk_r2 = p.disk_radius * p.disk_radius;
    a.pc.cos_thr = a.cos_thr;
    a.pc.eps = a.eps;
    a.pc.inv_clamp2 = p.dist_clamp > 0.0f ? 1.0f / a.clamp2 : INFINITY;
    a.pc.disk_r2 = a.disk_r2;
    a.disk_scale = p.disk_radius > 0.0f ? 1.0f / (kPi * p.disk_radius * p.disk_radius) : 0.0f;
    a.lim_rad = p.geo_limit_radiance > 0.0f ? p.geo_limit_radiance : INFINITY;
    a.lim_ar = p.geo_limit_antiradiance > 0.0f ? p.geo_limit_antiradiance : INFINITY;
    a.out_res = reinterpret_cast<float4*>(out->result);
    a.out_rad = reinterpret_cast<float4*>(out->radiance);
    a.out_ar = reinterpret_cast<float4*>(out->antiradiance);
    a.out_res64 = out->result_fp64;
    a.out_ar64 = nullptr;
    a.opitch = out->pitch;
    a.err = err;
    a.soa = *avpls;
    a.records = records;

    if (spec || p.geo_limit_radiance > 0.0f || p.geo_limit_antiradiance > 0.0f) {
        dim3 grid((gb.width + kTileW - 1) / kTileW, (gb.height + 15) / 16);
        if (p.precision == ARC_PREC_FP64) {
            if (p.ar_kind == 0) gather_general_kernel<0, double><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 1) gather_general_kernel<1, double><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 2) gather_general_kernel<2, double><<<grid, kThreads, 0, st>>>(a);
        } else {
            if (p.ar_kind == 0) gather_general_kernel<0, float><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 1) gather_general_kernel<1, float><<<grid, kThreads, 0, st>>>(a);
            if (p.ar_kind == 2) gather_general_kernel<2, float><<<grid, kThreads, 0, st>>>(a);
        }
        ARC_TRY_CUDA(cudaGetLastError());
    } else {
        if (a.n > 0) {
            // an odd count's zero pad record still fits: the scratch holds kNoAllocMaxAvpls (even)
            if (use_packed(p))
                pack_bf_pairs<<<(a.n + 1 + 255) / 256, 256, 0, st>>>(*avpls, mats, num_materials,
                                                                    reinterpret_cast<float*>(records), err);
            else
                pack_bf_records<<<(a.n + 255) / 256, 256, 0, st>>>(*avpls, mats, num_materials, records, err);
            ARC_TRY_CUDA(cudaGetLastError());
        }
        const TileShape ts = kTileShapes[p.tile_config < 0 ? kDefaultTileShape : p.tile_config];
        a.chunk = ts.chunk;
        ARC_TRY(launch_fast_path(a, p, ts.px, st));
    }
    if (device_error_word) {
        uint32_t w = 0;
        ARC_TRY_CUDA(cudaMemcpyAsync(&w, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        ARC_TRY_CUDA(cudaStreamSynchronize(st));
        *device_error_word = w;
    }
    return ARC_OK;
}

// Brute-force launch-shape autotuner (no counterpart in the reference): times every shape of
// kTileShapes on the caller's workload (one warm-up and one timed run each, CUDA events on the
// context's stream) and makes the fastest the context's default for tile_config = -1.
extern "C" int32_t arc_bruteforce_num_tile_shapes(void) { return arc::kNumTileShapes; }

extern "C" arc_status arc_context_set_tile_config(arc_context* ctx, int32_t tile_config) {
    ARC_CHECK_ARG(ctx, "NULL context");
    ARC_CHECK_ARG(tile_config >= -1 && tile_config < arc::kNumTileShapes, "tile_config out of range");
    ctx->bf_tile_config = tile_config;
    return ARC_OK;
}

extern "C" arc_status arc_autotune_bruteforce(arc_context* ctx, const ArcAvplsGpuParam* avpls,
                                              const ArcGBufferView* gbuffer, ArcFloat3 camera_position,
                                              const ArcGatherParams* params, const ArcOutputView* out, int32_t* best,
                                              float* times_ms, int32_t num_shapes) {
    using namespace arc;
    ARC_CHECK_ARG(ctx && avpls && gbuffer && params && out && best, "NULL argument");
    ARC_CHECK_ARG(!times_ms || num_shapes >= kNumTileShapes, "times_ms holds fewer entries than there are shapes");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    ScopedEvents<2> ev;
    ARC_TRY_CUDA(ev.create());
    const cudaEvent_t e0 = ev[0], e1 = ev[1];
    cudaError_t ce = cudaSuccess;
    arc_status s = ARC_OK;
    float best_ms = 0.0f;
    int best_i = -1;
    for (int i = 0; i < kNumTileShapes && s == ARC_OK; ++i) {
        ArcGatherParams p = *params;
        p.tile_config = i;
        s = arc_gather_bruteforce(ctx, avpls, gbuffer, camera_position, &p, out);  // warm-up
        if (s == ARC_OK) ce = cudaEventRecord(e0, ctx->stream);
        if (s == ARC_OK && ce == cudaSuccess) s = arc_gather_bruteforce(ctx, avpls, gbuffer, camera_position, &p, out);
        if (s == ARC_OK && ce == cudaSuccess) ce = cudaEventRecord(e1, ctx->stream);
        if (s == ARC_OK && ce == cudaSuccess) ce = cudaEventSynchronize(e1);
        float ms = -1.0f;
        if (s == ARC_OK && ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
        if (ce != cudaSuccess && s == ARC_OK) {
            set_last_error(std::string("arc_autotune_bruteforce: ") + cudaGetErrorString(ce));
            s = ARC_ERR_CUDA;
        }
        if (times_ms) times_ms[i] = ms;
        if (s == ARC_OK && (best_i < 0 || ms < best_ms)) {
            best_ms = ms;
            best_i = i;
        }
    }
    ARC_TRY(s);
    ctx->bf_tile_config = best_i;
    *best = best_i;
    return ARC_OK;
}

