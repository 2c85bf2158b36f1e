// Per-(pixel, AVPL record) arithmetic of the fast gather, shared by the brute-force kernel and the
// cut evaluation.  A record is 4 float4: {p.xyz, n.x}, {n.y, n.z, w.x, w.y}, {w.z, L'.rgb},
// {A.rgb, aux}; L' already carries the AVPL-side Lambertian BRDF and the receiver's diffuse/pi is
// applied by the caller once per pixel.
//
// Radiance geometry term (G of cudaGather.cu:45-57 with the distance clamp):
//     g = max(n.d^, 0) max(-n_a.d^, 0) / max(|d|^2, clamp^2),   d = p_a - p, d^ = d / |d|
// Cone antiradiance (Gather.frag:149-188): accepted when (-d^).w_a > max(cos h, 0.001) [<=> theta < h]
// and n.d^ > 0.001, with G_A = n.d^ / max(|d|^2, clamp^2).
// Disk antiradiance (cudaGather.cu:97-144): the ray p_a + t w^ hits the receiver plane at t > 0
// within radius r, w_a.n < 0 and n_a.(p - p_a) < 0.
#ifndef ARC_PAIR_MATH_CUH_
#define ARC_PAIR_MATH_CUH_

#include <type_traits>

#include "device_common.cuh"

namespace arc {

template <typename T>
__device__ __forceinline__ T rsqrt_t(T x);
template <>
__device__ __forceinline__ float rsqrt_t<float>(float x) {
    return rsqrtf(x);
}
template <>
__device__ __forceinline__ double rsqrt_t<double>(double x) {
    return 1.0 / sqrt(x);
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

template <typename T>
struct Pixel {
    T px, py, pz, nx, ny, nz;
    T r0, r1, r2, a0, a1, a2;  // running (or per-chunk partial) sums
};

struct PairConsts {
    float cos_thr;     // cone: max(cos(half angle), 0.001)
    float eps;         // cone: 0.001
    float inv_clamp2;  // 1 / clamp^2 or +inf
    float disk_r2;     // disk radius^2
};

template <int AR, typename T>
__device__ __forceinline__ void pair_terms(const float4& q0, const float4& q1, const float4& q2, const float4& q3,
                                           const Pixel<T>& s, const PairConsts& k, T& g, T& ga) {
    const T dx = (T)q0.x - s.px, dy = (T)q0.y - s.py, dz = (T)q0.z - s.pz;
    T l2 = dx * dx + dy * dy + dz * dz;
    l2 = l2 > (T)1e-30 ? l2 : (T)1e-30;
    const T r = rsqrt_t<T>(l2);
    const T nd = s.nx * dx + s.ny * dy + s.nz * dz;
    const T nad = (T)q0.w * dx + (T)q1.x * dy + (T)q1.y * dz;
    const T c1 = nd * r;
    const T c2 = -nad * r;
    const T rr = r * r;
    const T inv = rr < (T)k.inv_clamp2 ? rr : (T)k.inv_clamp2;
    g = (c1 > (T)0 ? c1 : (T)0) * (c2 > (T)0 ? c2 : (T)0) * inv;
    ga = (T)0;
    if (AR == ARC_AR_CONE) {
        const T wd = (T)q1.z * dx + (T)q1.w * dy + (T)q2.x * dz;
        const T cw = -wd * r;
        const bool acc = (cw > (T)k.cos_thr) && (c1 > (T)k.eps);
        ga = acc ? c1 * inv : (T)0;
    } else if (AR == ARC_AR_DISK) {
        const T wn = (T)q1.z * s.nx + (T)q1.w * s.ny + (T)q2.x * s.nz;
        const T t = -nd / wn;
        const T ts = t * (T)q3.w;
        const T hx = dx + ts * (T)q1.z, hy = dy + ts * (T)q1.w, hz = dz + ts * (T)q2.x;
        const T h2 = hx * hx + hy * hy + hz * hz;
        const bool acc = (wn < (T)0) && (t > (T)0) && (h2 < (T)k.disk_r2) && (nad > (T)0);
        ga = acc ? (T)1 : (T)0;
    }
}

}  // namespace arc

#endif  // ARC_PAIR_MATH_CUH_
