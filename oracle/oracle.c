/*
 * oracle.c - CPU restatement of the AntiradianceCuts gather and LBVH build.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the GPU library: only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it.  The product never calls
 * it, and nothing here is a fallback for the GPU path.
 *
 * Parity pinning:
 *   - Morton codes: pinned against the reference's own morton.h, compiled into
 *     oracle/_ref/libref_morton.so by oracle/Makefile and frozen into tests/golden/.
 *   - Radix tree: pinned against an independent top-down construction (the definition of a
 *     binary radix tree) and the reference's integrity invariants (bvh.cu:568-639).
 *   - Gather formulas: the reference's gather (cudaGather.cu) cannot be compiled here (it needs
 *     glm, GL interop headers and MSVC intrinsics), so they are pinned by closed-form
 *     known-answer cases in tests/golden/ instead of a reference run.
 *
 * Compiled with -ffp-contract=off so that float expressions round exactly as written: the
 * LBVH's integer outputs and the FP32 tree data are compared bit for bit.
 *
 * Reference paths are inside the reference's Framework/ tree.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------------------------------- */
/* Gather (cudaGather.cu:45-154, Shaders/Gather.frag:149-208)                               */
/* ---------------------------------------------------------------------------------------- */

typedef struct {
    double x, y, z;
} d3;

static d3 d3m(double x, double y, double z) {
    d3 r = {x, y, z};
    return r;
}
static d3 d3sub(d3 a, d3 b) { return d3m(a.x - b.x, a.y - b.y, a.z - b.z); }
static d3 d3add(d3 a, d3 b) { return d3m(a.x + b.x, a.y + b.y, a.z + b.z); }
static d3 d3s(double s, d3 a) { return d3m(s * a.x, s * a.y, s * a.z); }
static d3 d3mul(d3 a, d3 b) { return d3m(a.x * b.x, a.y * b.y, a.z * b.z); }
static double d3dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double d3len(d3 a) { return sqrt(d3dot(a, a)); }
static d3 d3norm(d3 a) { return d3s(1.0 / d3len(a), a); }
static d3 d3load(const float* p) { return d3m(p[0], p[1], p[2]); }
static double clampd(double v, double a, double b) { return v < a ? a : (v > b ? b : v); }

#define OR_PI 3.14159265358979323846

typedef struct {
    int32_t ar_kind; /* 0 none, 1 disk, 2 cone */
    float disk_radius;
    float cone_half_angle;
    float dist_clamp;
    float geo_limit_radiance;
    float geo_limit_antiradiance;
} oracle_params;

typedef struct {
    const float* diffuse;  /* [m][3] */
    const float* specular; /* [m][3] */
    const float* exponent; /* [m] */
    int32_t num;
} oracle_materials;

/* f_r(w_i, w_o, n, mat) (cudaGather.cu:59-68); reflect(I, N) = I - 2 (N.I) N. */
static d3 f_r(d3 w_i, d3 w_o, d3 n, const oracle_materials* m, int mat) {
    d3 dif = d3load(m->diffuse + 3 * mat), spe = d3load(m->specular + 3 * mat);
    d3 d = d3s(1.0 / OR_PI, dif);
    if (d3len(spe) > 0.0) {
        d3 I = d3s(-1.0, w_i);
        d3 r = d3sub(I, d3s(2.0 * d3dot(n, I), n));
        double c = fmax(0.0, d3dot(r, w_o));
        double e = m->exponent[mat];
        d = d3add(d, d3s(0.5 / OR_PI * (e + 2.0) * pow(c, e), spe));
    }
    return d;
}

/* G with the optional distance clamp and GeoTermLimitRadiance (cudaGather.cu:45-57,
 * Gather.frag:190-207). */
static double G(d3 p1, d3 n1, d3 p2, d3 n2, const oracle_params* P) {
    d3 n_1 = d3norm(n1), n_2 = d3norm(n2);
    d3 v = d3sub(p2, p1);
    double l2 = d3dot(v, v);
    if (l2 == 0.0) return 0.0;
    d3 w = d3s(1.0 / sqrt(l2), v);
    double c1 = clampd(d3dot(n_1, w), 0.0, 1.0);
    double c2 = clampd(-d3dot(n_2, w), 0.0, 1.0);
    double c = P->dist_clamp;
    if (c > 0.0 && l2 < c * c) l2 = c * c;
    double g = c1 * c2 / l2;
    if (P->geo_limit_radiance > 0.0f) g = clampd(g, 0.0, P->geo_limit_radiance);
    return g;
}

/* One AVPL's radiance at a pixel (getRadiance, cudaGather.cu:78-95). */
static d3 radiance_term(d3 pos, d3 n, int mat, d3 pa, d3 na, d3 wa, d3 La, int mat_a, d3 cam,
                        const oracle_materials* M, const oracle_params* P) {
    d3 diff = d3sub(pos, pa);
    if (d3dot(diff, diff) == 0.0) return d3m(0, 0, 0);
    d3 direction = d3norm(diff);
    d3 brdf_light = f_r(d3s(-1.0, wa), direction, na, M, mat_a);
    if (d3len(wa) == 0.0) brdf_light = d3m(1, 1, 1);
    d3 brdf = f_r(d3norm(d3sub(pa, pos)), d3norm(d3sub(cam, pos)), n, M, mat);
    double g = G(pos, n, pa, na, P);
    return d3s(g, d3mul(d3mul(La, brdf_light), brdf));
}

/* Disk antiradiance (getAntiradiance + intersectLinePlane, cudaGather.cu:97-144). */
static d3 antiradiance_disk(d3 pos, d3 n, int mat, d3 pa, d3 na, d3 wa, d3 Aa, d3 cam,
                            const oracle_materials* M, const oracle_params* P) {
    d3 zero = d3m(0, 0, 0);
    double denom = d3dot(wa, n);
    if (denom == 0.0) return zero;
    double t = d3dot(d3sub(pos, pa), n) / denom;
    if (t <= 0.0) return zero;
    d3 hit = d3add(pa, d3s(t, d3norm(wa)));
    double r = P->disk_radius;
    if (d3len(d3sub(hit, pos)) >= r) return zero;
    if (d3dot(d3norm(d3sub(hit, pa)), wa) <= 0.0) return zero;
    if (d3dot(n, wa) >= 0.0) return zero;
    d3 direction = d3norm(d3sub(pos, pa));
    if (d3dot(direction, na) >= 0.0) return zero;
    d3 brdf = f_r(d3norm(d3sub(pa, pos)), d3norm(d3sub(cam, pos)), n, M, mat);
    return d3s(1.0 / (OR_PI * r * r), d3mul(Aa, brdf));
}

/* Cone antiradiance (GetAntiradiance, Gather.frag:149-188) times the receiver BRDF (the
 * call site Gather.frag:134), with the distance clamp and GeoTermLimitAntiradiance.
 * theta < halfAngle is evaluated with acos as the shader does. */
static d3 antiradiance_cone(d3 pos, d3 n, int mat, d3 pa, d3 wa, d3 Aa, d3 cam, const oracle_materials* M,
                            const oracle_params* P) {
    const double eps = 0.001;
    d3 zero = d3m(0, 0, 0);
    d3 v = d3sub(pos, pa);
    double l2 = d3dot(v, v);
    if (l2 == 0.0) return zero;
    d3 avpl_to_pos = d3s(1.0 / sqrt(l2), v);
    d3 nn = d3norm(n);
    double cw = d3dot(avpl_to_pos, wa);
    if (cw <= eps) return zero;
    double cn = -d3dot(nn, avpl_to_pos);
    if (cn <= eps) return zero;
    double theta = acos(clampd(cw, -1.0, 1.0));
    if (!(theta < (double)P->cone_half_angle)) return zero;
    double c = P->dist_clamp;
    if (c > 0.0 && l2 < c * c) l2 = c * c;
    double ga = cn / l2;
    if (P->geo_limit_antiradiance > 0.0f) ga = clampd(ga, 0.0, P->geo_limit_antiradiance);
    d3 brdf = f_r(d3norm(d3sub(pa, pos)), d3norm(d3sub(cam, pos)), n, M, mat);
    return d3s(ga, d3mul(Aa, brdf));
}

/*
 * FP64 exact gather for a list of pixels: for each listed pixel, the radiance sum, the
 * antiradiance sum and result = radiance - antiradiance (kernel_radiance_simple,
 * kernel_antiradiance / cone variant, kernel_combine).  Pixels whose material index is 0
 * have no surface and give 0.  AVPL arrays are [n][3] floats.
 */
OR_EXPORT void oracle_gather_fp64(const float* gb_pos, const float* gb_nrm, int32_t width, const int32_t* pixels,
                                  int32_t num_pixels, const float* a_pos, const float* a_nrm, const float* a_w,
                                  const float* a_L, const float* a_A, const int32_t* a_mat, int32_t num_avpls,
                                  const float* diffuse, const float* specular, const float* exponent,
                                  int32_t num_materials, const float* cam, const oracle_params* P, double* out_rad,
                                  double* out_ar, double* out_res, int32_t num_threads) {
    (void)width;
    /* thread-private copies of the call's constants, as in oracle_gather_fp32 */
#pragma omp parallel num_threads(num_threads > 0 ? num_threads : 1)
    {
    const oracle_params Pl = *P;
    const oracle_materials M = {diffuse, specular, exponent, num_materials};
    const d3 c = d3load(cam);
#pragma omp for schedule(dynamic, 1)
    for (int32_t k = 0; k < num_pixels; ++k) {
        const int64_t px = pixels[k];
        const float* gp = gb_pos + 4 * px;
        const float* gn = gb_nrm + 4 * px;
        const int mat = (int)gn[3];
        d3 rad = d3m(0, 0, 0), ar = d3m(0, 0, 0);
        if (mat > 0 && mat < num_materials) {
            d3 pos = d3load(gp), n = d3load(gn);
            for (int32_t i = 0; i < num_avpls; ++i) {
                d3 pa = d3load(a_pos + 3 * i), na = d3load(a_nrm + 3 * i), wa = d3load(a_w + 3 * i);
                rad = d3add(rad, radiance_term(pos, n, mat, pa, na, wa, d3load(a_L + 3 * i), a_mat[i], c, &M, &Pl));
                if (Pl.ar_kind == 1)
                    ar = d3add(ar, antiradiance_disk(pos, n, mat, pa, na, wa, d3load(a_A + 3 * i), c, &M, &Pl));
                else if (Pl.ar_kind == 2)
                    ar = d3add(ar, antiradiance_cone(pos, n, mat, pa, wa, d3load(a_A + 3 * i), c, &M, &Pl));
            }
        }
        out_rad[3 * k + 0] = rad.x; out_rad[3 * k + 1] = rad.y; out_rad[3 * k + 2] = rad.z;
        out_ar[3 * k + 0] = ar.x; out_ar[3 * k + 1] = ar.y; out_ar[3 * k + 2] = ar.z;
        out_res[3 * k + 0] = rad.x - ar.x; out_res[3 * k + 1] = rad.y - ar.y; out_res[3 * k + 2] = rad.z - ar.z;
    }
    }
}

/*
 * Clustered deferred disk antiradiance, restated from the reference (VisiblePointsBvh,
 * bvh.cu:986-1179; kernel_gather_cluster_lights + intersectBB, cudaGather.cu:663-748;
 * kernel_antiradiance_clusterred, cudaGather.cu:605-659) with the build's two decisions: a cluster
 * is a (16 x 16 tile, depth slice k) of surface pixels, k = floor(log(d / z_near) /
 * log(1 + 2 tan(theta) / 16)), and its list holds the AVPLs whose ray (position, incDirection) meets
 * its box grown by twice the disk radius, in AVPL order.  Every surface pixel's antiradiance is the
 * FP64 disk term summed over its cluster's list.  out_ar: [W * H][3]; returns the number of list
 * entries over all clusters (*out_clusters: the number of clusters).
 */
static int ray_box_f(const float lo[3], const float hi[3], const float* o, const float* d) {
    float t1[3], t2[3];
    for (int k = 0; k < 3; ++k) {
        const float f = 1.0f / d[k];
        t1[k] = (lo[k] - o[k]) * f;
        t2[k] = (hi[k] - o[k]) * f;
    }
    const float tmin = fmaxf(fmaxf(fminf(t1[0], t2[0]), fminf(t1[1], t2[1])), fminf(t1[2], t2[2]));
    const float tmax = fminf(fminf(fmaxf(t1[0], t2[0]), fmaxf(t1[1], t2[1])), fmaxf(t1[2], t2[2]));
    return !(tmax < 0.0f || tmin > tmax);
}

OR_EXPORT int64_t oracle_clustered_disk_ar(const float* gb_pos, const float* gb_nrm, int32_t W, int32_t H,
                                           const float* a_pos, const float* a_nrm, const float* a_w, const float* a_A,
                                           int32_t num_avpls, const float* diffuse, const float* specular,
                                           const float* exponent, int32_t num_materials, const float* cam, float z_near,
                                           float theta, const oracle_params* P, double* out_ar, int32_t* out_clusters) {
    oracle_materials M = {diffuse, specular, exponent, num_materials};
    const d3 c = d3load(cam);
    const double step = log(1.0 + 2.0 * tan((double)theta) / 16.0);
    const int tiles_x = (W + 15) / 16, tiles_y = (H + 15) / 16;
    const float grow = 2.0f * P->disk_radius;
    int64_t entries = 0;
    int32_t clusters = 0;
    for (int64_t i = 0; i < (int64_t)W * H * 3; ++i) out_ar[i] = 0.0;
    int* list = (int*)malloc(sizeof(int) * (size_t)(num_avpls > 0 ? num_avpls : 1));
    for (int ty = 0; ty < tiles_y; ++ty)
        for (int tx = 0; tx < tiles_x; ++tx) {
            // depth slice of every surface pixel of the tile
            int kk[256], px[256], np = 0;
            for (int y = ty * 16; y < ty * 16 + 16 && y < H; ++y)
                for (int x = tx * 16; x < tx * 16 + 16 && x < W; ++x) {
                    const float* gn = gb_nrm + 4 * ((int64_t)y * W + x);
                    if (!(gn[3] > 0.0f)) continue;
                    const d3 p = d3load(gb_pos + 4 * ((int64_t)y * W + x));
                    const double d = d3len(d3sub(c, p));
                    kk[np] = (int)floor(log(d / (double)z_near) / step);
                    px[np++] = y * W + x;
                }
            // one cluster per distinct slice
            for (int a = 0; a < np; ++a) {
                int seen = 0;
                for (int b = 0; b < a; ++b) seen |= kk[b] == kk[a];
                if (seen) continue;
                ++clusters;
                float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
                for (int b = a; b < np; ++b) {
                    if (kk[b] != kk[a]) continue;
                    const float* p = gb_pos + 4 * (int64_t)px[b];
                    for (int k = 0; k < 3; ++k) {
                        lo[k] = fminf(lo[k], p[k]);
                        hi[k] = fmaxf(hi[k], p[k]);
                    }
                }
                for (int k = 0; k < 3; ++k) {
                    lo[k] = lo[k] - grow;
                    hi[k] = hi[k] + grow;
                }
                int nl = 0;
                for (int32_t i = 0; i < num_avpls; ++i)
                    if (ray_box_f(lo, hi, a_pos + 3 * i, a_w + 3 * i)) list[nl++] = i;
                entries += nl;
                for (int b = a; b < np; ++b) {
                    if (kk[b] != kk[a]) continue;
                    const float* gp = gb_pos + 4 * (int64_t)px[b];
                    const float* gn = gb_nrm + 4 * (int64_t)px[b];
                    const int mat = (int)gn[3];
                    if (mat <= 0 || mat >= num_materials) continue;
                    d3 ar = d3m(0, 0, 0);
                    for (int q = 0; q < nl; ++q) {
                        const int i = list[q];
                        ar = d3add(ar, antiradiance_disk(d3load(gp), d3load(gn), mat, d3load(a_pos + 3 * i),
                                                         d3load(a_nrm + 3 * i), d3load(a_w + 3 * i),
                                                         d3load(a_A + 3 * i), c, &M, P));
                    }
                    double* o = out_ar + 3 * (int64_t)px[b];
                    o[0] = ar.x;
                    o[1] = ar.y;
                    o[2] = ar.z;
                }
            }
        }
    free(list);
    if (out_clusters) *out_clusters = clusters;
    return entries;
}

/* ---------------------------------------------------------------------------------------- */
/* Scalar FP32 gather: the reference's arithmetic (plain float sums, float combine), used as */
/* the timed CPU baseline.  Lambertian fast form is not assumed: every term evaluates the     */
/* full f_r and G like kernel_radiance_simple / kernel_antiradiance.                          */
/* ---------------------------------------------------------------------------------------- */

typedef struct {
    float x, y, z;
} f3;
static inline f3 f3m(float x, float y, float z) {
    f3 r = {x, y, z};
    return r;
}
static inline f3 f3sub(f3 a, f3 b) { return f3m(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 f3add(f3 a, f3 b) { return f3m(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 f3s(float s, f3 a) { return f3m(s * a.x, s * a.y, s * a.z); }
static inline f3 f3mul(f3 a, f3 b) { return f3m(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float f3dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 f3load(const float* p) { return f3m(p[0], p[1], p[2]); }
static inline f3 f3norm(f3 a) { return f3s(1.0f / sqrtf(f3dot(a, a)), a); }
static inline float clampf(float v, float a, float b) { return v < a ? a : (v > b ? b : v); }

static inline f3 f_r32(f3 w_i, f3 w_o, f3 n, const oracle_materials* m, int mat) {
    f3 d = f3s(0.318309886f, f3load(m->diffuse + 3 * mat));
    f3 spe = f3load(m->specular + 3 * mat);
    if (sqrtf(f3dot(spe, spe)) > 0.0f) {
        f3 I = f3s(-1.0f, w_i);
        f3 r = f3sub(I, f3s(2.0f * f3dot(n, I), n));
        float c = fmaxf(0.0f, f3dot(r, w_o));
        float e = m->exponent[mat];
        d = f3add(d, f3s(0.5f * 0.318309886f * (e + 2.0f) * powf(c, e), spe));
    }
    return d;
}

OR_EXPORT void oracle_gather_fp32(const float* gb_pos, const float* gb_nrm, int32_t width, const int32_t* pixels,
                                  int32_t num_pixels, const float* a_pos, const float* a_nrm, const float* a_w,
                                  const float* a_L, const float* a_A, const int32_t* a_mat, int32_t num_avpls,
                                  const float* diffuse, const float* specular, const float* exponent,
                                  int32_t num_materials, const float* cam, const oracle_params* P, float* out_res,
                                  int32_t num_threads) {
    (void)width;
    /* Every thread keeps its own copy of the call's constants: read through the calling thread's
     * stack frame, they share cache lines with what that thread writes while it gathers, and the
     * team then runs little faster than one thread. */
#pragma omp parallel num_threads(num_threads > 0 ? num_threads : 1)
    {
    const oracle_params Pl = *P;
    const oracle_materials M = {diffuse, specular, exponent, num_materials};
    const f3 c = f3load(cam);
    const float eps = 0.001f;
    const float cos_half = cosf(Pl.cone_half_angle);
    const float clamp2 = Pl.dist_clamp * Pl.dist_clamp;
#pragma omp for schedule(dynamic, 1)
    for (int32_t k = 0; k < num_pixels; ++k) {
        const int64_t px = pixels[k];
        const int mat = (int)gb_nrm[4 * px + 3];
        f3 rad = f3m(0, 0, 0), ar = f3m(0, 0, 0);
        if (mat > 0 && mat < num_materials) {
            const f3 pos = f3load(gb_pos + 4 * px), n = f3norm(f3load(gb_nrm + 4 * px));
            const f3 w_o = f3norm(f3sub(c, pos));
            for (int32_t i = 0; i < num_avpls; ++i) {
                const f3 pa = f3load(a_pos + 3 * i), na = f3load(a_nrm + 3 * i), wa = f3load(a_w + 3 * i);
                const f3 v = f3sub(pa, pos);
                float l2 = f3dot(v, v);
                if (l2 == 0.0f) continue;
                const f3 w = f3s(1.0f / sqrtf(l2), v);
                const f3 brdf = f_r32(w, w_o, n, &M, mat);
                /* radiance */
                f3 brdf_light = f_r32(f3s(-1.0f, wa), f3s(-1.0f, w), na, &M, a_mat[i]);
                if (f3dot(wa, wa) == 0.0f) brdf_light = f3m(1, 1, 1);
                const float c1 = clampf(f3dot(n, w), 0.0f, 1.0f);
                const float c2 = clampf(-f3dot(na, w), 0.0f, 1.0f);
                const float l2c = (clamp2 > 0.0f && l2 < clamp2) ? clamp2 : l2;
                float g = c1 * c2 / l2c;
                if (Pl.geo_limit_radiance > 0.0f) g = clampf(g, 0.0f, Pl.geo_limit_radiance);
                rad = f3add(rad, f3s(g, f3mul(f3mul(f3load(a_L + 3 * i), brdf_light), brdf)));
                /* antiradiance */
                if (Pl.ar_kind == 2) {
                    const float cw = -f3dot(w, wa);
                    if (cw > eps && c1 > eps && cw > cos_half) {
                        float ga = f3dot(n, w) / l2c;
                        if (Pl.geo_limit_antiradiance > 0.0f) ga = clampf(ga, 0.0f, Pl.geo_limit_antiradiance);
                        ar = f3add(ar, f3s(ga, f3mul(f3load(a_A + 3 * i), brdf)));
                    }
                } else if (Pl.ar_kind == 1) {
                    const float denom = f3dot(wa, n);
                    if (denom != 0.0f) {
                        const float t = f3dot(f3s(-1.0f, v), n) / denom;
                        const f3 wn = f3norm(wa);
                        const f3 h = f3add(pa, f3s(t, wn));
                        const f3 hp = f3sub(h, pos);
                        const float r = Pl.disk_radius;
                        if (t > 0.0f && sqrtf(f3dot(hp, hp)) < r && f3dot(f3norm(f3sub(h, pa)), wa) > 0.0f &&
                            denom < 0.0f && -f3dot(w, na) < 0.0f)
                            ar = f3add(ar, f3s(1.0f / (3.14159265f * r * r), f3mul(f3load(a_A + 3 * i), brdf)));
                    }
                }
            }
        }
        out_res[3 * k + 0] = rad.x - ar.x;
        out_res[3 * k + 1] = rad.y - ar.y;
        out_res[3 * k + 2] = rad.z - ar.z;
    }
    }
}

/* ---------------------------------------------------------------------------------------- */
/* LBVH build (bvh.cu, morton.h)                                                              */
/* ---------------------------------------------------------------------------------------- */

/* expandBitsBy2 / interleave(x,y,z) (morton.h:34-42, 48-50): bit i of x, y, z goes to bit
 * 3i, 3i+1, 3i+2. */
static uint32_t spread3(uint32_t v) {
    uint32_t r = 0;
    for (int i = 0; i < 10; ++i) r |= ((v >> i) & 1u) << (3 * i);
    return r;
}

/* interleave of six 10-bit values into 64 bits (morton.h:67-79): bit i of the k-th value
 * goes to bit 6i + k; the build keeps the low 32 bits (MC_SIZE uint32_t, bvh.h:17). */
static uint64_t spread6(uint32_t v, int k) {
    uint64_t r = 0;
    for (int i = 0; i < 10; ++i) r |= (uint64_t)((v >> i) & 1u) << (6 * i + k);
    return r;
}

/* MortonCode3D quantisation (morton.h:82-92): clamp(v * 1024, 0, 1023) then truncate. */
static uint32_t quant10(float v) {
    float q = fminf(fmaxf(v * 1024.0f, 0.0f), 1023.0f);
    return (uint32_t)q;
}

static void bbox3(const float* p, int32_t n, int reference_mode, float mn[3], float mx[3]) {
    for (int k = 0; k < 3; ++k) {
        mn[k] = FLT_MAX;
        /* the reference seeds the max reduction with numeric_limits<float>::min() = FLT_MIN
         * (bvh.cu:349-350), so an all-negative axis keeps FLT_MIN */
        mx[k] = reference_mode ? FLT_MIN : -FLT_MAX;
    }
    for (int32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], p[3 * i + k]);
            mx[k] = fmaxf(mx[k], p[3 * i + k]);
        }
}

/*
 * Morton codes of n points (Bvh::create, bvh.cu:343-369): Normalize (v - min) / (max - min)
 * per axis with IEEE division (bvh.cu:73-81), then MortonCode3D, or MortonCode6D of the
 * normalised position and normal truncated to 32 bits.  bbox_mode 0 uses scene_min/max for
 * positions; 1 reduces the AVPL box as the reference does.  Normals are always normalised over
 * their own box (bvh.cu:354-361).
 */
OR_EXPORT void oracle_morton(const float* pos, const float* nrm, int32_t n, int32_t consider_normals,
                             int32_t bbox_mode, const float* scene_min, const float* scene_max, uint32_t* codes) {
    float mn[3], mx[3], nmn[3], nmx[3];
    if (bbox_mode == 1) {
        bbox3(pos, n, 1, mn, mx);
    } else {
        for (int k = 0; k < 3; ++k) {
            mn[k] = scene_min[k];
            mx[k] = scene_max[k];
        }
    }
    if (consider_normals) bbox3(nrm, n, 1, nmn, nmx);
    for (int32_t i = 0; i < n; ++i) {
        uint32_t q[3];
        for (int k = 0; k < 3; ++k) q[k] = quant10((pos[3 * i + k] - mn[k]) / (mx[k] - mn[k]));
        if (!consider_normals) {
            codes[i] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
        } else {
            uint32_t u[3];
            for (int k = 0; k < 3; ++k) u[k] = quant10((nrm[3 * i + k] - nmn[k]) / (nmx[k] - nmn[k]));
            uint64_t c = spread6(q[0], 0) | spread6(q[1], 1) | spread6(q[2], 2) | spread6(u[0], 3) |
                         spread6(u[1], 4) | spread6(u[2], 5);
            codes[i] = (uint32_t)c;
        }
    }
}

/* Stable sort of indices by key (thrust::sort_by_key, bvh.cu:793-808): bottom-up merge sort,
 * equal keys keep their input order. */
OR_EXPORT void oracle_stable_sort(const uint32_t* keys, int32_t n, int32_t* perm) {
    int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) perm[i] = i;
    for (int32_t w = 1; w < n; w *= 2) {
        for (int32_t lo = 0; lo < n; lo += 2 * w) {
            int32_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            int32_t a = lo, b = mid, o = lo;
            while (a < mid && b < hi) tmp[o++] = keys[perm[b]] < keys[perm[a]] ? perm[b++] : perm[a++];
            while (a < mid) tmp[o++] = perm[a++];
            while (b < hi) tmp[o++] = perm[b++];
        }
        memcpy(perm, tmp, sizeof(int32_t) * (size_t)n);
    }
    free(tmp);
}

static int clz32(uint32_t x) { return x == 0 ? 32 : __builtin_clz(x); }

/* delta(i, j) (cpu_delta, bvh.cu:151-162): -1 outside [0, numNodes]; common prefix length
 * of the codes, extended by the prefix of the indices when the codes are equal. */
static int delta(const uint32_t* m, int32_t num_nodes, int32_t i, int32_t j) {
    if (j < 0 || j > num_nodes) return -1;
    int d = clz32(m[i] ^ m[j]);
    if (d == 32) d += clz32((uint32_t)(i ^ j));
    return d;
}

/*
 * Karras radix tree (buildRadixTree, bvh.cu:189-266) over n sorted codes: left/right of the
 * n-1 inner nodes and parents[2n-1] (leaves, then inner nodes; the root's parent is -1).
 * The range search starts at 128 and grows x4 as the reference does.
 */
OR_EXPORT void oracle_karras(const uint32_t* m, int32_t n, int32_t* left, int32_t* right, int32_t* parents) {
    const int32_t num_nodes = n - 1, root = n;
    for (int32_t i = 0; i < num_nodes; ++i) {
        const int dd = delta(m, num_nodes, i, i + 1) - delta(m, num_nodes, i, i - 1);
        const int d = dd < 0 ? -1 : 1;
        const int delta_min = delta(m, num_nodes, i, i - d);
        int64_t l_max = 128;
        while (delta(m, num_nodes, i, (int32_t)(i + l_max * d)) > delta_min) l_max *= 4;
        int64_t l = 0;
        for (int64_t t = l_max / 2; t > 0; t /= 2)
            if (delta(m, num_nodes, i, (int32_t)(i + (l + t) * d)) > delta_min) l += t;
        const int32_t j = (int32_t)(i + l * d);
        const int delta_node = delta(m, num_nodes, i, j);
        int64_t s = 0, k = 2, t = (l + k - 1) / k;
        while (1) {
            if (delta(m, num_nodes, i, (int32_t)(i + (s + t) * d)) > delta_node) s += t;
            if (t <= 1) break;
            k *= 2;
            t = (l + k - 1) / k;
        }
        const int32_t split = (int32_t)(i + s * d + (d < 0 ? d : 0));
        const int32_t lo = i < j ? i : j, hi = i < j ? j : i;
        left[i] = lo == split ? split : -(split + 1);
        right[i] = hi == split + 1 ? split + 1 : -(split + 2);
        parents[left[i] >= 0 ? left[i] : root - (left[i] + 1)] = i;
        parents[right[i] >= 0 ? right[i] : root - (right[i] + 1)] = i;
    }
    if (n >= 1) parents[root] = -1;
}

/*
 * Independent top-down construction of the same binary radix tree: the node covering
 * [first, last] splits after the last index that shares the range's common prefix (codes
 * extended by their index, as delta does), and is numbered by the Karras convention (the
 * root is inner node 0; a child range starting at its split is inner node `split`, one ending
 * at split+1 is inner node `split+1`).  Used to pin oracle_karras.
 */
OR_EXPORT void oracle_topdown(const uint32_t* m, int32_t n, int32_t* left, int32_t* right) {
    if (n < 2) return;
    int32_t* sf = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)n);
    int32_t sp = 0;
    sf[0] = 0; sf[1] = n - 1; sf[2] = 0; sp = 1;
    while (sp > 0) {
        --sp;
        const int32_t first = sf[3 * sp], last = sf[3 * sp + 1], node = sf[3 * sp + 2];
        const int common = delta(m, n - 1, first, last);
        int32_t split = first;
        for (int32_t s = first; s < last; ++s)
            if (delta(m, n - 1, first, s) > common) split = s;
        const int32_t lnode = split == first ? split : -(split + 1);
        const int32_t rnode = split + 1 == last ? split + 1 : -(split + 2);
        left[node] = lnode;
        right[node] = rnode;
        if (lnode < 0) { sf[3 * sp] = first; sf[3 * sp + 1] = split; sf[3 * sp + 2] = split; ++sp; }
        if (rnode < 0) { sf[3 * sp] = split + 1; sf[3 * sp + 1] = last; sf[3 * sp + 2] = split + 1; ++sp; }
    }
    free(sf);
}

/* Integrity invariants of Bvh::checkTreeIntegrity (bvh.cu:568-639): every node reached
 * exactly once from the root, every inner node has two children whose parent entry points
 * back to it.  Returns 0 when they hold, else a negative code; *max_stack gets the largest
 * DFS stack (the reference's diagnostic). */
OR_EXPORT int32_t oracle_check_tree(const int32_t* left, const int32_t* right, const int32_t* parents, int32_t n,
                                    int32_t* max_stack) {
    const int32_t num_nodes = n - 1;
    int32_t* visited = (int32_t*)calloc((size_t)(2 * n), sizeof(int32_t));
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * n + 2));
    int32_t sp = 0, ms = 0, rc = 0;
    stack[sp++] = -1;
    while (sp > 0 && rc == 0) {
        const int32_t node = stack[--sp];
        int32_t idx;
        if (node >= 0) {
            if (node >= n) { rc = -1; break; }
            idx = node;
        } else {
            const int32_t k = -(node + 1);
            if (k >= num_nodes) { rc = -2; break; }
            idx = n + k;
            const int32_t ch[2] = {left[k], right[k]};
            for (int c = 0; c < 2; ++c) {
                const int32_t ci = ch[c] >= 0 ? ch[c] : n - (ch[c] + 1);
                if (ci < 0 || ci >= 2 * n - 1 || parents[ci] != k) rc = -3;
                stack[sp++] = ch[c];
            }
            if (sp > ms) ms = sp;
        }
        if (visited[idx]++) rc = -4;
    }
    for (int32_t i = 0; i < 2 * n - 1 && rc == 0; ++i)
        if (visited[i] != 1) rc = -5;
    if (rc == 0 && parents[n] != -1) rc = -6;
    if (max_stack) *max_stack = ms;
    free(visited);
    free(stack);
    return rc;
}

/* PCG32 (O'Neill 2014), restated: one output of stream (seed, node) as a float in [0,1). */
static float node_random(uint32_t seed, uint32_t node) {
    uint64_t state = 0, inc = ((uint64_t)node << 1u) | 1u;
    uint64_t old;
#define OR_STEP() (old = state, state = old * 6364136223846793005ULL + inc)
    OR_STEP();
    state += (uint64_t)seed;
    OR_STEP();
    OR_STEP();
#undef OR_STEP
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u), rot = (uint32_t)(old >> 59u);
    uint32_t v = (xs >> rot) | (xs << ((0u - rot) & 31u));
    return (float)(v >> 8) * (1.0f / 16777216.0f);
}

static float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* Cone of the union of two cones (axis a_i, cos half-angle c_i): axis along a1 + a2, and the
 * half-angle reaching both cones' far edges, using cos(x + y) = cos x cos y - sin x sin y.
 * cos = -1 is the whole sphere.  Written with one rounding per operation (no contraction)
 * so that the GPU build reproduces it bit for bit. */
static void cone_union(const float* a1, float c1, const float* a2, float c2, float* a, float* c) {
    if (c1 <= -1.0f || c2 <= -1.0f) {
        a[0] = a[1] = a[2] = 0.0f;
        *c = -1.0f;
        return;
    }
    float s[3] = {a1[0] + a2[0], a1[1] + a2[1], a1[2] + a2[2]};
    float l2 = dot3(s, s);
    if (!(l2 > 1e-12f)) {
        a[0] = a[1] = a[2] = 0.0f;
        *c = -1.0f;
        return;
    }
    float inv = 1.0f / sqrtf(l2);
    a[0] = s[0] * inv;
    a[1] = s[1] * inv;
    a[2] = s[2] * inv;
    float res = 1.0f;
    const float* ai[2] = {a1, a2};
    const float ci[2] = {c1, c2};
    for (int k = 0; k < 2; ++k) {
        float d = dot3(a, ai[k]);
        d = fminf(fmaxf(d, -1.0f), 1.0f);
        float sd = sqrtf(fmaxf(0.0f, 1.0f - d * d));
        float si = sqrtf(fmaxf(0.0f, 1.0f - ci[k] * ci[k]));
        float v = ci[k] < -d ? -1.0f : d * ci[k] - sd * si;
        res = fminf(res, v);
    }
    *c = res;
}

/*
 * Bottom-up pass (kernel_innerNodes + cluster, bvh.cu:280-316, 726-744) over a tree from
 * oracle_karras.  Inputs are the per-leaf data in sorted order.  Per inner node k:
 *   bounds[16k..]  {bbMin.xyz, left bits}, {bbMax.xyz, right bits}, {normal cone}, {direction cone}
 * Per node j in 0..2N-2 (leaf i -> i, inner k -> N+k):
 *   size, materialIndex, randomNumbers, position, normal, incRadiance (raw sum of L), incDirection
 *   records[16j..] {p.xyz, n.x}, {n.y, n.z, w.x, w.y}, {w.z, L'.rgb}, {A.rgb, count}
 *   dirstat[4j..]  {S.xyz, a}: a = sum of the antiradiance luminances a_i, S = sum of a_i w_i/|w_i|
 * The representative is left or right by rand(N+k) > |L_l| / (|L_l| + |L_r|), rand from the
 * counter-based PCG32 stream (seed, N+k).  L' = L * (0.318309886 * diffuse) of the AVPL's
 * material, or L when w = 0 (the light-source case of getRadiance).  The record's direction w is
 * that of a second representative drawn in proportion to antiradiance luminance,
 * rand(N+k) > a_l / (a_l + a_r), since w only enters the antiradiance cone test (the node-data
 * incDirection keeps the radiance representative's, as the reference's cluster() does).
 */
OR_EXPORT void oracle_bottom_up(int32_t n, const float* pos, const float* nrm, const float* w, const float* L,
                                const float* A, const int32_t* mat, const float* diffuse, const int32_t* left,
                                const int32_t* right, uint32_t seed, float* bounds, int32_t* size, int32_t* matidx,
                                float* rnd, float* npos, float* nnrm, float* nL, float* nw, float* records,
                                float* dirstat) {
    const int32_t total = 2 * n - 1;
    /* leaves */
    for (int32_t i = 0; i < n; ++i) {
        size[i] = 1;
        matidx[i] = mat[i];
        rnd[i] = node_random(seed, (uint32_t)i);
        for (int k = 0; k < 3; ++k) {
            npos[3 * i + k] = pos[3 * i + k];
            nnrm[3 * i + k] = nrm[3 * i + k];
            nL[3 * i + k] = L[3 * i + k];
            nw[3 * i + k] = w[3 * i + k];
        }
        float* r = records + 16 * (size_t)i;
        const int light = (w[3 * i] == 0.0f && w[3 * i + 1] == 0.0f && w[3 * i + 2] == 0.0f);
        float Lp[3];
        for (int k = 0; k < 3; ++k) Lp[k] = light ? L[3 * i + k] : L[3 * i + k] * (0.318309886f * diffuse[3 * mat[i] + k]);
        r[0] = pos[3 * i]; r[1] = pos[3 * i + 1]; r[2] = pos[3 * i + 2]; r[3] = nrm[3 * i];
        r[4] = nrm[3 * i + 1]; r[5] = nrm[3 * i + 2]; r[6] = w[3 * i]; r[7] = w[3 * i + 1];
        r[8] = w[3 * i + 2]; r[9] = Lp[0]; r[10] = Lp[1]; r[11] = Lp[2];
        r[12] = A[3 * i]; r[13] = A[3 * i + 1]; r[14] = A[3 * i + 2]; r[15] = 1.0f;
    }
    if (n < 2) return;
    /* leaf cones: normal cone = (n, 1); direction cone = (w/|w|, 1), or the sphere when w = 0;
       direction statistics (a w/|w|, a) */
    float* cone = (float*)malloc(sizeof(float) * 8 * (size_t)total);
    float* ds = (float*)malloc(sizeof(float) * 4 * (size_t)total);
    for (int32_t i = 0; i < n; ++i) {
        float* c = cone + 8 * (size_t)i;
        float* d = ds + 4 * (size_t)i;
        c[0] = nrm[3 * i]; c[1] = nrm[3 * i + 1]; c[2] = nrm[3 * i + 2]; c[3] = 1.0f;
        const float* wi = w + 3 * i;
        const float* ai = A + 3 * i;
        const float a = (0.2126f * ai[0] + 0.7152f * ai[1]) + 0.0722f * ai[2];
        float l2 = dot3(wi, wi);
        if (l2 > 0.0f) {
            float inv = 1.0f / sqrtf(l2);
            c[4] = wi[0] * inv; c[5] = wi[1] * inv; c[6] = wi[2] * inv; c[7] = 1.0f;
            d[0] = a * c[4]; d[1] = a * c[5]; d[2] = a * c[6];
        } else {
            c[4] = c[5] = c[6] = 0.0f; c[7] = -1.0f;
            d[0] = d[1] = d[2] = 0.0f;
        }
        d[3] = a;
    }
    float* bb = (float*)malloc(sizeof(float) * 6 * (size_t)total);
    for (int32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) bb[6 * i + k] = bb[6 * i + 3 + k] = pos[3 * i + k];
    /* post-order over inner nodes: explicit stack of (node, state) */
    int32_t* st = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)(n + 2));
    int32_t sp = 0;
    st[0] = 0; st[1] = 0; sp = 1;
    while (sp > 0) {
        int32_t k = st[2 * (sp - 1)], state = st[2 * (sp - 1) + 1];
        if (state == 0) {
            st[2 * (sp - 1) + 1] = 1;
            if (right[k] < 0) { st[2 * sp] = -(right[k] + 1); st[2 * sp + 1] = 0; ++sp; }
            if (left[k] < 0) { st[2 * sp] = -(left[k] + 1); st[2 * sp + 1] = 0; ++sp; }
            continue;
        }
        --sp;
        const int32_t t = n + k;
        const int32_t l = left[k] >= 0 ? left[k] : n - (left[k] + 1);
        const int32_t r = right[k] >= 0 ? right[k] : n - (right[k] + 1);
        for (int c = 0; c < 3; ++c) {
            bb[6 * t + c] = fminf(bb[6 * l + c], bb[6 * r + c]);
            bb[6 * t + 3 + c] = fmaxf(bb[6 * l + 3 + c], bb[6 * r + 3 + c]);
        }
        const float i1 = sqrtf(dot3(nL + 3 * l, nL + 3 * l));
        const float i2 = sqrtf(dot3(nL + 3 * r, nL + 3 * r));
        rnd[t] = node_random(seed, (uint32_t)t);
        const int32_t repr = rnd[t] > i1 / (i1 + i2) ? r : l;
        size[t] = size[l] + size[r];
        matidx[t] = matidx[repr];
        for (int c = 0; c < 3; ++c) {
            nL[3 * t + c] = nL[3 * l + c] + nL[3 * r + c];
            nw[3 * t + c] = nw[3 * repr + c];
            npos[3 * t + c] = npos[3 * repr + c];
            nnrm[3 * t + c] = nnrm[3 * repr + c];
        }
        float* rt = records + 16 * (size_t)t;
        const float* rl = records + 16 * (size_t)l;
        const float* rr = records + 16 * (size_t)r;
        const float* rp = records + 16 * (size_t)repr;
        for (int c = 0; c < 4; ++c) ds[4 * (size_t)t + c] = ds[4 * (size_t)l + c] + ds[4 * (size_t)r + c];
        const float at = ds[4 * (size_t)t + 3];
        const int32_t arep = at > 0.0f ? (rnd[t] > ds[4 * (size_t)l + 3] / at ? r : l) : repr;
        const float* ra = records + 16 * (size_t)arep;
        for (int c = 0; c < 6; ++c) rt[c] = rp[c];
        for (int c = 6; c < 9; ++c) rt[c] = ra[c];
        for (int c = 9; c < 15; ++c) rt[c] = rl[c] + rr[c];
        rt[15] = (float)size[t];
        cone_union(cone + 8 * l, cone[8 * l + 3], cone + 8 * r, cone[8 * r + 3], cone + 8 * t, cone + 8 * t + 3);
        cone_union(cone + 8 * l + 4, cone[8 * l + 7], cone + 8 * r + 4, cone[8 * r + 7], cone + 8 * t + 4,
                   cone + 8 * t + 7);
        float* b = bounds + 16 * (size_t)k;
        b[0] = bb[6 * t]; b[1] = bb[6 * t + 1]; b[2] = bb[6 * t + 2];
        memcpy(&b[3], &left[k], 4);
        b[4] = bb[6 * t + 3]; b[5] = bb[6 * t + 4]; b[6] = bb[6 * t + 5];
        memcpy(&b[7], &right[k], 4);
        for (int c = 0; c < 8; ++c) b[8 + c] = cone[8 * t + c];
    }
    if (dirstat) memcpy(dirstat, ds, sizeof(float) * 4 * (size_t)total);
    free(st);
    free(bb);
    free(cone);
    free(ds);
}

/* ---------------------------------------------------------------------------------------- */
/* Cuts                                                                                       */
/* ---------------------------------------------------------------------------------------- */

static const float kOneOverPiF = 0.318309886f; /* CUDA_ONE_OVER_PI */
static const float kPiF = 3.14159265f;         /* CUDA_PI */

/* FP64 getRadiance (cudaGather.cu:78-95) for one node-data element with the distance clamp. */
static d3 node_radiance64(d3 pos, d3 n, int mat, const float* npos, const float* nnrm, const float* nw,
                          const float* nL, const int32_t* nmat, int idx, d3 cam, const oracle_materials* M,
                          const oracle_params* P) {
    d3 pa = d3load(npos + 3 * idx), na = d3load(nnrm + 3 * idx), wa = d3load(nw + 3 * idx), La = d3load(nL + 3 * idx);
    int ma = nmat[idx];
    if (ma < 0 || ma >= M->num) ma = 0;
    return radiance_term(pos, n, mat, pa, na, wa, La, ma, cam, M, P);
}

/*
 * Per-pixel solid-angle lightcut (kernel_bvh, cudaGather.cu:316-444) over a tree from
 * oracle_bottom_up: the traversal decisions use FP32 with one rounding per operation in the
 * order the GPU kernel uses, the contributions are FP64.  Stack capacity `stack_cap`; on
 * overflow the pixel is (1e5, 0, 1e5) and err[k] = 1.
 */
OR_EXPORT void oracle_cut_solid_angle(const float* gb_pos, const float* gb_nrm, const int32_t* pixels, int32_t num_pixels,
                                      int32_t n, const float* bounds, const float* npos, const float* nnrm,
                                      const float* nw, const float* nL, const int32_t* nmat, const float* diffuse,
                                      const float* specular, const float* exponent, int32_t num_materials,
                                      const float* cam, float thresh, float dist_clamp, int32_t stack_cap,
                                      double* out_rad, int32_t* err, int32_t num_threads) {
    /* thread-private copies of the call's constants, as in oracle_gather_fp32 */
#pragma omp parallel num_threads(num_threads > 0 ? num_threads : 1)
    {
    const oracle_materials M = {diffuse, specular, exponent, num_materials};
    oracle_params P;
    memset(&P, 0, sizeof(P));
    P.dist_clamp = dist_clamp;
    const d3 c = d3load(cam);
    const float two_pi = 2.0f * kPiF;
#pragma omp for schedule(dynamic, 1)
    for (int32_t q = 0; q < num_pixels; ++q) {
        const int64_t px = pixels[q];
        const float* gp = gb_pos + 4 * px;
        const float* gn = gb_nrm + 4 * px;
        const int mat = (int)gn[3];
        d3 rad = d3m(0, 0, 0);
        int error = 0;
        if (mat > 0 && mat < num_materials) {
            d3 pos = d3load(gp), nn = d3load(gn);
            int32_t stack[256];
            int32_t sp = 0;
            stack[sp++] = -1;
            while (sp > 0) {
                const int32_t node = stack[--sp];
                int idx;
                if (node >= 0) {
                    idx = node;
                } else {
                    const int32_t k = -(node + 1);
                    const float* b = bounds + 16 * (size_t)k;
                    const float v1 = (gn[0] * (b[4] - gp[0]) + gn[1] * (b[5] - gp[1])) + gn[2] * (b[6] - gp[2]);
                    const float v0 = (gn[0] * (b[0] - gp[0]) + gn[1] * (b[1] - gp[1])) + gn[2] * (b[2] - gp[2]);
                    if (!(v1 > 0.0f || v0 > 0.0f)) continue;
                    idx = n + k;
                    const float* pr = npos + 3 * idx;
                    const float ex = b[4] - b[0], ey = b[5] - b[1], ez = b[6] - b[2];
                    const float radius = 0.5f * sqrtf((ex * ex + ey * ey) + ez * ez);
                    const float vx = pr[0] - gp[0], vy = pr[1] - gp[1], vz = pr[2] - gp[2];
                    const float dist = sqrtf((vx * vx + vy * vy) + vz * vz);
                    const float solid = two_pi * (1.0f - dist / sqrtf(radius * radius + dist * dist));
                    if (!(solid < thresh)) {
                        if (sp + 2 > stack_cap) {
                            error = 1;
                            break;
                        }
                        int32_t l, r;
                        memcpy(&l, &b[3], 4);
                        memcpy(&r, &b[7], 4);
                        stack[sp++] = l;
                        stack[sp++] = r;
                        continue;
                    }
                }
                rad = d3add(rad, node_radiance64(pos, nn, mat, npos, nnrm, nw, nL, nmat, idx, c, &M, &P));
            }
        }
        if (error) rad = d3m(100000.0, 0.0, 100000.0);
        out_rad[3 * q] = rad.x;
        out_rad[3 * q + 1] = rad.y;
        out_rad[3 * q + 2] = rad.z;
        err[q] = error;
    }
    }
}

/* --- tile cut (error bound) --------------------------------------------------------------- */

static float lum3f(float r, float g, float b) { return (0.2126f * r + 0.7152f * g) + 0.0722f * b; }

/* (a2, c2, s2): the second cone's axis, cosine and sine of its half-angle */
static float cone_max_cos(const float* a1, float c1, const float* a2, float c2, float s2) {
    if (c1 <= -1.0f || c2 <= -1.0f) return 1.0f;
    float cb = dot3(a1, a2);
    cb = fminf(fmaxf(cb, -1.0f), 1.0f);
    const float sb = sqrtf(fmaxf(0.0f, 1.0f - cb * cb));
    const float s1 = sqrtf(fmaxf(0.0f, 1.0f - c1 * c1));
    const float cg = c1 * c2 - s1 * s2;
    const float sg = s1 * c2 + c1 * s2;
    if (sg < 0.0f) return 1.0f;
    if (cb >= cg) return 1.0f;
    return cb * cg + sb * sg;
}

typedef struct {
    float tmin[3], tmax[3];
    float ncone[4];
    float kdl, tau, mean;
    int valid;
} tile_info;

/* Tile set-up of the GPU's cut_tile_setup: bounding box and normal cone of the valid pixels,
 * max receiver luminance factor, mean coarse estimate over the depth-5 cut, tau = eps * mean. */
static void tile_setup(const float* gb_pos, const float* gb_nrm, int W, int H, int tx, int ty, int n,
                       const float* bounds, const float* records, const float* diffuse, int num_materials,
                       float eps_bound, float clamp2, tile_info* t) {
    const int depth_max = 5;
    for (int k = 0; k < 3; ++k) {
        t->tmin[k] = FLT_MAX;
        t->tmax[k] = -FLT_MAX;
    }
    t->kdl = 0.0f;
    t->valid = 0;
    float P[64][6], KD[64][3];
    int V[64];
    for (int i = 0; i < 64; ++i) {
        const int x = tx * 8 + i % 8, y = ty * 8 + i / 8;
        V[i] = 0;
        for (int k = 0; k < 6; ++k) P[i][k] = 0.0f;
        if (x >= W || y >= H) continue;
        const float* gp = gb_pos + 4 * ((size_t)y * W + x);
        const float* gn = gb_nrm + 4 * ((size_t)y * W + x);
        for (int k = 0; k < 3; ++k) {
            P[i][k] = gp[k];
            P[i][3 + k] = gn[k];
        }
        const int m = (int)gn[3];
        if (m <= 0 || m >= num_materials) continue;
        V[i] = 1;
        for (int k = 0; k < 3; ++k) KD[i][k] = kOneOverPiF * diffuse[3 * m + k];
        t->kdl = fmaxf(t->kdl, lum3f(KD[i][0], KD[i][1], KD[i][2]));
        for (int k = 0; k < 3; ++k) {
            t->tmin[k] = fminf(t->tmin[k], gp[k]);
            t->tmax[k] = fmaxf(t->tmax[k], gp[k]);
        }
        t->valid++;
    }
    /* coarse cut, left-first DFS to depth 5 */
    int coarse[64], nc = 0;
    int st[64][2], top = 0;
    st[top][0] = n; st[top][1] = 0; ++top;
    while (top > 0) {
        --top;
        const int node = st[top][0], depth = st[top][1];
        if (node < n || depth == depth_max) {
            coarse[nc++] = node;
            continue;
        }
        const float* b = bounds + 16 * (size_t)(node - n);
        int32_t l, r;
        memcpy(&l, &b[3], 4);
        memcpy(&r, &b[7], 4);
        st[top][0] = r >= 0 ? r : n - (r + 1); st[top][1] = depth + 1; ++top;
        st[top][0] = l >= 0 ? l : n - (l + 1); st[top][1] = depth + 1; ++top;
    }
    float sum = 0.0f;
    float cone[4] = {0, 0, 0, -2.0f};
    for (int i = 0; i < 64; ++i) {
        if (!V[i]) continue;
        float est = 0.0f;
        for (int j = 0; j < nc; ++j) {
            const float* q = records + 16 * (size_t)coarse[j];
            const float dx = q[0] - P[i][0], dy = q[1] - P[i][1], dz = q[2] - P[i][2];
            const float l2 = (dx * dx + dy * dy) + dz * dz;
            float g = 0.0f;
            if (l2 > 0.0f) {
                const float r = 1.0f / sqrtf(l2);
                const float c1 = fmaxf(0.0f, ((P[i][3] * dx + P[i][4] * dy) + P[i][5] * dz) * r);
                const float c2 = fmaxf(0.0f, -((q[3] * dx + q[4] * dy) + q[5] * dz) * r);
                g = (c1 * c2) / fmaxf(l2, clamp2);
            }
            const float l = lum3f(KD[i][0] * q[9], KD[i][1] * q[10], KD[i][2] * q[11]);
            est = est + l * g;
        }
        sum = sum + est;
        float ci[4] = {P[i][3], P[i][4], P[i][5], 1.0f};
        if (cone[3] < -1.5f) {
            memcpy(cone, ci, sizeof(ci));
        } else if (cone[3] > -1.0f) {
            float a[3], cc;
            cone_union(cone, cone[3], ci, ci[3], a, &cc);
            cone[0] = a[0]; cone[1] = a[1]; cone[2] = a[2]; cone[3] = cc;
        }
    }
    if (cone[3] < -1.5f) { cone[0] = cone[1] = cone[2] = 0.0f; cone[3] = -1.0f; }
    memcpy(t->ncone, cone, sizeof(cone));
    t->mean = t->valid > 0 ? sum / (float)t->valid : 0.0f;
    t->tau = eps_bound * t->mean;
}

typedef struct {
    float clamp2;
    int ar_kind;
    float cos_thr, eps_cone, disk_scale;
    float ar_uncertain; /* bound multiplier when the cone test is not the same for all pairs */
} bound_params;

/* min over members of two cones of cos(angle between them); -1 when they can point opposite. */
static float cone_min_cos(const float* a1, float c1, const float* a2, float c2, float s2) {
    if (c1 <= -1.0f || c2 <= -1.0f) return -1.0f;
    float cb = dot3(a1, a2);
    cb = fminf(fmaxf(cb, -1.0f), 1.0f);
    const float sb = sqrtf(fmaxf(0.0f, 1.0f - cb * cb));
    const float s1 = sqrtf(fmaxf(0.0f, 1.0f - c1 * c1));
    const float cg = c1 * c2 - s1 * s2;
    const float sg = s1 * c2 + c1 * s2;
    if (sg < 0.0f) return -1.0f;
    if (cg < -cb) return -1.0f;
    return cb * cg - sb * sg;
}

/* node_geom + node_bound of the GPU selection (cut_bounds.cuh), same operation order. */
static float node_bound(const tile_info* t, const float* b, const float* rec, const bound_params* bp, float geom[7]) {
    const float* bmin = b;
    const float* bmax = b + 4;
    float d2 = 0.0f;
    for (int k = 0; k < 3; ++k) {
        const float gap = fmaxf(0.0f, fmaxf(bmin[k] - t->tmax[k], t->tmin[k] - bmax[k]));
        d2 = d2 + gap * gap;
    }
    const float d2c = fmaxf(d2, bp->clamp2);
    float v[3], en[3], et[3];
    for (int k = 0; k < 3; ++k) {
        const float cn = 0.5f * (bmin[k] + bmax[k]);
        const float ct = 0.5f * (t->tmin[k] + t->tmax[k]);
        v[k] = ct - cn;
        en[k] = bmax[k] - bmin[k];
        et[k] = t->tmax[k] - t->tmin[k];
    }
    const float dc = sqrtf(dot3(v, v));
    const float rn = 0.5f * sqrtf(dot3(en, en));
    const float rt = 0.5f * sqrtf(dot3(et, et));
    const float rs = rn + rt;
    float ca = -1.0f, sa = 0.0f, ax[3] = {0, 0, 0}, nax[3];
    if (dc > rs) {
        const float inv = 1.0f / dc;
        sa = rs * inv;
        ca = sqrtf(fmaxf(0.0f, 1.0f - sa * sa));
        ax[0] = v[0] * inv; ax[1] = v[1] * inv; ax[2] = v[2] * inv;
    }
    nax[0] = -ax[0]; nax[1] = -ax[1]; nax[2] = -ax[2];
    const float c2 = cone_max_cos(b + 8, b[11], ax, ca, sa);
    const float c1 = cone_max_cos(t->ncone, t->ncone[3], nax, ca, sa);
    const float cos2 = fminf(fmaxf(c2, 0.0f), 1.0f);
    const float cos1 = fminf(fmaxf(c1, 0.0f), 1.0f);
    float ar_ok = 0.0f;
    if (bp->ar_kind == 2) {
        const float cw = cone_max_cos(b + 12, b[15], ax, ca, sa);
        if (cw > bp->cos_thr && cos1 > bp->eps_cone) {
            /* every pair passes the cone test -> 1; some may fail -> the uncertainty factor */
            const float cwmin = cone_min_cos(b + 12, b[15], ax, ca, sa);
            const float c1min = cone_min_cos(t->ncone, t->ncone[3], nax, ca, sa);
            ar_ok = (cwmin > bp->cos_thr && c1min > bp->eps_cone) ? 1.0f : bp->ar_uncertain;
        }
    } else if (bp->ar_kind == 1) {
        ar_ok = 1.0f;
    }
    if (geom) {
        geom[0] = d2c; geom[1] = cos1; geom[2] = cos2; geom[3] = ar_ok; geom[4] = dc; geom[5] = rs; geom[6] = rn;
    }
    if (!(d2c > 0.0f)) return INFINITY;
    const float Ls = lum3f(rec[9], rec[10], rec[11]);
    const float As = lum3f(rec[12], rec[13], rec[14]);
    const float id2 = 1.0f / d2c;
    const float grad = (cos1 * cos2) * id2;
    float m = Ls * grad;
    if (bp->ar_kind == 2) m = m + As * (ar_ok * (cos1 * id2));
    else if (bp->ar_kind == 1) m = m + As * bp->disk_scale;
    return t->kdl * m;
}

/*
 * Error-bound tile cuts for every 8x8 tile of a W x H G-buffer: out_counts[tile] nodes in
 * out_nodes[tile * max_cut ...] (node-record index space, DFS order).  Also writes tau per
 * tile.  Returns the number of tiles whose cut exceeded max_cut (truncated).
 */
OR_EXPORT int32_t oracle_tile_cut(const float* gb_pos, const float* gb_nrm, int32_t W, int32_t H, int32_t n,
                                  const float* bounds, const float* records, const float* diffuse, int32_t num_materials,
                                  float eps_bound, float dist_clamp, int32_t ar_kind, float cone_half_angle,
                                  float disk_radius, float ar_uncertain, int32_t max_cut, int32_t* out_nodes,
                                  int32_t* out_counts, float* out_tau, int32_t num_threads) {
    const int tx_n = (W + 7) / 8, ty_n = (H + 7) / 8;
    bound_params bp;
    bp.clamp2 = dist_clamp > 0.0f ? dist_clamp * dist_clamp : 0.0f;
    bp.ar_kind = ar_kind;
    bp.eps_cone = 0.001f;
    bp.cos_thr = fmaxf(cosf(cone_half_angle), 0.001f);
    bp.disk_scale = disk_radius > 0.0f ? 1.0f / (kPiF * disk_radius * disk_radius) : 0.0f;
    bp.ar_uncertain = ar_uncertain;
    int32_t overflow = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(num_threads > 0 ? num_threads : 1) reduction(+ : overflow)
    for (int tile = 0; tile < tx_n * ty_n; ++tile) {
        tile_info t;
        tile_setup(gb_pos, gb_nrm, W, H, tile % tx_n, tile / tx_n, n, bounds, records, diffuse, num_materials,
                   eps_bound, bp.clamp2, &t);
        if (out_tau) out_tau[tile] = t.tau;
        int32_t cnt = 0;
        if (t.valid > 0) {
            int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * n + 4));
            int32_t sp = 0;
            stack[sp++] = n;
            while (sp > 0) {
                const int32_t node = stack[--sp];
                int accept = 1;
                if (node >= n) {
                    const float* b = bounds + 16 * (size_t)(node - n);
                    const float M = node_bound(&t, b, records + 16 * (size_t)node, &bp, NULL);
                    if (M > t.tau) {
                        accept = 0;
                        int32_t l, r;
                        memcpy(&l, &b[3], 4);
                        memcpy(&r, &b[7], 4);
                        stack[sp++] = r >= 0 ? r : n - (r + 1);
                        stack[sp++] = l >= 0 ? l : n - (l + 1);
                    }
                }
                if (accept) {
                    if (cnt < max_cut) out_nodes[(size_t)tile * max_cut + cnt] = node;
                    ++cnt;
                }
            }
            free(stack);
        }
        if (cnt > max_cut) {
            overflow += 1;
            cnt = max_cut;
        }
        out_counts[tile] = cnt;
    }
    return overflow;
}

/* Tile geometry and bound of one (tile, inner node) pair: geom[7] = d2c, cos1, cos2, ar_ok,
 * dc, rs, rn; returns the bound.  For feature checks. */
OR_EXPORT float oracle_node_bound(const float* gb_pos, const float* gb_nrm, int32_t W, int32_t H, int32_t tile,
                                  int32_t n, const float* bounds, const float* records, const float* diffuse,
                                  int32_t num_materials, float eps_bound, float dist_clamp, int32_t ar_kind,
                                  float cone_half_angle, float ar_uncertain, int32_t inner, float* geom,
                                  float* tile_out) {
    const int tx_n = (W + 7) / 8;
    bound_params bp;
    bp.clamp2 = dist_clamp > 0.0f ? dist_clamp * dist_clamp : 0.0f;
    bp.ar_kind = ar_kind;
    bp.eps_cone = 0.001f;
    bp.cos_thr = fmaxf(cosf(cone_half_angle), 0.001f);
    bp.disk_scale = 0.0f;
    bp.ar_uncertain = ar_uncertain;
    tile_info t;
    tile_setup(gb_pos, gb_nrm, W, H, tile % tx_n, tile / tx_n, n, bounds, records, diffuse, num_materials, eps_bound,
               bp.clamp2, &t);
    if (tile_out) {
        for (int k = 0; k < 3; ++k) {
            tile_out[k] = t.tmin[k];
            tile_out[3 + k] = t.tmax[k];
        }
        for (int k = 0; k < 4; ++k) tile_out[6 + k] = t.ncone[k];
        tile_out[10] = t.kdl;
        tile_out[11] = t.tau;
        tile_out[12] = t.mean;
        tile_out[13] = (float)t.valid;
    }
    return node_bound(&t, bounds + 16 * (size_t)inner, records + 16 * (size_t)(n + inner), &bp, geom);
}

/*
 * FP64 evaluation of given per-tile cuts over the packed node records (the GPU's cut_eval
 * arithmetic in FP64): every pixel of tile t sums the radiance and antiradiance terms of the
 * records in its cut, Lambertian receiver factor applied once.  Writes rad / antirad /
 * result [H*W*3].
 */
OR_EXPORT void oracle_eval_cut(const float* gb_pos, const float* gb_nrm, int32_t W, int32_t H, const float* records,
                               const int32_t* nodes, const int32_t* counts, int32_t stride, const float* diffuse,
                               int32_t num_materials, int32_t ar_kind, float cone_half_angle, float dist_clamp,
                               float disk_radius, double* out_rad, double* out_ar, double* out_res,
                               int32_t num_threads) {
    /* thread-private copies of the call's constants, as in oracle_gather_fp32 */
#pragma omp parallel num_threads(num_threads > 0 ? num_threads : 1)
    {
    const int tx_n = (W + 7) / 8;
    const double cos_thr = fmax(cos((double)cone_half_angle), 0.001);
    const double c2 = (double)dist_clamp * dist_clamp;
#pragma omp for schedule(dynamic, 64)
    for (int64_t px = 0; px < (int64_t)W * H; ++px) {
        const int x = (int)(px % W), y = (int)(px / W);
        const int tile = (y / 8) * tx_n + x / 8;
        const float* gp = gb_pos + 4 * px;
        const float* gn = gb_nrm + 4 * px;
        const int mat = (int)gn[3];
        double r[3] = {0, 0, 0}, a[3] = {0, 0, 0};
        if (mat > 0 && mat < num_materials) {
            d3 p = d3load(gp), nn = d3norm(d3load(gn));
            for (int j = 0; j < counts[tile]; ++j) {
                const float* q = records + 16 * (size_t)nodes[(size_t)tile * stride + j];
                d3 d = d3sub(d3m(q[0], q[1], q[2]), p);
                double l2 = d3dot(d, d);
                if (l2 < 1e-30) l2 = 1e-30;
                const double rr = 1.0 / sqrt(l2);
                const double nd = d3dot(nn, d), nad = q[3] * d.x + q[4] * d.y + q[5] * d.z;
                const double c1 = nd * rr, cc2 = -nad * rr;
                const double inv = 1.0 / (l2 > c2 ? l2 : c2);
                const double g = (c1 > 0 ? c1 : 0) * (cc2 > 0 ? cc2 : 0) * inv;
                double ga = 0;
                if (ar_kind == 2) {
                    const double cw = -(q[6] * d.x + q[7] * d.y + q[8] * d.z) * rr;
                    if (cw > cos_thr && c1 > 0.001) ga = c1 * inv;
                } else if (ar_kind == 1) {
                    const double wn = q[6] * nn.x + q[7] * nn.y + q[8] * nn.z;
                    const double ww = (double)q[6] * q[6] + (double)q[7] * q[7] + (double)q[8] * q[8];
                    if (wn < 0 && ww > 0) {
                        const double t = -nd / wn, ts = t / sqrt(ww);
                        const double hx = d.x + ts * q[6], hy = d.y + ts * q[7], hz = d.z + ts * q[8];
                        if (t > 0 && hx * hx + hy * hy + hz * hz < (double)disk_radius * disk_radius && nad > 0)
                            ga = 1.0 / (OR_PI * (double)disk_radius * disk_radius);
                    }
                }
                for (int k = 0; k < 3; ++k) {
                    r[k] += q[9 + k] * g;
                    a[k] += q[12 + k] * ga;
                }
            }
            for (int k = 0; k < 3; ++k) {
                const double kd = (double)(kOneOverPiF * diffuse[3 * mat + k]);
                r[k] *= kd;
                a[k] *= kd;
            }
        }
        for (int k = 0; k < 3; ++k) {
            out_rad[3 * px + k] = r[k];
            out_ar[3 * px + k] = a[k];
            out_res[3 * px + k] = r[k] - a[k];
        }
    }
    }
}

/* ---------------------------------------------------------------------------------------- */
/* Learned cut: tile records, the 16 features of a (tile, inner node) pair, training labels  */
/* (no counterpart in the reference; restates antiradiancecuts_b200/csrc/learned.cu with     */
/* correctly rounded operations where the GPU uses approximate log2 / rsqrt / division)      */
/* ---------------------------------------------------------------------------------------- */

/* tile record: [tmin3, tmax3, ncone4, kdl, tau, mean, valid, rt, sn] */
enum { OR_TREC = 16 };

static void tile_record(const tile_info* t, float* r) {
    for (int k = 0; k < 3; ++k) {
        r[k] = t->tmin[k];
        r[3 + k] = t->tmax[k];
    }
    for (int k = 0; k < 4; ++k) r[6 + k] = t->ncone[k];
    r[10] = t->kdl;
    r[11] = t->tau;
    r[12] = t->mean;
    r[13] = (float)t->valid;
    float et[3] = {t->tmax[0] - t->tmin[0], t->tmax[1] - t->tmin[1], t->tmax[2] - t->tmin[2]};
    r[14] = t->valid > 0 ? 0.5f * sqrtf(dot3(et, et)) : 0.0f;
    r[15] = sqrtf(fmaxf(0.0f, 1.0f - t->ncone[3] * t->ncone[3]));
}

static void tile_from_record(const float* r, tile_info* t) {
    for (int k = 0; k < 3; ++k) {
        t->tmin[k] = r[k];
        t->tmax[k] = r[3 + k];
    }
    for (int k = 0; k < 4; ++k) t->ncone[k] = r[6 + k];
    t->kdl = r[10];
    t->tau = r[11];
    t->mean = r[12];
    t->valid = (int)r[13];
}

/* Tile records of every 8x8 tile (cut_tile_setup's quantities): out [tiles][16]. */
OR_EXPORT void oracle_tile_records(const float* gb_pos, const float* gb_nrm, int32_t W, int32_t H, int32_t n,
                                   const float* bounds, const float* records, const float* diffuse,
                                   int32_t num_materials, float eps_bound, float dist_clamp, float* out,
                                   int32_t num_threads) {
    const int tx_n = (W + 7) / 8, ty_n = (H + 7) / 8;
    const float clamp2 = dist_clamp > 0.0f ? dist_clamp * dist_clamp : 0.0f;
#pragma omp parallel for schedule(dynamic, 4) num_threads(num_threads > 0 ? num_threads : 1)
    for (int tile = 0; tile < tx_n * ty_n; ++tile) {
        tile_info t;
        tile_setup(gb_pos, gb_nrm, W, H, tile % tx_n, tile / tx_n, n, bounds, records, diffuse, num_materials,
                   eps_bound, clamp2, &t);
        tile_record(&t, out + (size_t)OR_TREC * tile);
    }
}

/* Radiance and antiradiance luminance of a record {p, n, w} with luminances L, A at the point c
 * with unit normal nn (record_at of learned.cu). */
static void record_at(const float* q, float L, float A, const float* c, const float* nn, float clamp2, float cos_thr,
                      float* rad, float* ar) {
    const float dx = q[0] - c[0], dy = q[1] - c[1], dz = q[2] - c[2];
    const float l2 = fmaxf((dx * dx + dy * dy) + dz * dz, 1e-12f);
    const float r = 1.0f / sqrtf(l2);
    const float c1 = ((nn[0] * dx + nn[1] * dy) + nn[2] * dz) * r;
    const float c2 = -((q[3] * dx + q[4] * dy) + q[5] * dz) * r;
    const float inv = 1.0f / fmaxf(l2, clamp2);
    *rad = ((L * fmaxf(c1, 0.0f)) * fmaxf(c2, 0.0f)) * inv;
    const float cw = -((q[6] * dx + q[7] * dy) + q[8] * dz) * r;
    *ar = (cw > cos_thr && c1 > 0.001f) ? (A * c1) * inv : 0.0f;
}

static float clampf2(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
static float safe_log2f(float v) { return log2f(fmaxf(v, 1e-30f)); }

/* The 16 features of (tile, inner node) (node_features of learned.cu).  geom: node_bound's
 * d2c, cos1, cos2, ar_ok, dc, rs, rn; b: the node's 16-float bounds record (cones at 8 and 12);
 * rec, rl, rr: records of the node and its children; ds: the node's direction statistics.
 * aux (may be NULL): |rad - rad_l - rad_r| s, (|rad| + |rad_l| + |rad_r|) s and the same for
 * antiradiance, the conditioning of features 12 and 13. */
static void node_features(const tile_info* t, const float* geom, float M, const float* b, const float* rec,
                          const float* rl, const float* rr, const float* ds, int depth, float clamp2, float cos_thr,
                          float* f, float* aux) {
    const float E = fmaxf(t->mean, 1e-30f);
    const float dc = geom[4], rs = geom[5], rn = geom[6];
    const float inv_dc = 1.0f / fmaxf(dc, 1e-6f);
    const float rt = rs - rn;
    const float c[3] = {0.5f * (t->tmin[0] + t->tmax[0]), 0.5f * (t->tmin[1] + t->tmax[1]),
                        0.5f * (t->tmin[2] + t->tmax[2])};
    float nn[3] = {t->ncone[0], t->ncone[1], t->ncone[2]};
    const float nl = dot3(nn, nn);
    if (nl > 0.0f) {
        const float s = 1.0f / sqrtf(nl);
        nn[0] *= s;
        nn[1] *= s;
        nn[2] *= s;
    }
    const float Ls = lum3f(rec[9], rec[10], rec[11]), As = lum3f(rec[12], rec[13], rec[14]);
    float rad, ar, radl, arl, radr, arr;
    record_at(rec, Ls, As, c, nn, clamp2, cos_thr, &rad, &ar);
    record_at(rl, lum3f(rl[9], rl[10], rl[11]), lum3f(rl[12], rl[13], rl[14]), c, nn, clamp2, cos_thr, &radl, &arl);
    record_at(rr, lum3f(rr[9], rr[10], rr[11]), lum3f(rr[12], rr[13], rr[14]), c, nn, clamp2, cos_thr, &radr, &arr);
    const float s = t->kdl / E;
    f[0] = clampf2((M > 0.0f ? safe_log2f(M / fmaxf(t->tau, 1e-30f)) : -32.0f) * 0.125f, -4.0f, 4.0f);
    f[1] = clampf2(safe_log2f(Ls * s) * 0.125f, -4.0f, 4.0f);
    f[2] = clampf2(safe_log2f(As * s + 1e-20f) * 0.125f, -4.0f, 4.0f);
    f[3] = clampf2(rn * inv_dc, 0.0f, 4.0f);
    f[4] = clampf2(rt * inv_dc, 0.0f, 4.0f);
    f[5] = clampf2(sqrtf(geom[0]) * inv_dc, 0.0f, 4.0f);
    f[6] = geom[1];
    f[7] = geom[2];
    f[8] = geom[3] == 1.0f ? 1.0f : 0.0f;
    f[9] = geom[3] > 0.0f ? 1.0f : 0.0f;
    f[10] = b[11];
    f[11] = b[15];
    const float dr = fabsf((rad - radl) - radr), da = fabsf((ar - arl) - arr);
    f[12] = clampf2(safe_log2f(dr * s + 1e-20f) * 0.125f, -4.0f, 4.0f);
    f[13] = clampf2(safe_log2f(da * s + 1e-20f) * 0.125f, -4.0f, 4.0f);
    f[14] = (float)depth * (1.0f / 32.0f);
    const float sl = sqrtf((ds[0] * ds[0] + ds[1] * ds[1]) + ds[2] * ds[2]);
    f[15] = ds[3] > 0.0f ? clampf2(2.0f * (sl / ds[3]) - 1.0f, -1.0f, 1.0f) : -1.0f;
    if (aux) {
        aux[0] = dr * s;
        aux[1] = ((fabsf(rad) + fabsf(radl)) + fabsf(radr)) * s;
        aux[2] = da * s;
        aux[3] = ((fabsf(ar) + fabsf(arl)) + fabsf(arr)) * s;
    }
}

static void fill_bound_params(bound_params* bp, float dist_clamp, int32_t ar_kind, float cone_half_angle,
                              float disk_radius, float ar_uncertain) {
    bp->clamp2 = dist_clamp > 0.0f ? dist_clamp * dist_clamp : 0.0f;
    bp->ar_kind = ar_kind;
    bp->eps_cone = 0.001f;
    bp->cos_thr = fmaxf(cosf(cone_half_angle), 0.001f);
    bp->disk_scale = disk_radius > 0.0f ? 1.0f / (kPiF * disk_radius * disk_radius) : 0.0f;
    bp->ar_uncertain = ar_uncertain;
}

static int child_of(const float* b, int which, int32_t n) {
    int32_t c;
    memcpy(&c, &b[which ? 7 : 3], 4);
    return c >= 0 ? c : n - (c + 1);
}

/* Analytic bound and features of listed (tile, inner node) pairs: tile records from
 * oracle_tile_records; nodes in record index space (inner k at n + k); out_M [k], out_feat
 * [k][16], out_aux [k][4] (may be NULL). */
OR_EXPORT void oracle_pair_features(const float* tile_records, int32_t num_pairs, const int32_t* tiles,
                                    const int32_t* nodes, const int32_t* depths, int32_t n, const float* bounds,
                                    const float* records, const float* dirstat, float dist_clamp, int32_t ar_kind,
                                    float cone_half_angle, float disk_radius, float ar_uncertain, float* out_M,
                                    float* out_feat, float* out_aux, int32_t num_threads) {
    bound_params bp;
    fill_bound_params(&bp, dist_clamp, ar_kind, cone_half_angle, disk_radius, ar_uncertain);
#pragma omp parallel for schedule(static) num_threads(num_threads > 0 ? num_threads : 1)
    for (int32_t i = 0; i < num_pairs; ++i) {
        tile_info t;
        tile_from_record(tile_records + (size_t)OR_TREC * tiles[i], &t);
        const int node = nodes[i];
        const float* b = bounds + 16 * (size_t)(node - n);
        const float* rec = records + 16 * (size_t)node;
        float geom[7];
        const float M = node_bound(&t, b, rec, &bp, geom);
        out_M[i] = M;
        node_features(&t, geom, M, b, rec, records + 16 * (size_t)child_of(b, 0, n),
                      records + 16 * (size_t)child_of(b, 1, n), dirstat + 4 * (size_t)node, depths[i], bp.clamp2,
                      bp.cos_thr, out_feat + 16 * (size_t)i, out_aux ? out_aux + 4 * (size_t)i : NULL);
    }
}

/* FP64 luminance of one record's signed contribution at a pixel (p, unit normal nn) with the
 * receiver's diffuse/pi kd (record_lum of learned.cu over the pair terms of pair_math.cuh). */
static double record_lum64(const float* q, const double* p, const double* nn, const double* kd, int ar_kind,
                           double cos_thr, double inv_clamp2, double disk_r2, double disk_scale) {
    const double dx = (double)q[0] - p[0], dy = (double)q[1] - p[1], dz = (double)q[2] - p[2];
    double l2 = dx * dx + dy * dy + dz * dz;
    if (!(l2 > 1e-30)) l2 = 1e-30;
    const double r = 1.0 / sqrt(l2);
    const double nd = nn[0] * dx + nn[1] * dy + nn[2] * dz;
    const double nad = q[3] * dx + q[4] * dy + q[5] * dz;
    const double c1 = nd * r, c2 = -nad * r;
    const double rr = r * r;
    const double inv = rr < inv_clamp2 ? rr : inv_clamp2;
    const double g = (c1 > 0 ? c1 : 0) * (c2 > 0 ? c2 : 0) * inv;
    double ga = 0.0, as = 1.0;
    if (ar_kind == 2) {
        const double cw = -(q[6] * dx + q[7] * dy + q[8] * dz) * r;
        ga = (cw > cos_thr && c1 > 0.001) ? c1 * inv : 0.0;
    } else if (ar_kind == 1) {
        const double ww = (double)q[6] * q[6] + (double)q[7] * q[7] + (double)q[8] * q[8];
        const double wn = q[6] * nn[0] + q[7] * nn[1] + q[8] * nn[2];
        if (ww > 0 && wn < 0) {
            const double t = -nd / wn, ts = t / sqrt(ww);
            const double hx = dx + ts * q[6], hy = dy + ts * q[7], hz = dz + ts * q[8];
            if (t > 0 && hx * hx + hy * hy + hz * hz < disk_r2 && nad > 0) ga = 1.0;
        }
        as = disk_scale;
    }
    const double c0 = kd[0] * (q[9] * g - as * q[12] * ga), cc1 = kd[1] * (q[10] * g - as * q[13] * ga),
                 cc2 = kd[2] * (q[11] * g - as * q[14] * ga);
    return 0.2126 * c0 + 0.7152 * cc1 + 0.0722 * cc2;
}

/*
 * Training samples of the learned cut (arc_cut_training_samples): for every 8x8 tile with a
 * surface, the exact per-pixel contribution of each node (FP64 over its leaves), and the
 * labelling walk of label_traverse: depth-first from the root, nodes the analytic bound
 * accepts are skipped, nodes above band times tau are refined without a sample, every other
 * node gets a sample (features, label = RMS over the tile's pixels of |exact - node estimate| >
 * delta * mean |exact tile value|, error = that RMS / the mean) and its children are walked; the
 * children of an accepted node are sampled one level only.  Samples are written tile after tile,
 * each tile's in walk order.  keys [cap][2] = (tile, node).  Returns the number of samples (may
 * exceed capacity: only the first `capacity` are written).
 */
OR_EXPORT int32_t oracle_training_samples(const float* gb_pos, const float* gb_nrm, int32_t W, int32_t H, int32_t n,
                                          const float* bounds, const float* records, const float* dirstat,
                                          const float* diffuse, int32_t num_materials, float eps_bound,
                                          float dist_clamp, int32_t ar_kind, float cone_half_angle,
                                          float disk_radius, float ar_uncertain, float band, float delta,
                                          int32_t capacity, int32_t* out_keys, float* out_feat, float* out_labels,
                                          float* out_errs, int32_t num_threads) {
    const int tx_n = (W + 7) / 8, ty_n = (H + 7) / 8, tiles = tx_n * ty_n;
    bound_params bp;
    fill_bound_params(&bp, dist_clamp, ar_kind, cone_half_angle, disk_radius, ar_uncertain);
    const double cos_thr = (double)bp.cos_thr;
    const double inv_clamp2 = dist_clamp > 0.0f ? 1.0 / (double)bp.clamp2 : INFINITY;
    const double disk_r2 = (double)disk_radius * disk_radius;
    const double disk_scale = (double)bp.disk_scale;
    /* leaf range [first, last] of every inner node: the leftmost and rightmost leaf below it */
    int32_t* range = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)(n > 1 ? n - 1 : 1));
    for (int32_t k = 0; k + 1 < n; ++k) {
        int node = n + k;
        while (node >= n) node = child_of(bounds + 16 * (size_t)(node - n), 0, n);
        range[2 * k] = node;
        node = n + k;
        while (node >= n) node = child_of(bounds + 16 * (size_t)(node - n), 1, n);
        range[2 * k + 1] = node;
    }
    int32_t* tcount = (int32_t*)calloc((size_t)tiles, sizeof(int32_t));
    int32_t** tkeys = (int32_t**)calloc((size_t)tiles, sizeof(int32_t*));
    float** tfeat = (float**)calloc((size_t)tiles, sizeof(float*));
    float** tlab = (float**)calloc((size_t)tiles, sizeof(float*));
#pragma omp parallel num_threads(num_threads > 0 ? num_threads : 1)
    {
        double* P = (double*)malloc(sizeof(double) * 64 * (size_t)(n + 1));
        int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * 3 * 256);
#pragma omp for schedule(dynamic, 1)
        for (int tile = 0; tile < tiles; ++tile) {
            tile_info t;
            tile_setup(gb_pos, gb_nrm, W, H, tile % tx_n, tile / tx_n, n, bounds, records, diffuse, num_materials,
                       eps_bound, bp.clamp2, &t);
            if (t.valid == 0) continue;
            double px[64][3], nn[64][3], kd[64][3];
            int valid[64], nv = 0;
            for (int p = 0; p < 64; ++p) {
                const int x = (tile % tx_n) * 8 + p % 8, y = (tile / tx_n) * 8 + p / 8;
                valid[p] = 0;
                if (x >= W || y >= H) continue;
                const float* gp = gb_pos + 4 * ((size_t)y * W + x);
                const float* gn = gb_nrm + 4 * ((size_t)y * W + x);
                const int m = (int)gn[3];
                if (m <= 0 || m >= num_materials) continue;
                const double l = sqrt((double)gn[0] * gn[0] + (double)gn[1] * gn[1] + (double)gn[2] * gn[2]);
                for (int k = 0; k < 3; ++k) {
                    px[p][k] = gp[k];
                    nn[p][k] = gn[k] / l;
                    kd[p][k] = (double)(kOneOverPiF * diffuse[3 * m + k]);
                }
                valid[p] = 1;
                ++nv;
            }
            /* P[i][p]: sum of the first i leaves' contributions at pixel p */
            for (int p = 0; p < 64; ++p) P[p] = 0.0;
            for (int32_t i = 0; i < n; ++i) {
                const float* q = records + 16 * (size_t)i;
                for (int p = 0; p < 64; ++p)
                    P[64 * (size_t)(i + 1) + p] =
                        P[64 * (size_t)i + p] +
                        (valid[p] ? record_lum64(q, px[p], nn[p], kd[p], ar_kind, cos_thr, inv_clamp2, disk_r2,
                                                 disk_scale)
                                  : 0.0);
            }
            double E = 0.0;
            for (int p = 0; p < 64; ++p)
                if (valid[p]) E += fabs(P[64 * (size_t)n + p]);
            E /= (double)nv;
            const double thr = (double)delta * E;
            int cap_t = 256, cnt = 0;
            int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * 2 * cap_t);
            float* feat = (float*)malloc(sizeof(float) * 16 * cap_t);
            float* lab = (float*)malloc(sizeof(float) * 2 * cap_t);
            /* stack entries: node, depth, extra */
            int sp = 0;
            stack[0] = n; stack[1] = 0; stack[2] = 0; sp = 1;
            int64_t budget = 4 * (int64_t)n;
            while (sp > 0 && --budget > 0) {
                --sp;
                const int node = stack[3 * sp], depth = stack[3 * sp + 1], extra = stack[3 * sp + 2];
                if (node < n) continue;
                const float* b = bounds + 16 * (size_t)(node - n);
                const float* rec = records + 16 * (size_t)node;
                float geom[7];
                const float M = node_bound(&t, b, rec, &bp, geom);
                if (!(M > t.tau)) continue;
                const int c0 = child_of(b, 0, n), c1 = child_of(b, 1, n);
                const int d1 = depth + 1 < 127 ? depth + 1 : 127;
                if (M > band * t.tau) {
                    if (!extra && sp + 2 <= 256) {
                        stack[3 * sp] = c1; stack[3 * sp + 1] = d1; stack[3 * sp + 2] = 0; ++sp;
                        stack[3 * sp] = c0; stack[3 * sp + 1] = d1; stack[3 * sp + 2] = 0; ++sp;
                    }
                    continue;
                }
                const int k = node - n, f0 = range[2 * k], l0 = range[2 * k + 1];
                double e2 = 0.0;
                for (int p = 0; p < 64; ++p) {
                    if (!valid[p]) continue;
                    const double exact = P[64 * (size_t)(l0 + 1) + p] - P[64 * (size_t)f0 + p];
                    const double approx =
                        record_lum64(rec, px[p], nn[p], kd[p], ar_kind, cos_thr, inv_clamp2, disk_r2, disk_scale);
                    e2 += (exact - approx) * (exact - approx);
                }
                const double erms = sqrt(e2 / (double)nv);
                const int refine = erms > thr;
                if (cnt == cap_t) {
                    cap_t *= 2;
                    keys = (int32_t*)realloc(keys, sizeof(int32_t) * 2 * cap_t);
                    feat = (float*)realloc(feat, sizeof(float) * 16 * cap_t);
                    lab = (float*)realloc(lab, sizeof(float) * 2 * cap_t);
                }
                keys[2 * cnt] = tile;
                keys[2 * cnt + 1] = node;
                node_features(&t, geom, M, b, rec, records + 16 * (size_t)c0, records + 16 * (size_t)c1,
                              dirstat + 4 * (size_t)node, depth, bp.clamp2, bp.cos_thr, feat + 16 * (size_t)cnt, NULL);
                lab[2 * cnt] = refine ? 1.0f : 0.0f;
                lab[2 * cnt + 1] = E > 0.0 ? (float)(erms / E) : 0.0f;
                ++cnt;
                if (extra || sp + 2 > 256) continue;
                stack[3 * sp] = c1; stack[3 * sp + 1] = d1; stack[3 * sp + 2] = !refine; ++sp;
                stack[3 * sp] = c0; stack[3 * sp + 1] = d1; stack[3 * sp + 2] = !refine; ++sp;
            }
            tcount[tile] = cnt;
            tkeys[tile] = keys;
            tfeat[tile] = feat;
            tlab[tile] = lab;
        }
        free(stack);
        free(P);
    }
    int64_t total = 0;
    for (int tile = 0; tile < tiles; ++tile) {
        for (int j = 0; j < tcount[tile]; ++j, ++total) {
            if (total >= capacity) continue;
            out_keys[2 * total] = tkeys[tile][2 * j];
            out_keys[2 * total + 1] = tkeys[tile][2 * j + 1];
            memcpy(out_feat + 16 * (size_t)total, tfeat[tile] + 16 * (size_t)j, 16 * sizeof(float));
            out_labels[total] = tlab[tile][2 * j];
            out_errs[total] = tlab[tile][2 * j + 1];
        }
        free(tkeys[tile]);
        free(tfeat[tile]);
        free(tlab[tile]);
    }
    free(tcount);
    free(tkeys);
    free(tfeat);
    free(tlab);
    free(range);
    return (int32_t)(total < INT32_MAX ? total : INT32_MAX);
}
