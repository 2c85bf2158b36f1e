// Synthetic-scene math shared by the CPU generator (scene_gen.cpp, g++) and the GPU one
// (scene_gpu.cu, nvcc with -fmad=false): geometry, ray / rectangle intersection, the cosine
// sampler, the Phong BRDF, the light-path tracer with the AVPL semantics of
// AvplShooter::createPath (AvplShooter.h:77-142) and the primary-ray G-buffer.  Every
// floating-point operation is a single IEEE-rounded add, multiply, divide or square root, in
// source order and never contracted into an FMA, so the G-buffer is the same bits on both.  The
// tracer's azimuth goes through cosf / sinf (and a specular lobe through powf), whose host and
// device libraries may differ in the last bit: the GPU's AVPLs then differ from the CPU's by
// rounding, and a path that grazes an edge may take another turn.
#ifndef ARC_SCENE_MATH_H_
#define ARC_SCENE_MATH_H_

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "arc_api.h"
#include "pcg32.h"

namespace arc {
namespace scene {

struct V3 {
    float x, y, z;
};

ARC_HD inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
ARC_HD inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
ARC_HD inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
ARC_HD inline V3 scale(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
ARC_HD inline V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
ARC_HD inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
ARC_HD inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
ARC_HD inline V3 normalize(V3 a) { return scale(1.0f / sqrtf(dot(a, a)), a); }
ARC_HD inline float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
ARC_HD inline V3 fromA(ArcFloat3 a) { return v3(a.x, a.y, a.z); }
ARC_HD inline ArcFloat3 toA(V3 a) { return ArcFloat3{a.x, a.y, a.z}; }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kEps = 1e-4f;    // Defines.h:13
constexpr float kRRProb = 0.8f;  // AvplShooter.h:78

// Axis-aligned rectangle: plane `axis` = c, spanning [u0,u1] x [v0,v1] in the two other axes,
// facing `sign` along the axis.  Only its front side is hit (Triangle::FRONT_FACE).
struct Rect {
    int axis;
    float c;
    float u0, u1, v0, v1;
    float sign;
    int material;
};

// 5 room faces + the light + 6 faces per box
constexpr int kMaxRects = 6 + 6 * ARC_SCENE_MAX_BOXES;

// The two in-plane axes of `axis`, in increasing order.
ARC_HD inline void other_axes(int axis, int& a, int& b) {
    a = axis == 0 ? 1 : 0;
    b = axis == 2 ? 1 : 2;
}

// The scene's rectangles in intersection order; returns their count (<= kMaxRects).
ARC_HD inline int build_rects(const ArcSceneDesc& s, Rect* r) {
    int n = 0;
    // Room [0,1]^3 with the z = 0 face open; normals point into the room.
    // materials: 1 gray, 2 red (left, x = 0), 3 green (right, x = 1)
    r[n++] = Rect{1, 0.0f, 0, 1, 0, 1, +1.0f, 1};  // floor
    r[n++] = Rect{1, 1.0f, 0, 1, 0, 1, -1.0f, 1};  // ceiling
    r[n++] = Rect{2, 1.0f, 0, 1, 0, 1, -1.0f, 1};  // back wall
    r[n++] = Rect{0, 0.0f, 0, 1, 0, 1, +1.0f, 2};  // left wall
    r[n++] = Rect{0, 1.0f, 0, 1, 0, 1, -1.0f, 3};  // right wall
    const float h = s.light_half_size;
    r[n++] = Rect{1,
                  s.light_center.y,
                  s.light_center.x - h,
                  s.light_center.x + h,
                  s.light_center.z - h,
                  s.light_center.z + h,
                  -1.0f,
                  s.light_material};
    const int nb = s.num_boxes < 0 ? 0 : (s.num_boxes > ARC_SCENE_MAX_BOXES ? ARC_SCENE_MAX_BOXES : s.num_boxes);
    for (int i = 0; i < nb; ++i) {
        const ArcBox& b = s.boxes[i];
        const float lo[3] = {b.lo.x, b.lo.y, b.lo.z};
        const float hi[3] = {b.hi.x, b.hi.y, b.hi.z};
        for (int axis = 0; axis < 3; ++axis) {
            int a, c;
            other_axes(axis, a, c);
            r[n++] = Rect{axis, lo[axis], lo[a], hi[a], lo[c], hi[c], -1.0f, b.material};
            r[n++] = Rect{axis, hi[axis], lo[a], hi[a], lo[c], hi[c], +1.0f, b.material};
        }
    }
    return n;
}

struct Hit {
    float t;
    V3 p;
    V3 n;
    int material;
};

// Nearest front-facing rectangle along o + t d (t > 0); the hit point is snapped onto its plane.
ARC_HD inline bool intersect(const Rect* rects, int nrects, V3 o, V3 d, Hit& hit) {
    hit.t = INFINITY;
    int best = -1;
    for (int i = 0; i < nrects; ++i) {
        const Rect& r = rects[i];
        const float dk = comp(d, r.axis);
        if (dk * r.sign >= 0.0f) continue;  // back face or parallel
        const float t = (r.c - comp(o, r.axis)) / dk;
        if (!(t > 0.0f) || t >= hit.t) continue;
        int a, b;
        other_axes(r.axis, a, b);
        const float pa = comp(o, a) + t * comp(d, a);
        const float pb = comp(o, b) + t * comp(d, b);
        if (pa < r.u0 || pa > r.u1 || pb < r.v0 || pb > r.v1) continue;
        hit.t = t;
        best = i;
    }
    if (best < 0) return false;
    const Rect& r = rects[best];
    hit.p = add(o, scale(hit.t, d));
    float n[3] = {0, 0, 0};
    n[r.axis] = r.sign;
    hit.n = v3(n[0], n[1], n[2]);
    if (r.axis == 0) hit.p.x = r.c;
    if (r.axis == 1) hit.p.y = r.c;
    if (r.axis == 2) hit.p.z = r.c;
    hit.material = r.material;
    return true;
}

// Orthonormal basis around unit n (Duff et al., "Building an Orthonormal Basis, Revisited", 2017).
ARC_HD inline void onb(V3 n, V3& t, V3& b) {
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float bb = n.x * n.y * a;
    t = v3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = v3(bb, sign + n.y * n.y * a, -n.y);
}

// Cosine-weighted direction around n: cos(theta) = sqrt(u1), phi = 2 pi u2, pdf = cos/pi
// (sampleCosCone with order 1, Sampler.h:13-35).
ARC_HD inline V3 sample_cosine(V3 n, float u1, float u2, float& pdf) {
    const float cos_t = sqrtf(u1);
    const float sin_t = sqrtf(fmaxf(0.0f, 1.0f - u1));
    const float phi = 2.0f * kPi * u2;
    const float cp = cosf(phi), sp = sinf(phi);
    V3 t, b;
    onb(n, t, b);
    V3 d = add(add(scale(sin_t * cp, t), scale(sin_t * sp, b)), scale(cos_t, n));
    d = normalize(d);
    pdf = cos_t / kPi;
    return d;
}

// phong_eval (Brdf.h:9-21)
ARC_HD inline V3 phong_eval(V3 w_i, V3 w_o, V3 n, const ArcMaterial& m) {
    if (dot(w_i, n) <= 0.0f || dot(w_o, n) <= 0.0f) return v3(0, 0, 0);
    V3 res = v3(0, 0, 0);
    const V3 spec = fromA(m.specular);
    if (sqrtf(dot(spec, spec)) > 0.0f) {
        const V3 r = sub(scale(2.0f * dot(w_i, n), n), w_i);  // reflect(w_i, n) mirrored about n
        const float c = fmaxf(0.0f, dot(r, w_o));
        res = add(res, scale((0.5f / kPi) * (m.exponent + 2.0f) * powf(c, m.exponent), spec));
    }
    res = add(res, scale(1.0f / kPi, fromA(m.diffuse)));
    return res;
}

// One light path (PCG32 stream `path` of `seed`); calls emit(avpl) for each of its indirect
// AVPLs, at most max_bounces of them.
template <typename Emit>
ARC_HD inline void trace_path(const ArcSceneDesc& s, const Rect* rects, int nrects, uint64_t seed, uint64_t path,
                              int max_bounces, bool explicit_direct, Emit&& emit) {
    arc_pcg32 rng;
    arc_pcg32_seed(&rng, seed, path);
    // sample the light: uniform on the square, pdf = 1 / area (AreaLight::samplePos)
    const float u0 = arc_pcg32_float(&rng), u1 = arc_pcg32_float(&rng);
    const float h = s.light_half_size;
    V3 pos = v3(s.light_center.x - h + 2.0f * h * u0, s.light_center.y, s.light_center.z - h + 2.0f * h * u1);
    V3 normal = v3(0.0f, -1.0f, 0.0f);
    const float area = 4.0f * h * h;
    V3 L = scale(area, fromA(s.light_radiance));  // rad / pdf
    V3 w = v3(0, 0, 0);
    int bounce = 0;
    int material = s.light_material;

    // each direction takes two draws: the first is the azimuth u2, the second the cosine u1
    float pdf;
    const float r2 = arc_pcg32_float(&rng);
    const float r1 = arc_pcg32_float(&rng);
    V3 dir = sample_cosine(normal, r1, r2, pdf);
    while (true) {
        Hit hit;
        if (!intersect(rects, nrects, add(pos, scale(kEps, normal)), dir, hit)) break;
        const float cos_t = dot(normal, dir);
        V3 contrib = scale(cos_t / pdf, L);
        if (bounce > 0) contrib = mul(contrib, phong_eval(scale(-1.0f, w), dir, normal, s.materials[material]));
        pos = sub(hit.p, scale(kEps, hit.n));
        normal = hit.n;
        w = dir;
        bounce += 1;
        material = hit.material;
        V3 A = contrib;
        if (bounce == 1 && explicit_direct) A = v3(0, 0, 0);
        const bool terminate = arc_pcg32_float(&rng) > kRRProb;
        L = terminate ? v3(0, 0, 0) : scale(1.0f / kRRProb, contrib);
        ArcAvplHost a;
        a.position = toA(pos);
        a.normal = toA(normal);
        a.incRadiance = toA(L);
        a.antiradiance = toA(A);
        a.incDirection = toA(w);
        a.bounce = bounce;
        a.materialIndex = material;
        emit(a);
        if (terminate || bounce >= max_bounces) break;
        const float q2 = arc_pcg32_float(&rng);
        const float q1 = arc_pcg32_float(&rng);
        dir = sample_cosine(normal, q1, q2, pdf);
        if (pdf < 1e-4f) break;  // AvplShooter.h:137-140
    }
}

// Pinhole camera of the scene for a width x height image: eye, unit forward / right / up, and
// tan of half the vertical field of view (computed once on the host: tanf is not shared).
struct Camera {
    V3 eye, fwd, right, up;
    float tan_half, aspect;
};

inline Camera make_camera(const ArcSceneDesc& s, int width, int height) {
    Camera c;
    c.eye = fromA(s.camera_position);
    c.fwd = normalize(sub(fromA(s.camera_target), c.eye));
    c.right = normalize(cross(c.fwd, v3(0, 1, 0)));
    c.up = cross(c.right, c.fwd);
    c.tan_half = tanf(0.5f * s.camera_fov_deg * kPi / 180.0f);
    c.aspect = (float)width / (float)height;
    return c;
}

// G-buffer texel (x, y): position (x, y, z, 1) and normal (n, material) of the primary hit, or
// zeros.
ARC_HD inline void gbuffer_texel(const Camera& c, const Rect* rects, int nrects, int width, int height, int x, int y,
                                 float* P, float* N) {
    const float sx = (2.0f * ((float)x + 0.5f) / (float)width - 1.0f) * c.aspect * c.tan_half;
    const float sy = (1.0f - 2.0f * ((float)y + 0.5f) / (float)height) * c.tan_half;
    const V3 d = normalize(add(add(c.fwd, scale(sx, c.right)), scale(sy, c.up)));
    Hit hit;
    if (intersect(rects, nrects, c.eye, d, hit)) {
        P[0] = hit.p.x; P[1] = hit.p.y; P[2] = hit.p.z; P[3] = 1.0f;
        N[0] = hit.n.x; N[1] = hit.n.y; N[2] = hit.n.z; N[3] = (float)hit.material;
    } else {
        P[0] = P[1] = P[2] = P[3] = 0.0f;
        N[0] = N[1] = N[2] = N[3] = 0.0f;
    }
}

}  // namespace scene
}  // namespace arc

#endif  // ARC_SCENE_MATH_H_
