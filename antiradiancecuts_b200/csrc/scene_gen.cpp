// Synthetic scenes for the gather: an open-front box room with axis-aligned boxes, a square
// area light, a pinhole camera, a light tracer that emits AVPLs with the semantics of
// AvplShooter::createPath (AvplShooter.h:77-142), and a primary-ray G-buffer that stands in for
// the reference's rasterised CreateGBuffer pass (Render.cpp:740-750).  CPU only: these make the
// inputs of the GPU path, they are not part of it.
#include "arc_api.h"
#include "pcg32.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

struct V3 {
    float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline V3 normalize(V3 a) { return (1.0f / std::sqrt(dot(a, a))) * a; }
inline float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
inline V3 fromA(ArcFloat3 a) { return v3(a.x, a.y, a.z); }
inline ArcFloat3 toA(V3 a) { return ArcFloat3{a.x, a.y, a.z}; }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kEps = 1e-4f;      // Defines.h:13
constexpr float kRRProb = 0.8f;    // AvplShooter.h:78

// Axis-aligned rectangle: plane `axis` = c, spanning [u0,u1] x [v0,v1] in the two other axes,
// facing `sign` along the axis.  Only its front side is hit (Triangle::FRONT_FACE).
struct Rect {
    int axis;
    float c;
    float u0, u1, v0, v1;
    float sign;
    int material;
};

struct Geometry {
    std::vector<Rect> rects;
};

void add_rect(Geometry& g, int axis, float c, float u0, float u1, float v0, float v1, float sign, int mat) {
    g.rects.push_back(Rect{axis, c, u0, u1, v0, v1, sign, mat});
}

// The two in-plane axes of `axis`, in increasing order.
inline void other_axes(int axis, int& a, int& b) {
    a = axis == 0 ? 1 : 0;
    b = axis == 2 ? 1 : 2;
}

void add_box(Geometry& g, const ArcBox& b) {
    const float lo[3] = {b.lo.x, b.lo.y, b.lo.z};
    const float hi[3] = {b.hi.x, b.hi.y, b.hi.z};
    for (int axis = 0; axis < 3; ++axis) {
        int a, c;
        other_axes(axis, a, c);
        add_rect(g, axis, lo[axis], lo[a], hi[a], lo[c], hi[c], -1.0f, b.material);
        add_rect(g, axis, hi[axis], lo[a], hi[a], lo[c], hi[c], +1.0f, b.material);
    }
}

Geometry build_geometry(const ArcSceneDesc& s) {
    Geometry g;
    // Room [0,1]^3 with the z = 0 face open; normals point into the room.
    // materials: 1 gray, 2 red (left, x = 0), 3 green (right, x = 1)
    add_rect(g, 1, 0.0f, 0, 1, 0, 1, +1.0f, 1);   // floor
    add_rect(g, 1, 1.0f, 0, 1, 0, 1, -1.0f, 1);   // ceiling
    add_rect(g, 2, 1.0f, 0, 1, 0, 1, -1.0f, 1);   // back wall
    add_rect(g, 0, 0.0f, 0, 1, 0, 1, +1.0f, 2);   // left wall
    add_rect(g, 0, 1.0f, 0, 1, 0, 1, -1.0f, 3);   // right wall
    const float h = s.light_half_size;
    add_rect(g, 1, s.light_center.y, s.light_center.x - h, s.light_center.x + h, s.light_center.z - h,
             s.light_center.z + h, -1.0f, s.light_material);
    for (int i = 0; i < s.num_boxes; ++i) add_box(g, s.boxes[i]);
    return g;
}

struct Hit {
    float t;
    V3 p;
    V3 n;
    int material;
};

bool intersect(const Geometry& g, V3 o, V3 d, Hit& hit) {
    hit.t = INFINITY;
    const Rect* best = nullptr;
    for (const Rect& r : g.rects) {
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
        best = &r;
    }
    if (!best) return false;
    hit.p = o + hit.t * d;
    float n[3] = {0, 0, 0};
    n[best->axis] = best->sign;
    hit.n = v3(n[0], n[1], n[2]);
    // snap the hit onto the plane exactly
    if (best->axis == 0) hit.p.x = best->c;
    if (best->axis == 1) hit.p.y = best->c;
    if (best->axis == 2) hit.p.z = best->c;
    hit.material = best->material;
    return true;
}

// Orthonormal basis around unit n (Duff et al., "Building an Orthonormal Basis, Revisited", 2017).
void onb(V3 n, V3& t, V3& b) {
    const float sign = std::copysign(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float bb = n.x * n.y * a;
    t = v3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = v3(bb, sign + n.y * n.y * a, -n.y);
}

// Cosine-weighted direction around n: cos(theta) = sqrt(u1), phi = 2 pi u2, pdf = cos/pi
// (sampleCosCone with order 1, Sampler.h:13-35).
V3 sample_cosine(V3 n, float u1, float u2, float& pdf) {
    const float cos_t = std::sqrt(u1);
    const float sin_t = std::sqrt(std::fmax(0.0f, 1.0f - u1));
    const float phi = 2.0f * kPi * u2;
    V3 t, b;
    onb(n, t, b);
    V3 d = (sin_t * std::cos(phi)) * t + (sin_t * std::sin(phi)) * b + cos_t * n;
    d = normalize(d);
    pdf = cos_t / kPi;
    return d;
}

// phong_eval (Brdf.h:9-21)
V3 phong_eval(V3 w_i, V3 w_o, V3 n, const ArcMaterial& m) {
    if (dot(w_i, n) <= 0.0f || dot(w_o, n) <= 0.0f) return v3(0, 0, 0);
    V3 res = v3(0, 0, 0);
    const V3 spec = fromA(m.specular);
    if (std::sqrt(dot(spec, spec)) > 0.0f) {
        const V3 r = 2.0f * dot(w_i, n) * n - w_i;  // reflect(w_i, n) mirrored about n
        const float c = std::fmax(0.0f, dot(r, w_o));
        res = res + ((0.5f / kPi) * (m.exponent + 2.0f) * std::pow(c, m.exponent)) * spec;
    }
    res = res + (1.0f / kPi) * fromA(m.diffuse);
    return res;
}

// One light path; appends its indirect AVPLs to `out` (at most max_bounces of them).
void trace_path(const ArcSceneDesc& s, const Geometry& g, uint64_t seed, uint64_t path, int max_bounces,
                bool explicit_direct, std::vector<ArcAvplHost>& out) {
    arc_pcg32 rng;
    arc_pcg32_seed(&rng, seed, path);
    // sample the light: uniform on the square, pdf = 1 / area (AreaLight::samplePos)
    const float u0 = arc_pcg32_float(&rng), u1 = arc_pcg32_float(&rng);
    const float h = s.light_half_size;
    V3 pos = v3(s.light_center.x - h + 2.0f * h * u0, s.light_center.y, s.light_center.z - h + 2.0f * h * u1);
    V3 normal = v3(0.0f, -1.0f, 0.0f);
    const float area = 4.0f * h * h;
    V3 L = area * fromA(s.light_radiance);  // rad / pdf
    V3 w = v3(0, 0, 0);
    int bounce = 0;
    int material = s.light_material;

    float pdf;
    V3 dir = sample_cosine(normal, arc_pcg32_float(&rng), arc_pcg32_float(&rng), pdf);
    while (true) {
        Hit hit;
        if (!intersect(g, pos + kEps * normal, dir, hit)) break;
        const float cos_t = dot(normal, dir);
        V3 contrib = (cos_t / pdf) * L;
        if (bounce > 0) contrib = mul(contrib, phong_eval(-1.0f * w, dir, normal, s.materials[material]));
        ArcAvplHost a;
        pos = hit.p - kEps * hit.n;
        normal = hit.n;
        w = dir;
        bounce += 1;
        material = hit.material;
        V3 A = contrib;
        if (bounce == 1 && explicit_direct) A = v3(0, 0, 0);
        const bool terminate = arc_pcg32_float(&rng) > kRRProb;
        L = terminate ? v3(0, 0, 0) : (1.0f / kRRProb) * contrib;
        a.position = toA(pos);
        a.normal = toA(normal);
        a.incRadiance = toA(L);
        a.antiradiance = toA(A);
        a.incDirection = toA(w);
        a.bounce = bounce;
        a.materialIndex = material;
        out.push_back(a);
        if (terminate || bounce >= max_bounces) break;
        dir = sample_cosine(normal, arc_pcg32_float(&rng), arc_pcg32_float(&rng), pdf);
        if (pdf < 1e-4f) break;  // AvplShooter.h:137-140
    }
}

ArcMaterial lambert(float r, float g, float b) {
    ArcMaterial m;
    std::memset(&m, 0, sizeof(m));
    m.diffuse = ArcFloat3{r, g, b};
    m.exponent = 1.0f;
    return m;
}

}  // namespace

extern "C" arc_status arc_scene_preset_desc(int32_t preset, uint64_t seed, int32_t num_boxes, ArcSceneDesc* out) {
    if (!out || preset < 0 || preset > ARC_SCENE_TRAIN_VARIANT || num_boxes < 0 ||
        num_boxes > ARC_SCENE_MAX_BOXES - 2)
        return ARC_ERR_INVALID_ARG;
    ArcSceneDesc& s = *out;
    std::memset(&s, 0, sizeof(s));
    // material 0: no surface; 1 gray; 2 red; 3 green; 4 light (black, emissive)
    s.materials[0] = lambert(0, 0, 0);
    s.materials[1] = lambert(0.7f, 0.7f, 0.7f);
    s.materials[2] = lambert(0.63f, 0.065f, 0.05f);
    s.materials[3] = lambert(0.14f, 0.45f, 0.09f);
    s.materials[4] = lambert(0, 0, 0);
    s.materials[4].emissive = ArcFloat3{17.0f, 12.0f, 4.0f};
    s.num_materials = 5;
    s.light_center = ArcFloat3{0.5f, 0.999f, 0.5f};
    s.light_half_size = 0.125f;
    s.light_radiance = ArcFloat3{17.0f, 12.0f, 4.0f};
    s.light_material = 4;
    s.camera_position = ArcFloat3{0.5f, 0.5f, -1.4f};
    s.camera_target = ArcFloat3{0.5f, 0.5f, 0.0f};
    s.camera_fov_deg = 40.0f;
    s.scene_min = ArcFloat3{0, 0, 0};
    s.scene_max = ArcFloat3{1, 1, 1};

    arc_pcg32 rng;
    arc_pcg32_seed(&rng, seed, 0x5ce9e5ULL);
    if (preset == ARC_SCENE_ROOM_2BOXES) {
        s.num_boxes = 2;
        s.boxes[0] = ArcBox{{0.2f, 0.0f, 0.55f}, {0.5f, 0.3f, 0.85f}, 1};
        s.boxes[1] = ArcBox{{0.55f, 0.0f, 0.2f}, {0.85f, 0.6f, 0.5f}, 1};
    } else if (preset == ARC_SCENE_ROOM_RANDOM || preset == ARC_SCENE_TRAIN_VARIANT) {
        int nb = num_boxes;
        if (preset == ARC_SCENE_TRAIN_VARIANT) {
            nb = (int)(arc_pcg32_next(&rng) % 17u);  // 0..16 boxes
            const float lx = 0.2f + 0.6f * arc_pcg32_float(&rng);
            const float lz = 0.2f + 0.6f * arc_pcg32_float(&rng);
            s.light_center = ArcFloat3{lx, 0.999f, lz};
            const float g = 0.4f + 0.5f * arc_pcg32_float(&rng);  // wall albedo
            s.materials[1] = lambert(g, g, g);
        }
        for (int i = 0; i < nb; ++i) {
            float e[3], lo[3];
            for (int k = 0; k < 3; ++k) e[k] = 0.05f + 0.2f * arc_pcg32_float(&rng);
            for (int k = 0; k < 3; ++k) {
                const float top = (k == 1 ? 0.9f : 1.0f) - e[k];
                lo[k] = top * arc_pcg32_float(&rng);
            }
            const int mat = s.num_materials++;
            const float r = 0.3f + 0.5f * arc_pcg32_float(&rng);
            const float gg = 0.3f + 0.5f * arc_pcg32_float(&rng);
            const float b = 0.3f + 0.5f * arc_pcg32_float(&rng);
            s.materials[mat] = lambert(r, gg, b);
            s.boxes[i] = ArcBox{{lo[0], lo[1], lo[2]}, {lo[0] + e[0], lo[1] + e[1], lo[2] + e[2]}, mat};
        }
        s.num_boxes = nb;
    }
    return ARC_OK;
}

extern "C" arc_status arc_scene_trace_avpls(const ArcSceneDesc* scene, uint64_t seed, int32_t max_bounces,
                                            int32_t explicit_direct_illum, int32_t num_avpls, ArcAvplHost* out,
                                            int64_t* num_paths) {
    if (!scene || !out || num_avpls < 0 || max_bounces < 1) return ARC_ERR_INVALID_ARG;
    const Geometry g = build_geometry(*scene);
    // Paths are independent (one PCG32 stream each), so batches of paths are traced in
    // parallel and appended in path order: the output does not depend on the thread count.
    const int64_t batch = 4096;
    int64_t produced = 0, path0 = 0;
    std::vector<std::vector<ArcAvplHost>> per(batch);
    while (produced < num_avpls) {
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < batch; ++i) {
            per[i].clear();
            trace_path(*scene, g, seed, (uint64_t)(path0 + i), max_bounces, explicit_direct_illum != 0, per[i]);
        }
        for (int64_t i = 0; i < batch && produced < num_avpls; ++i) {
            for (const ArcAvplHost& a : per[i]) {
                if (produced >= num_avpls) break;
                out[produced++] = a;
            }
            if (produced >= num_avpls && num_paths) *num_paths = path0 + i + 1;
        }
        path0 += batch;
        if (path0 > (int64_t)num_avpls * 1000 + 100000) return ARC_ERR_INVALID_ARG;  // light sees nothing
    }
    if (num_avpls == 0 && num_paths) *num_paths = 0;
    return ARC_OK;
}

extern "C" arc_status arc_scene_gbuffer(const ArcSceneDesc* scene, int32_t width, int32_t height, float* position,
                                        float* normal) {
    if (!scene || !position || !normal || width <= 0 || height <= 0) return ARC_ERR_INVALID_ARG;
    const Geometry g = build_geometry(*scene);
    const V3 eye = fromA(scene->camera_position);
    const V3 fwd = normalize(fromA(scene->camera_target) - eye);
    const V3 right = normalize(cross(fwd, v3(0, 1, 0)));
    const V3 up = cross(right, fwd);
    const float tan_half = std::tan(0.5f * scene->camera_fov_deg * kPi / 180.0f);
    const float aspect = (float)width / (float)height;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            const float sx = (2.0f * ((float)x + 0.5f) / (float)width - 1.0f) * aspect * tan_half;
            const float sy = (1.0f - 2.0f * ((float)y + 0.5f) / (float)height) * tan_half;
            const V3 d = normalize(fwd + sx * right + sy * up);
            Hit hit;
            float* P = position + 4 * ((size_t)y * width + x);
            float* N = normal + 4 * ((size_t)y * width + x);
            if (intersect(g, eye, d, hit)) {
                P[0] = hit.p.x; P[1] = hit.p.y; P[2] = hit.p.z; P[3] = 1.0f;
                N[0] = hit.n.x; N[1] = hit.n.y; N[2] = hit.n.z; N[3] = (float)hit.material;
            } else {
                P[0] = P[1] = P[2] = P[3] = 0.0f;
                N[0] = N[1] = N[2] = N[3] = 0.0f;
            }
        }
    }
    return ARC_OK;
}

extern "C" arc_status arc_scene_batch_views(const ArcSceneDesc* scene, uint64_t seed, int32_t count,
                                            ArcBatchViewDesc* out) {
    if (!scene || !out || count < 0) return ARC_ERR_INVALID_ARG;
    static const int32_t kRes[4][2] = {{256, 256}, {512, 512}, {1280, 720}, {1920, 1080}};
    arc_pcg32 rng;
    arc_pcg32_seed(&rng, seed, 0);
    const float lo[3] = {scene->scene_min.x, scene->scene_min.y, scene->scene_min.z};
    const float hi[3] = {scene->scene_max.x, scene->scene_max.y, scene->scene_max.z};
    auto inside_box = [&](const float* p) {
        for (int b = 0; b < scene->num_boxes; ++b) {
            const ArcBox& x = scene->boxes[b];
            if (p[0] > x.lo.x && p[0] < x.hi.x && p[1] > x.lo.y && p[1] < x.hi.y && p[2] > x.lo.z && p[2] < x.hi.z)
                return true;
        }
        return false;
    };
    for (int32_t v = 0; v < count; ++v) {
        ArcBatchViewDesc& d = out[v];
        const int r = (int)(arc_pcg32_next(&rng) % 4u);
        d.width = kRes[r][0];
        d.height = kRes[r][1];
        // log-uniform in [2^13, 2^18]
        d.num_avpls = (int32_t)std::lround(std::exp2(13.0 + 5.0 * (double)arc_pcg32_float(&rng)));
        d.avpl_seed = ((uint64_t)arc_pcg32_next(&rng) << 32) | arc_pcg32_next(&rng);
        float c[3], t[3];
        for (int tries = 0; tries < 1000; ++tries) {  // a camera outside every box, 10% in from the walls
            for (int k = 0; k < 3; ++k) c[k] = lo[k] + (hi[k] - lo[k]) * (0.1f + 0.8f * arc_pcg32_float(&rng));
            if (!inside_box(c)) break;
        }
        for (int tries = 0; tries < 1000; ++tries) {  // a target at least 0.3 away
            for (int k = 0; k < 3; ++k) t[k] = lo[k] + (hi[k] - lo[k]) * arc_pcg32_float(&rng);
            const float dx = t[0] - c[0], dy = t[1] - c[1], dz = t[2] - c[2];
            if (dx * dx + dy * dy + dz * dz >= 0.09f) break;
        }
        d.camera_position = ArcFloat3{c[0], c[1], c[2]};
        d.camera_target = ArcFloat3{t[0], t[1], t[2]};
    }
    return ARC_OK;
}
