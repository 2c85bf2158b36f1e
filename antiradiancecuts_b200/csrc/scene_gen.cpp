// Synthetic scenes for the gather: an open-front box room with axis-aligned boxes, a square
// area light, a pinhole camera, a light tracer that emits AVPLs with the semantics of
// AvplShooter::createPath (AvplShooter.h:77-142), and a primary-ray G-buffer that stands in for
// the reference's rasterised CreateGBuffer pass (Render.cpp:740-750).  The CPU versions here make
// the inputs of tests and benchmarks; scene_gpu.cu runs the same math (scene_math.h) on the GPU.
#include "arc_api.h"
#include "pcg32.h"
#include "scene_math.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace arc {
void set_last_error(const std::string& msg);  // api.cu: the thread's arc_last_error() message
}

using namespace arc::scene;

namespace {

arc_status invalid(const char* msg) {
    arc::set_last_error(msg);
    return ARC_ERR_INVALID_ARG;
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
    if (!out) return invalid("arc_scene_preset_desc: out is NULL");
    if (preset < 0 || preset > ARC_SCENE_TRAIN_VARIANT) return invalid("arc_scene_preset_desc: unknown preset");
    if (num_boxes < 0 || num_boxes > ARC_SCENE_MAX_BOXES - 2)
        return invalid("arc_scene_preset_desc: num_boxes must be in [0, ARC_SCENE_MAX_BOXES - 2]");
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
    if (!scene || !out) return invalid("arc_scene_trace_avpls: NULL argument");
    if (num_avpls < 0 || max_bounces < 1) return invalid("arc_scene_trace_avpls: num_avpls < 0 or max_bounces < 1");
    Rect rects[kMaxRects];
    const int nrects = build_rects(*scene, rects);
    // Paths are independent (one PCG32 stream each), so batches of paths are traced in
    // parallel and appended in path order: the output does not depend on the thread count.
    const int64_t batch = 4096;
    int64_t produced = 0, path0 = 0;
    std::vector<std::vector<ArcAvplHost>> per(batch);
    while (produced < num_avpls) {
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < batch; ++i) {
            per[i].clear();
            std::vector<ArcAvplHost>& dst = per[i];
            trace_path(*scene, rects, nrects, seed, (uint64_t)(path0 + i), max_bounces, explicit_direct_illum != 0,
                       [&dst](const ArcAvplHost& a) { dst.push_back(a); });
        }
        for (int64_t i = 0; i < batch && produced < num_avpls; ++i) {
            for (const ArcAvplHost& a : per[i]) {
                if (produced >= num_avpls) break;
                out[produced++] = a;
            }
            if (produced >= num_avpls && num_paths) *num_paths = path0 + i + 1;
        }
        path0 += batch;
        if (path0 > (int64_t)num_avpls * 1000 + 100000)
            return invalid("arc_scene_trace_avpls: the light paths make no indirect AVPLs (light sees nothing)");
    }
    if (num_avpls == 0 && num_paths) *num_paths = 0;
    return ARC_OK;
}

extern "C" arc_status arc_scene_gbuffer(const ArcSceneDesc* scene, int32_t width, int32_t height, float* position,
                                        float* normal) {
    if (!scene || !position || !normal) return invalid("arc_scene_gbuffer: NULL argument");
    if (width <= 0 || height <= 0) return invalid("arc_scene_gbuffer: width and height must be positive");
    Rect rects[kMaxRects];
    const int nrects = build_rects(*scene, rects);
    const Camera cam = make_camera(*scene, width, height);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x)
            gbuffer_texel(cam, rects, nrects, width, height, x, y, position + 4 * ((size_t)y * width + x),
                          normal + 4 * ((size_t)y * width + x));
    return ARC_OK;
}

extern "C" arc_status arc_scene_batch_views(const ArcSceneDesc* scene, uint64_t seed, int32_t count,
                                            ArcBatchViewDesc* out) {
    if (!scene || !out) return invalid("arc_scene_batch_views: NULL argument");
    if (count < 0) return invalid("arc_scene_batch_views: negative count");
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
