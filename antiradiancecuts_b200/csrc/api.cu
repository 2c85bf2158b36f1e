// C ABI of libarc: contexts, device arena, AVPL / material uploads (AvplsGpu / MaterialsGpu,
// data_gpu.cu:5-86), the gather entry points and CudaGather::run (cudaGather.cu:836-1051).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "arc_internal.h"

namespace arc {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

Arena::~Arena() {
    for (auto& kv : bufs_)
        if (kv.second.ptr) cudaFree(kv.second.ptr);
}

arc_status Arena::get(const char* name, size_t bytes, void** out) {
    Buf& b = bufs_[name];
    if (b.bytes < bytes) {
        if (b.ptr) {
            ARC_TRY_CUDA(cudaFree(b.ptr));
            b.ptr = nullptr;
            b.bytes = 0;
        }
        const size_t want = bytes + bytes / 8 + 256;  // headroom so small growth does not reallocate
        ARC_TRY_CUDA(cudaMalloc(&b.ptr, want));
        b.bytes = want;
    }
    *out = b.ptr;
    return ARC_OK;
}

void stage_begin(arc_context* ctx, const char* name) {
    StageTimer& t = ctx->timer;
    if (!t.enabled) return;
    if (t.used == t.begin.size()) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess) return;
        if (cudaEventCreate(&b) != cudaSuccess) {
            cudaEventDestroy(a);
            return;
        }
        t.begin.push_back(a);
        t.end.push_back(b);
        t.names.emplace_back();
    }
    t.names[t.used] = name;
    cudaEventRecord(t.begin[t.used], ctx->stream);
    t.open.push_back(t.used);
    ++t.used;
}

void stage_end(arc_context* ctx, int kernels_launched) {
    ctx->launches += (uint64_t)kernels_launched;
    StageTimer& t = ctx->timer;
    if (!t.enabled || t.open.empty()) return;
    cudaEventRecord(t.end[t.open.back()], ctx->stream);
    t.open.pop_back();
}

size_t Arena::bytes_held() const {
    size_t s = 0;
    for (const auto& kv : bufs_) s += kv.second.bytes;
    return s;
}

}  // namespace arc

using namespace arc;

namespace {

arc_status check_device_errors(arc_context* ctx) {
    uint32_t word = 0;
    ARC_TRY_CUDA(cudaMemcpyAsync(&word, ctx->d_error, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    if (word) {
        ARC_TRY_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(uint32_t), ctx->stream));
        char buf[128];
        snprintf(buf, sizeof(buf), "device error word 0x%x", word);
        set_last_error(buf);
        if (word & ARC_DEVERR_TIMEOUT) return ARC_ERR_TIMEOUT;
        if (word & ARC_DEVERR_STACK_OVERFLOW) return ARC_ERR_STACK_OVERFLOW;
        return ARC_ERR_DEVICE;
    }
    return ARC_OK;
}

float3 to_f3(ArcFloat3 a) { return make_float3(a.x, a.y, a.z); }

}  // namespace

extern "C" {

int32_t arc_api_version(void) { return ARC_API_VERSION; }

const char* arc_status_string(int32_t s) {
    switch (s) {
        case ARC_OK: return "ARC_OK";
        case ARC_ERR_INVALID_ARG: return "ARC_ERR_INVALID_ARG";
        case ARC_ERR_TOO_FEW_AVPLS: return "ARC_ERR_TOO_FEW_AVPLS";
        case ARC_ERR_STACK_OVERFLOW: return "ARC_ERR_STACK_OVERFLOW";
        case ARC_ERR_TIMEOUT: return "ARC_ERR_TIMEOUT";
        case ARC_ERR_CUDA: return "ARC_ERR_CUDA";
        case ARC_ERR_OUT_OF_MEMORY: return "ARC_ERR_OUT_OF_MEMORY";
        case ARC_ERR_DEVICE: return "ARC_ERR_DEVICE";
        case ARC_ERR_UNSUPPORTED: return "ARC_ERR_UNSUPPORTED";
        case ARC_ERR_IO: return "ARC_ERR_IO";
        default: return "ARC_ERR_UNKNOWN";
    }
}

const char* arc_last_error(void) { return g_last_error.c_str(); }

void arc_gather_params_default(ArcGatherParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->ar_kind = ARC_AR_CONE;
    p->cone_half_angle = 30.0f * 3.14159265358979f / 180.0f;
    p->precision = ARC_PREC_KAHAN;
    p->tile_config = -1;
}

void arc_lbvh_params_default(ArcLbvhParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->bbox_mode = ARC_BBOX_SCENE;
    p->scene_min = ArcFloat3{0.0f, 0.0f, 0.0f};
    p->scene_max = ArcFloat3{1.0f, 1.0f, 1.0f};
    p->repr_seed = 5489u;  // mt19937's default seed, the reference's representative RNG seed
}

void arc_cut_params_default(ArcCutParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->kind = ARC_CUT_ERROR_BOUND;
    p->solid_angle_threshold = 3.14159265f / 10.0f;  // ClusterRefinementThreshold (CConfigManager.cpp:37)
    p->error_bound = 0.01f;
    p->ar_uncertain_factor = 16.0f;
    p->max_cut_nodes = 1 << 20;
    p->cut_pool_entries = 0;
    p->mlp_threshold = 0.5f;
    p->mlp_band = 4096.0f;
    p->debug_pixel_x = -1;
    p->debug_pixel_y = -1;
}

void arc_run_config_default(ArcRunConfig* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->useLightCuts = 1;  // CConfigManager.cpp defaults
    c->cut_kind = ARC_CUT_SOLID_ANGLE;
    c->clusterRefinementThreshold = 3.14159265f / 10.0f;
    c->error_bound = 0.01f;
    c->photonRadiusScale = 2.0f;
    c->ar_kind = ARC_AR_DISK;
    c->cone_half_angle = 30.0f * 3.14159265358979f / 180.0f;
    c->precision = ARC_PREC_KAHAN;
    ArcCutParams cp;
    arc_cut_params_default(&cp);
    c->ar_uncertain_factor = cp.ar_uncertain_factor;
    c->mlp_threshold = cp.mlp_threshold;
    c->mlp_band = cp.mlp_band;
    c->cut_pool_entries = cp.cut_pool_entries;
    c->useClusteredDeferred = 0;
    c->cluster_z_near = 0.1f;
    c->cluster_theta = 20.0f * 3.14159265358979f / 180.0f;  // half of a 40 degree field of view
}

arc_status arc_context_create(int32_t device, void* cuda_stream, arc_context** out) {
    ARC_CHECK_ARG(out != nullptr, "out is NULL");
    *out = nullptr;
    int count = 0;
    ARC_TRY_CUDA(cudaGetDeviceCount(&count));
    ARC_CHECK_ARG(device >= 0 && device < count, "no such CUDA device");
    ARC_TRY_CUDA(cudaSetDevice(device));
    arc_context* ctx = new arc_context();
    ctx->device = device;
    cudaError_t e = cudaSuccess;
    if (cuda_stream) {
        ctx->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        ctx->owns_stream = true;
    }
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_error, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(ctx->d_error, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_materials, sizeof(MaterialRecord) * ARC_MAX_MATERIALS);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_learned_rows, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(ctx->d_learned_rows, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        set_last_error(std::string("context creation: ") + cudaGetErrorString(e));
        arc_context_destroy(ctx);
        return ARC_ERR_CUDA;
    }
    *out = ctx;
    return ARC_OK;
}

arc_status arc_context_destroy(arc_context* ctx) {
    if (!ctx) return ARC_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->run_bvh) arc_lbvh_destroy(ctx->run_bvh);
    for (auto e : ctx->timer.begin) cudaEventDestroy(e);
    for (auto e : ctx->timer.end) cudaEventDestroy(e);
    if (ctx->d_error) cudaFree(ctx->d_error);
    if (ctx->d_materials) cudaFree(ctx->d_materials);
    if (ctx->d_learned_rows) cudaFree(ctx->d_learned_rows);
    for (int i = 0; i < 2; ++i) {
        if (ctx->h_staging[i]) cudaFreeHost(ctx->h_staging[i]);
        if (ctx->staged[i]) cudaEventDestroy(ctx->staged[i]);
    }
    if (ctx->owns_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ARC_OK;
}

arc_status arc_context_synchronize(arc_context* ctx, uint32_t* device_error_word) {
    ARC_CHECK_ARG(ctx != nullptr, "ctx is NULL");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    uint32_t word = 0;
    ARC_TRY_CUDA(cudaMemcpyAsync(&word, ctx->d_error, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    if (word) ARC_TRY_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(uint32_t), ctx->stream));
    if (device_error_word) *device_error_word = word;
    return ARC_OK;
}

void* arc_context_stream(arc_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

arc_status arc_context_profile(arc_context* ctx, int32_t enable) {
    ARC_CHECK_ARG(ctx != nullptr, "ctx is NULL");
    ctx->timer.enabled = enable != 0;
    ctx->timer.used = 0;
    ctx->timer.open.clear();
    return ARC_OK;
}

arc_status arc_context_stage_times(arc_context* ctx, char* names, size_t names_len, float* ms, int32_t max_stages,
                                   int32_t* num_stages) {
    ARC_CHECK_ARG(ctx && names && ms && num_stages && names_len > 0, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    StageTimer& t = ctx->timer;
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    std::string joined;
    int32_t n = 0;
    for (size_t i = 0; i < t.used && n < max_stages; ++i, ++n) {
        float v = 0.0f;
        ARC_TRY_CUDA(cudaEventElapsedTime(&v, t.begin[i], t.end[i]));
        ms[n] = v;
        if (i) joined += ",";
        joined += t.names[i];
    }
    std::snprintf(names, names_len, "%s", joined.c_str());
    *num_stages = n;
    t.used = 0;
    t.open.clear();
    return ARC_OK;
}

uint64_t arc_context_launch_count(arc_context* ctx) { return ctx ? ctx->launches : 0; }

uint64_t arc_context_learned_rows(arc_context* ctx) {
    if (!ctx || !ctx->d_learned_rows) return 0;
    unsigned long long rows = 0;
    if (cudaSetDevice(ctx->device) != cudaSuccess ||
        cudaMemcpyAsync(&rows, ctx->d_learned_rows, sizeof(rows), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return 0;
    return rows;
}

arc_status arc_device_alloc(arc_context* ctx, size_t bytes, void** out) {
    ARC_CHECK_ARG(ctx && out, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    ARC_TRY_CUDA(cudaMalloc(out, bytes > 0 ? bytes : 1));
    return ARC_OK;
}

arc_status arc_device_free(arc_context* ctx, void* ptr) {
    ARC_CHECK_ARG(ctx != nullptr, "ctx is NULL");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    if (ptr) ARC_TRY_CUDA(cudaFree(ptr));
    return ARC_OK;
}

arc_status arc_copy_h2d(arc_context* ctx, void* dst, const void* src, size_t bytes) {
    ARC_CHECK_ARG(ctx && dst && src, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    ARC_TRY_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return ARC_OK;
}

arc_status arc_copy_d2h(arc_context* ctx, void* dst, const void* src, size_t bytes) {
    ARC_CHECK_ARG(ctx && dst && src, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    ARC_TRY_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return ARC_OK;
}

arc_status arc_materials_upload(arc_context* ctx, const ArcMaterial* materials, int32_t num) {
    ARC_CHECK_ARG(ctx && materials, "NULL argument");
    ARC_CHECK_ARG(num > 0 && num <= ARC_MAX_MATERIALS, "material count must be in [1, ARC_MAX_MATERIALS]");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    MaterialRecord recs[ARC_MAX_MATERIALS];
    std::memset(recs, 0, sizeof(recs));
    bool spec = false;
    for (int i = 0; i < num; ++i) {
        const ArcMaterial& m = materials[i];
        const float sl = std::sqrt(m.specular.x * m.specular.x + m.specular.y * m.specular.y +
                                   m.specular.z * m.specular.z);
        recs[i].diffuse_exp = make_float4(m.diffuse.x, m.diffuse.y, m.diffuse.z, m.exponent);
        recs[i].specular_flag = make_float4(m.specular.x, m.specular.y, m.specular.z, sl > 0.0f ? 1.0f : 0.0f);
        spec = spec || sl > 0.0f;
    }
    ARC_TRY_CUDA(cudaMemcpyAsync(ctx->d_materials, recs, sizeof(MaterialRecord) * num, cudaMemcpyHostToDevice,
                                 ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->num_materials = num;
    ctx->any_specular = spec;
    ctx->host_materials.assign(materials, materials + num);
    return ARC_OK;
}

arc_status arc_avpls_upload(arc_context* ctx, const ArcAvplHost* avpls, int32_t num, ArcAvplsGpuParam* out) {
    ARC_CHECK_ARG(ctx && out && (avpls || num == 0), "NULL argument");
    ARC_CHECK_ARG(num >= 0, "negative AVPL count");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    // AoS -> SoA on the host (all cores) into pinned staging, one copy, then device views
    // (data_gpu.cu:5-52).  The staging buffers alternate: this one was last read by the copy two
    // uploads ago, which is all the host waits for.
    const size_t n = (size_t)num;
    const size_t bytes = n * (5 * sizeof(ArcFloat3) + 2 * sizeof(int32_t));
    const int turn = ctx->staging_turn;
    ctx->staging_turn ^= 1;
    if (!ctx->staged[turn]) ARC_TRY_CUDA(cudaEventCreateWithFlags(&ctx->staged[turn], cudaEventDisableTiming));
    ARC_TRY_CUDA(cudaEventSynchronize(ctx->staged[turn]));
    if (ctx->h_staging_bytes[turn] < bytes) {
        if (ctx->h_staging[turn]) {
            ARC_TRY_CUDA(cudaFreeHost(ctx->h_staging[turn]));
            ctx->h_staging[turn] = nullptr;
            ctx->h_staging_bytes[turn] = 0;
        }
        ARC_TRY_CUDA(cudaMallocHost(&ctx->h_staging[turn], bytes > 0 ? bytes : 64));
        ctx->h_staging_bytes[turn] = bytes;
    }
    char* h = reinterpret_cast<char*>(ctx->h_staging[turn]);
    ArcFloat3* hp = reinterpret_cast<ArcFloat3*>(h);
    ArcFloat3* hn = hp + n;
    ArcFloat3* hw = hn + n;
    ArcFloat3* hL = hw + n;
    ArcFloat3* hA = hL + n;
    int32_t* hm = reinterpret_cast<int32_t*>(hA + n);
    int32_t* hb = hm + n;
#pragma omp parallel for schedule(static) if (n >= 65536)
    for (size_t i = 0; i < n; ++i) {
        hp[i] = avpls[i].position;
        hn[i] = avpls[i].normal;
        hw[i] = avpls[i].incDirection;
        hL[i] = avpls[i].incRadiance;
        hA[i] = avpls[i].antiradiance;
        hm[i] = avpls[i].materialIndex;
        hb[i] = avpls[i].bounce;
    }
    void* d = nullptr;
    ARC_TRY(ctx->arena.get("avpls_soa", bytes > 0 ? bytes : 64, &d));
    if (bytes) ARC_TRY_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ARC_TRY_CUDA(cudaEventRecord(ctx->staged[turn], ctx->stream));
    char* dc = reinterpret_cast<char*>(d);
    out->position = reinterpret_cast<ArcFloat3*>(dc);
    out->normal = out->position + n;
    out->incDirection = out->normal + n;
    out->incRadiance = out->incDirection + n;
    out->antiradiance = out->incRadiance + n;
    out->materialIndex = reinterpret_cast<int32_t*>(out->antiradiance + n);
    out->bounce = out->materialIndex + n;
    out->numAvpls = num;
    return ARC_OK;
}

arc_status arc_gather_bruteforce(arc_context* ctx, const ArcAvplsGpuParam* avpls, const ArcGBufferView* gbuffer,
                                 ArcFloat3 camera_position, const ArcGatherParams* params, const ArcOutputView* out) {
    ARC_CHECK_ARG(ctx && avpls && gbuffer && params && out, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    GatherLaunch g{avpls, gbuffer, to_f3(camera_position), params, out};
    return launch_gather_bruteforce(ctx, g);
}

arc_status arc_lbvh_create(arc_context* ctx, arc_lbvh** out) {
    ARC_CHECK_ARG(ctx && out, "NULL argument");
    arc_lbvh* b = new arc_lbvh();
    b->ctx = ctx;
    *out = b;
    return ARC_OK;
}

arc_status arc_lbvh_destroy(arc_lbvh* bvh) {
    if (!bvh) return ARC_OK;
    cudaSetDevice(bvh->ctx->device);
    cudaStreamSynchronize(bvh->ctx->stream);
    delete bvh;
    return ARC_OK;
}

arc_status arc_lbvh_build(arc_lbvh* bvh, const ArcAvplsGpuParam* avpls, const ArcLbvhParams* params) {
    ARC_CHECK_ARG(bvh && avpls && params, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(bvh->ctx->device));
    return launch_lbvh_build(bvh, avpls, params);
}

arc_status arc_lbvh_get_view(const arc_lbvh* bvh, ArcLbvhView* out) {
    ARC_CHECK_ARG(bvh && out, "NULL argument");
    ARC_CHECK_ARG(bvh->n >= 2, "LBVH not built");
    *out = bvh->view;
    return ARC_OK;
}

arc_status arc_lbvh_reference_views(arc_lbvh* bvh, ArcBvhParam* bvh_param, ArcAvplBvhNodeDataParam* node_data) {
    ARC_CHECK_ARG(bvh && bvh_param && node_data, "NULL argument");
    ARC_CHECK_ARG(bvh->n >= 2, "LBVH not built");
    ARC_TRY_CUDA(cudaSetDevice(bvh->ctx->device));
    if (!bvh->has_reference_nodes) ARC_TRY(launch_lbvh_reference_nodes(bvh));
    *bvh_param = bvh->ref_param;
    *node_data = bvh->ref_data;
    return ARC_OK;
}

arc_status arc_gather_cut(arc_context* ctx, const arc_lbvh* bvh, const ArcAvplsGpuParam* avpls,
                          const ArcGBufferView* gbuffer, ArcFloat3 camera_position, const ArcGatherParams* params,
                          const ArcCutParams* cut, const ArcOutputView* out) {
    ARC_CHECK_ARG(ctx && bvh && gbuffer && params && cut && out, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    return launch_gather_cut(ctx, bvh, avpls, gbuffer, to_f3(camera_position), params, cut, out);
}

arc_status arc_last_cut(arc_context* ctx, ArcCutLists* out) {
    ARC_CHECK_ARG(ctx && out, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    const CutPool& p = ctx->last_cut.pool;
    int32_t used = 0;
    if (p.next) {
        ARC_TRY_CUDA(cudaMemcpyAsync(&used, p.next, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    out->num_tiles = ctx->last_cut.num_tiles;
    out->chunk_size = 1024;
    out->max_chunks = p.max_chunks;
    out->pool_chunks_used = used < p.num_chunks ? used : p.num_chunks;
    out->counts = p.counts;
    out->tables = p.tables;
    out->pool = p.entries;
    return ARC_OK;
}

arc_status arc_run(arc_context* ctx, const ArcAvplHost* avpls, int32_t num, ArcFloat3 camera_position,
                   float scene_extent, const ArcRunConfig* config, const ArcGBufferView* gbuffer,
                   const ArcOutputView* out) {
    ARC_CHECK_ARG(ctx && config && gbuffer && out, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    ScopedEvents<4> ev;
    const bool prof = config->profile != 0;
    if (prof) ARC_TRY_CUDA(ev.create());
    if (prof) ARC_TRY_CUDA(cudaEventRecord(ev[0], ctx->stream));
    ArcAvplsGpuParam d;
    ARC_TRY(arc_avpls_upload(ctx, avpls, num, &d));
    if (prof) ARC_TRY_CUDA(cudaEventRecord(ev[1], ctx->stream));

    ArcGatherParams gp;
    arc_gather_params_default(&gp);
    gp.ar_kind = config->ar_kind;
    gp.disk_radius = config->photonRadiusScale * scene_extent / 100.0f;  // cudaGather.cu:949
    gp.cone_half_angle = config->cone_half_angle;
    gp.dist_clamp = config->dist_clamp;
    gp.precision = config->precision;
    // clustered deferred antiradiance: the radiance pass gathers no antiradiance, the clustered
    // pass adds it
    const bool clustered = config->useClusteredDeferred != 0 && config->ar_kind == ARC_AR_DISK;
    if (clustered) gp.ar_kind = ARC_AR_NONE;

    arc_status s = ARC_OK;
    if (config->useLightCuts) {
        // the tree is rebuilt every frame, as AvplBvh is in run() (cudaGather.cu:856-859); its
        // buffers live in the context and are reused
        if (!ctx->run_bvh) ARC_TRY(arc_lbvh_create(ctx, &ctx->run_bvh));
        arc_lbvh* tl_bvh = ctx->run_bvh;
        ArcLbvhParams lp;
        arc_lbvh_params_default(&lp);
        lp.consider_normals = config->considerNormals;
        s = arc_lbvh_build(tl_bvh, &d, &lp);
        if (s != ARC_OK) return s;
        if (prof) ARC_TRY_CUDA(cudaEventRecord(ev[2], ctx->stream));
        ArcCutParams cp;
        arc_cut_params_default(&cp);
        cp.kind = config->cut_kind;
        cp.solid_angle_threshold = config->clusterRefinementThreshold;
        cp.error_bound = config->error_bound;
        cp.model = config->model;
        cp.ar_uncertain_factor = config->ar_uncertain_factor;
        cp.mlp_threshold = config->mlp_threshold;
        cp.mlp_band = config->mlp_band;
        cp.cut_pool_entries = config->cut_pool_entries;
        s = arc_gather_cut(ctx, tl_bvh, &d, gbuffer, camera_position, &gp, &cp, out);
    } else {
        if (prof) ARC_TRY_CUDA(cudaEventRecord(ev[2], ctx->stream));
        s = arc_gather_bruteforce(ctx, &d, gbuffer, camera_position, &gp, out);
    }
    if (s != ARC_OK) return s;
    if (clustered) {
        ArcGatherParams ga = gp;
        ga.ar_kind = ARC_AR_DISK;
        ArcClusterParams cl{config->cluster_z_near, config->cluster_theta};
        s = launch_run_clustered_antiradiance(ctx, &d, gbuffer, camera_position, &cl, &ga, out);
        if (s != ARC_OK) return s;
    }
    if (prof) {
        ARC_TRY_CUDA(cudaEventRecord(ev[3], ctx->stream));
        ARC_TRY_CUDA(cudaEventSynchronize(ev[3]));
        float t01, t12, t23;
        cudaEventElapsedTime(&t01, ev[0], ev[1]);
        cudaEventElapsedTime(&t12, ev[1], ev[2]);
        cudaEventElapsedTime(&t23, ev[2], ev[3]);
        printf("transfer avpl data to gpu took: %.3fms\n", t01);
        if (config->useLightCuts) printf("gather build bvh took: %.3fms\n", t12);
        printf("gather radiance and antiradiance took: %.3fms\n", t23);
    }
    return check_device_errors(ctx);
}

}  // extern "C"
