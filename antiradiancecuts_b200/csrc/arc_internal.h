// Internal host-side declarations of libarc: the context, its grow-only device arena, error
// reporting and the launchers each kernel file provides.
#ifndef ARC_INTERNAL_H_
#define ARC_INTERNAL_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "arc_api.h"

namespace arc {

void set_last_error(const std::string& msg);

#define ARC_TRY_CUDA(expr)                                                                    \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) {                                                              \
            ::arc::set_last_error(std::string(#expr) + ": " + cudaGetErrorString(_e));         \
            return _e == cudaErrorMemoryAllocation ? ARC_ERR_OUT_OF_MEMORY : ARC_ERR_CUDA;    \
        }                                                                                     \
    } while (0)

#define ARC_CHECK_ARG(cond, msg)                    \
    do {                                            \
        if (!(cond)) {                              \
            ::arc::set_last_error(msg);             \
            return ARC_ERR_INVALID_ARG;             \
        }                                           \
    } while (0)

#define ARC_TRY(expr)                      \
    do {                                   \
        arc_status _s = (expr);            \
        if (_s != ARC_OK) return _s;       \
    } while (0)

// N CUDA events that a host function creates (create()) and that are destroyed on every return.
template <int N>
struct ScopedEvents {
    cudaEvent_t e[N] = {};
    cudaError_t create() {
        for (cudaEvent_t& x : e) {
            const cudaError_t r = cudaEventCreate(&x);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    }
    ~ScopedEvents() {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
    cudaEvent_t operator[](int i) const { return e[i]; }
};

// Per-material data the kernels read: {diffuse.xyz, exponent}, {specular.xyz, has_specular}.
struct MaterialRecord {
    float4 diffuse_exp;
    float4 specular_flag;
};

// Grow-only named device buffers.  A buffer is reallocated only when a call needs more bytes
// than it holds, so steady-state frames allocate nothing.
class Arena {
  public:
    ~Arena();
    arc_status get(const char* name, size_t bytes, void** out);
    size_t bytes_held() const;

  private:
    struct Buf {
        void* ptr = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> bufs_;
};

// Optional per-stage CUDA-event timing (the reference's CudaTimer around each stage of run(),
// cudaGather.cu:845-1049) and a count of the library's kernel launches.
struct StageTimer {
    bool enabled = false;
    std::vector<std::string> names;
    std::vector<cudaEvent_t> begin, end;
    size_t used = 0;
    std::vector<size_t> open;  // stages begun and not yet ended (stages may nest)
};

// Per-tile cut lists: each tile's nodes live in 1024-entry chunks of one device pool, listed in
// the tile's row of `tables` (max_chunks per tile); `next` is the pool's allocation counter.
struct CutPool {
    int32_t* entries = nullptr;
    int32_t* tables = nullptr;
    int32_t* counts = nullptr;
    int32_t* next = nullptr;
    int32_t num_chunks = 0;
    int32_t max_chunks = 0;
};

struct CutState {
    int32_t num_tiles = 0;
    CutPool pool;
};

}  // namespace arc

struct arc_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    arc::Arena arena;
    uint32_t* d_error = nullptr;  // device error word (ARC_DEVERR_*)
    // materials
    arc::MaterialRecord* d_materials = nullptr;
    int32_t num_materials = 0;
    bool any_specular = false;
    std::vector<ArcMaterial> host_materials;
    // AVPL upload buffers (AvplsGpu): two pinned staging buffers used in turn, so that the host
    // conversion of one upload overlaps the device work queued before it; staged[i] is recorded
    // after the copy out of buffer i
    void* h_staging[2] = {nullptr, nullptr};
    size_t h_staging_bytes[2] = {0, 0};
    cudaEvent_t staged[2] = {nullptr, nullptr};
    int staging_turn = 0;
    arc::CutState last_cut;
    int sm_count = 148;
    arc_lbvh* run_bvh = nullptr;  // tree rebuilt by arc_run every frame
    arc::StageTimer timer;
    uint64_t launches = 0;  // kernels launched by this context
    unsigned long long* d_learned_rows = nullptr;  // rows scored by the cut network so far (device counter)
    int32_t bf_tile_config = -1;  // brute-force launch shape for tile_config = -1 (arc_autotune_bruteforce)
};

struct arc_lbvh {
    arc_context* ctx = nullptr;
    arc::Arena arena;
    int32_t n = 0;
    ArcLbvhView view{};
    bool has_reference_nodes = false;
    ArcBvhParam ref_param{};
    ArcAvplBvhNodeDataParam ref_data{};
    ArcFloat3* sorted_positions = nullptr;
    ArcFloat3* sorted_normals = nullptr;
};

namespace arc {

// Stage timing and launch counting around a group of kernel launches on ctx->stream.
void stage_begin(arc_context* ctx, const char* name);
void stage_end(arc_context* ctx, int kernels_launched);

struct GatherLaunch {
    const ArcAvplsGpuParam* avpls;
    const ArcGBufferView* gbuffer;
    float3 cam;
    const ArcGatherParams* params;
    const ArcOutputView* out;
};

arc_status launch_gather_bruteforce(arc_context* ctx, const GatherLaunch& g);
// 64-byte brute-force records of the AVPLs (p, n, w, L', A, 1/|w|) in the context's "bf_records"
// buffer (valid until the next gather on this context)
arc_status launch_pack_records(arc_context* ctx, const ArcAvplsGpuParam* avpls, const float4** records);
// arc_run's clustered deferred antiradiance: `out` holds the radiance-only result; writes the
// clustered disk antiradiance into out->antiradiance and result = radiance - antiradiance
arc_status launch_run_clustered_antiradiance(arc_context* ctx, const ArcAvplsGpuParam* avpls,
                                             const ArcGBufferView* gbuffer, ArcFloat3 camera_position,
                                             const ArcClusterParams* cl, const ArcGatherParams* gp,
                                             const ArcOutputView* out);
arc_status launch_lbvh_build(arc_lbvh* bvh, const ArcAvplsGpuParam* avpls, const ArcLbvhParams* p);
arc_status launch_lbvh_reference_nodes(arc_lbvh* bvh);
arc_status launch_gather_cut(arc_context* ctx, const arc_lbvh* bvh, const ArcAvplsGpuParam* avpls,
                             const ArcGBufferView* gb, float3 cam, const ArcGatherParams* gp, const ArcCutParams* cp,
                             const ArcOutputView* out);
arc_status launch_antiradiance_only(arc_context* ctx, const GatherLaunch& g, double* ar64);
// per-tile set-up of the tile cuts (bounds, normal cone, albedo, coarse estimate, threshold) and
// the per-node parts of the cut bound (NodeExtra, two float4 per inner node)
arc_status launch_tile_setup(arc_context* ctx, const arc_lbvh* bvh, const ArcGBufferView* gb, const ArcGatherParams* gp,
                             const ArcCutParams* cp, float4** info_out, float4** extra_out);

}  // namespace arc

#endif  // ARC_INTERNAL_H_
