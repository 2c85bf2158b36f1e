/*
 * arc_api.h - C ABI of the B200 (sm_100a) AntiradianceCuts gather + LBVH library (libarc.so).
 *
 * Every entry point takes plain pointers and sizes, returns an arc_status, and enqueues its
 * GPU work on the stream owned by the arc_context it is given.  The library never falls back
 * to the CPU: when no CUDA device is usable, a call returns ARC_ERR_CUDA.  The only CPU
 * functions are the synthetic-scene helpers at the end (arc_scene_*), which make inputs.
 *
 * Reference interface each group replaces (paths are inside the reference's Framework/ tree):
 *   - AvplsGpu / AvplsGpuParam         data_gpu.h:14-40, data_gpu.cu:5-52
 *   - MaterialsGpu / MaterialsGpuParam data_gpu.h:42-62, data_gpu.cu:54-86
 *   - CudaGather ctor / run()          cudaGather.h:25-70, cudaGather.cu:805-1051
 *   - kernel_radiance_simple + kernel_antiradiance + kernel_combine
 *                                      cudaGather.cu:269-314, 446-557, 782-803
 *   - kernel_bvh (lightcut)            cudaGather.cu:316-444
 *   - AvplBvh ctor, Bvh::create, getBvhParam/getAvplBvhNodeDataParam
 *                                      bvh.h:53-148, bvh.cu:325-454, 673-808
 *   - BvhNode / BvhParam / AvplBvhNodeDataParam layouts
 *                                      bvh.h:21-51, 104-113
 */
#ifndef ARC_API_H_
#define ARC_API_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ARC_API_VERSION 1
/* The reference caches at most 20 materials in shared memory (cudaGather.cu:18); this
 * library keeps a device table of up to 64 (staged into shared memory by the kernels that read
 * it per pixel) and rejects more with ARC_ERR_INVALID_ARG. */
#define ARC_MAX_MATERIALS 64

typedef enum arc_status {
    ARC_OK = 0,
    ARC_ERR_INVALID_ARG = 1,     /* bad pointer, size, enum or parameter value */
    ARC_ERR_TOO_FEW_AVPLS = 2,   /* LBVH needs >= 2 AVPLs (reference prints and returns, bvh.cu:327-330) */
    ARC_ERR_STACK_OVERFLOW = 3,  /* cut traversal stack overflowed (reference paints magenta, cudaGather.cu:438-442) */
    ARC_ERR_TIMEOUT = 4,         /* a bounded device wait gave up (mbarrier / look-back) */
    ARC_ERR_CUDA = 5,            /* CUDA runtime error (message in arc_last_error) */
    ARC_ERR_OUT_OF_MEMORY = 6,
    ARC_ERR_DEVICE = 7,          /* device-side error word set; see ARC_DEVERR_* */
    ARC_ERR_UNSUPPORTED = 8,
    ARC_ERR_IO = 9               /* a file could not be written */
} arc_status;

/* Bits of the device error word returned by arc_context_synchronize. */
#define ARC_DEVERR_STACK_OVERFLOW 0x1u
#define ARC_DEVERR_TIMEOUT 0x2u
#define ARC_DEVERR_BAD_MATERIAL 0x4u
#define ARC_DEVERR_BAD_NODE 0x8u
#define ARC_DEVERR_CUT_OVERFLOW 0x10u

typedef struct ArcFloat3 {
    float x, y, z;
} ArcFloat3;

/* Host AVPL record.  Mirrors class Avpl (AVPL.h:7-57) without its shadow-map view/projection
 * matrices, which the CUDA path never reads. */
typedef struct ArcAvplHost {
    ArcFloat3 position;
    ArcFloat3 normal;
    ArcFloat3 incRadiance;  /* L */
    ArcFloat3 antiradiance; /* A */
    ArcFloat3 incDirection; /* w; zero for light-source AVPLs */
    int32_t bounce;
    int32_t materialIndex;
} ArcAvplHost;

/* Device structure-of-arrays view of AVPLs.  Same fields and meaning as AvplsGpuParam
 * (data_gpu.h:14-23); float3 arrays have a 12-byte stride. */
typedef struct ArcAvplsGpuParam {
    ArcFloat3* position;
    ArcFloat3* normal;
    ArcFloat3* incDirection;
    ArcFloat3* incRadiance;
    ArcFloat3* antiradiance;
    int32_t* materialIndex;
    int32_t* bounce;
    int32_t numAvpls;
} ArcAvplsGpuParam;

/* MATERIAL (Material.h:6-12).  Index 0 is the "no surface" material (CMaterialBuffer.cpp:5-17). */
typedef struct ArcMaterial {
    ArcFloat3 emissive;
    ArcFloat3 diffuse;
    ArcFloat3 specular;
    float exponent;
} ArcMaterial;

/* G-buffer, replacing the two GL textures read with surf2Dread (cudaGather.cu:285-290).
 * Pitch-linear float4 planes in device memory:
 *   position: (x, y, z, 1)          normal: (nx, ny, nz, float(materialIndex))
 * A pixel whose material index is 0 has no surface and gathers 0. */
typedef struct ArcGBufferView {
    const float* position;
    const float* normal;
    int32_t width;
    int32_t height;
    int64_t pitch; /* row pitch in float4 elements (>= width) */
} ArcGBufferView;

/* Outputs, replacing the three GL render-target attachments (cudaGather.cu:805-826, where
 * attachment 0 is the result).  float4 planes with w = 1, like the reference's surf2Dwrite.
 * radiance / antiradiance / result_fp64 may be NULL.  result_fp64 holds 3 doubles per pixel
 * (the FP64 signed combine before it is rounded to float). */
typedef struct ArcOutputView {
    float* result;
    float* radiance;
    float* antiradiance;
    double* result_fp64;
    int64_t pitch; /* row pitch in pixels, shared by all planes */
} ArcOutputView;

typedef enum arc_ar_kind {
    ARC_AR_NONE = 0,
    ARC_AR_DISK = 1, /* CUDA getAntiradiance (cudaGather.cu:97-144) */
    ARC_AR_CONE = 2  /* GLSL GetAntiradiance (Shaders/Gather.frag:149-188) */
} arc_ar_kind;

typedef enum arc_precision {
    ARC_PREC_KAHAN = 0,        /* FP32 terms, per-chunk FP32 partials folded into Kahan sums, FP64 combine (default) */
    ARC_PREC_KAHAN_STRICT = 1, /* FP32 terms, every term Kahan-added, FP64 combine */
    ARC_PREC_NAIVE = 2,        /* FP32 terms, plain FP32 sums, FP32 combine (the reference's arithmetic) */
    ARC_PREC_FP64 = 3          /* every operation in FP64 */
} arc_precision;

typedef struct ArcGatherParams {
    int32_t ar_kind;              /* arc_ar_kind */
    float disk_radius;            /* DISK: photonRadius = photonRadiusScale * sceneExtent / 100 (cudaGather.cu:949) */
    float cone_half_angle;        /* CONE: radians; the reference's pi / coneFactor (Gather.frag:166) */
    float dist_clamp;             /* geometry-term distance clamp: dist^2 -> max(dist^2, clamp^2); 0 = off */
    float geo_limit_radiance;     /* clamp(G, 0, limit) as GeoTermLimitRadiance (Gather.frag:190-194); 0 = off */
    float geo_limit_antiradiance; /* clamp(G_A, 0, limit) as GeoTermLimitAntiradiance (Gather.frag:182); 0 = off */
    int32_t precision;            /* arc_precision */
    int32_t tile_config;          /* brute-force tile shape index, -1 = autotuned choice */
} ArcGatherParams;

/* Fill *p with the library defaults: cone 30 deg, no clamp, ARC_PREC_KAHAN, tile_config -1. */
void arc_gather_params_default(ArcGatherParams* p);

/* ---------------------------------------------------------------------------------------- */
/* Context, errors, memory                                                                  */
/* ---------------------------------------------------------------------------------------- */

typedef struct arc_context arc_context;

int32_t arc_api_version(void);
const char* arc_status_string(int32_t status);
/* Message of the last failing call on this host thread ("" if none). */
const char* arc_last_error(void);

/* Threading and ownership.  A context owns one stream, one device arena and its device error
 * word; the trees (arc_lbvh), networks (arc_mlp) and batches (arc_batch) created from it share
 * them, so destroy them before the context.  A context and its objects are not thread-safe: use
 * them from one host thread at a time.
 * Distinct contexts share no mutable state and may be used from different threads at once, on
 * the same or different devices.  Every call on a context selects the context's device first.
 * Inputs and outputs (device arrays, G-buffer and output planes) belong to the caller; the
 * library allocates only its own scratch, from the context's grow-only arena.
 *
 * cuda_stream: a cudaStream_t to run on, or NULL to let the context create its own. */
arc_status arc_context_create(int32_t device, void* cuda_stream, arc_context** out);
arc_status arc_context_destroy(arc_context* ctx);
/* Waits for the context's stream; returns and clears the device error word. */
arc_status arc_context_synchronize(arc_context* ctx, uint32_t* device_error_word);
/* The context's stream (cudaStream_t). */
void* arc_context_stream(arc_context* ctx);

/* Per-stage CUDA-event timing, as the reference's CudaTimer around each stage of run()
 * (cudaGather.cu:845-1049).  While enabled, every library stage records an event pair on the
 * context's stream; arc_context_stage_times waits for the stream and returns the recorded
 * stages (comma-separated names, elapsed ms) since the last call, then clears them. */
arc_status arc_context_profile(arc_context* ctx, int32_t enable);
arc_status arc_context_stage_times(arc_context* ctx, char* names, size_t names_len, float* ms, int32_t max_stages,
                                   int32_t* num_stages);
/* Number of kernels this context has launched so far. */
uint64_t arc_context_launch_count(arc_context* ctx);
/* Number of (tile, node) rows the learned cut's network has scored on this context so far. */
uint64_t arc_context_learned_rows(arc_context* ctx);
/* FP32 FMA throughput of the device with scalar FFMA and packed fma.rn.f32x2 chains (TFLOP/s),
 * the roofline denominator of the gather kernels.  No reference counterpart. */
arc_status arc_measure_fp32_peak(arc_context* ctx, double* scalar_tflops, double* packed_tflops);

/* Device memory helpers for hosts without their own CUDA binding. */
arc_status arc_device_alloc(arc_context* ctx, size_t bytes, void** out);
arc_status arc_device_free(arc_context* ctx, void* ptr);
arc_status arc_copy_h2d(arc_context* ctx, void* dst, const void* src, size_t bytes);
arc_status arc_copy_d2h(arc_context* ctx, void* dst, const void* src, size_t bytes);

/* ---------------------------------------------------------------------------------------- */
/* Scene data uploads (MaterialsGpu / AvplsGpu constructors)                                */
/* ---------------------------------------------------------------------------------------- */

/* MaterialsGpu(materials) (data_gpu.cu:54-86).  num <= ARC_MAX_MATERIALS. */
arc_status arc_materials_upload(arc_context* ctx, const ArcMaterial* materials, int32_t num);

/* AvplsGpu(avpls) (data_gpu.cu:5-52): AoS -> SoA, host -> device, into context-owned buffers
 * that stay valid until the next upload on this context.  *out receives the device view. */
arc_status arc_avpls_upload(arc_context* ctx, const ArcAvplHost* avpls, int32_t num, ArcAvplsGpuParam* out);

/* ---------------------------------------------------------------------------------------- */
/* Brute-force gather (kernel_radiance_simple + kernel_antiradiance + kernel_combine)        */
/* ---------------------------------------------------------------------------------------- */

/* Radiance minus antiradiance over every AVPL for every pixel, in one fused kernel. */
arc_status arc_gather_bruteforce(arc_context* ctx, const ArcAvplsGpuParam* avpls, const ArcGBufferView* gbuffer,
                                 ArcFloat3 camera_position, const ArcGatherParams* params,
                                 const ArcOutputView* out);

/* Allocation-free variant of arc_gather_bruteforce, for callers that may not allocate device
 * memory through the library: hosts that pre-allocate a fixed device budget and forbid
 * cudaMalloc/cudaFree after start-up (an allocation can synchronise the device and stall a
 * frame), or plugin hosts that own every device allocation themselves.  No counterpart in the
 * reference.  It needs no arc_context: work is enqueued on `cuda_stream` (NULL = the legacy
 * default stream) of the current device, materials come from the host array, and the caller
 * passes the AVPL arrays, the G-buffer and the outputs.  Its scratch (packed AVPL records, the
 * material table, the device error word) is one fixed file-scope device array that every GPU
 * loading libarc holds until process exit; it is sized for at most 65,536 AVPLs, and larger
 * inputs are rejected with ARC_ERR_INVALID_ARG.  The first call on a device (and the first after
 * a device reset, or in another driver context) looks up that array's device address; make it
 * before any stream capture.  Every device holds its own copy of the array, which keeps the last
 * call's contents: calls whose GPU work overlaps on the same device (different streams) race on
 * that device's copy; calls on different devices do not share it.  The material table is passed
 * to the GPU as a kernel argument, so `materials` may be released when the call returns.
 * If device_error_word is non-NULL the call waits for the stream and returns the error word
 * (ARC_DEVERR_*) of this call. */
arc_status arc_gather_bruteforce_noalloc(void* cuda_stream, const ArcMaterial* materials, int32_t num_materials,
                                         const ArcAvplsGpuParam* avpls, const ArcGBufferView* gbuffer,
                                         ArcFloat3 camera_position, const ArcGatherParams* params,
                                         const ArcOutputView* out, uint32_t* device_error_word);

/* ---------------------------------------------------------------------------------------- */
/* LBVH (AvplBvh)                                                                            */
/* ---------------------------------------------------------------------------------------- */

typedef enum arc_bbox_mode {
    ARC_BBOX_SCENE = 0,         /* normalise positions over the given scene box */
    ARC_BBOX_AVPL_REFERENCE = 1 /* normalise over the AVPL box, max seeded with FLT_MIN as bvh.cu:346-353 */
} arc_bbox_mode;

typedef struct ArcLbvhParams {
    int32_t consider_normals; /* 6D codes truncated to 32 bits (morton.h:94-107 into MC_SIZE uint32, bvh.h:17) */
    int32_t bbox_mode;        /* arc_bbox_mode */
    ArcFloat3 scene_min;
    ArcFloat3 scene_max;
    uint32_t repr_seed; /* seed of the counter-based hash that replaces the host mt19937 of bvh.cu:694-697 */
    /* Polls after which the radix sort's look-back (a bounded wait on another tile's published
     * offsets) gives up.  0 (default): 2^26, after which the wait sets ARC_DEVERR_TIMEOUT and the
     * rest of the build is skipped on the device (the object then holds no valid tree until the
     * next build).  Non-zero: that limit, and arc_lbvh_build waits for the build and returns
     * ARC_ERR_TIMEOUT (the object left unbuilt) if the wait gave up -- a knob for tests of the
     * timeout path. */
    uint32_t wait_limit;
} ArcLbvhParams;

void arc_lbvh_params_default(ArcLbvhParams* p);

/* BvhNode (bvh.h:21-28): 36-byte record; left/right >= 0 are leaves, -(k+1) is inner node k. */
typedef struct ArcBvhNode {
    int32_t left;
    int32_t right;
    ArcFloat3 bbMin;
    ArcFloat3 bbMax;
    int32_t visited;
} ArcBvhNode;

/* BvhParam (bvh.h:44-51). */
typedef struct ArcBvhParam {
    int32_t numLeafs;
    int32_t numNodes;
    ArcBvhNode* nodes;
    ArcFloat3* positions;
    ArcFloat3* normals;
} ArcBvhParam;

/* AvplBvhNodeDataParam (bvh.h:104-113): 2N-1 elements, inner node k at index N+k. */
typedef struct ArcAvplBvhNodeDataParam {
    int32_t* size;
    int32_t* materialIndex;
    float* randomNumbers;
    ArcFloat3* position;
    ArcFloat3* normal;
    ArcFloat3* incRadiance;
    ArcFloat3* incDirection;
} ArcAvplBvhNodeDataParam;

/* Device views of the library's own tree layout (all device pointers, valid until the next
 * build on the same arc_lbvh).  Node index space: leaf i -> i, inner node k -> N + k.
 *   morton[N]          sorted Morton codes
 *   sorted_index[N]    original AVPL index of sorted leaf i
 *   left/right[N-1]    children of inner node k (reference encoding: leaf >= 0, inner -(k+1))
 *   parents[2N-1]      leaves first, then inner nodes; the root's parent is -1 (bvh.cu:192-265)
 *   range[2(N-1)]      first and last sorted leaf under inner node k
 *   bounds[16(N-1)]    per inner node {bbMin.xyz, left}, {bbMax.xyz, right},
 *                      {normal-cone axis.xyz, cos half-angle}, {direction-cone axis.xyz, cos half-angle}
 *                      (left/right stored as int32 bit patterns)
 *   records[16(2N-1)]  per node the packed gather record {p.xyz, n.x}, {n.y, n.z, w.x, w.y},
 *                      {w.z, L'.rgb}, {A.rgb, count}: representative position/normal/direction,
 *                      summed L' (L times the AVPL-side Lambertian BRDF) and summed A
 *   node_data          reference AvplBvhNodeDataParam arrays (raw summed L, representative) */
typedef struct ArcLbvhView {
    int32_t num_leaves;
    int32_t num_nodes;
    const uint32_t* morton;
    const int32_t* sorted_index;
    const int32_t* left;
    const int32_t* right;
    const int32_t* parents;
    const int32_t* range;
    const float* bounds;
    const float* records;
    ArcAvplBvhNodeDataParam node_data;
    /* [2N-1][4] per node {S.xyz, a}: a = sum over its AVPLs of the antiradiance luminance a_i,
       S = sum of a_i * w_i / |w_i|.  An inner node's packed-record direction w is that of an
       antiradiance representative drawn in proportion to a (w only enters the antiradiance
       cone test); |S| / a measures how concentrated its directions are. */
    const float* dirstat;
} ArcLbvhView;

typedef struct arc_lbvh arc_lbvh;

arc_status arc_lbvh_create(arc_context* ctx, arc_lbvh** out);
arc_status arc_lbvh_destroy(arc_lbvh* bvh);
/* AvplBvh(avpls, considerNormals) (bvh.cu:746-774): Morton codes, stable radix sort,
 * Karras radix tree, bottom-up bounds and cluster data.  Every AVPL passed is a leaf (the
 * reference's caller passes only bounce >= 1 AVPLs, Render.cpp:289-298).  num < 2 gives
 * ARC_ERR_TOO_FEW_AVPLS. */
arc_status arc_lbvh_build(arc_lbvh* bvh, const ArcAvplsGpuParam* avpls, const ArcLbvhParams* params);
arc_status arc_lbvh_get_view(const arc_lbvh* bvh, ArcLbvhView* out);
/* getBvhParam() / getAvplBvhNodeDataParam() (bvh.h:72, 141): writes host structs whose
 * pointers address device arrays in the reference layouts (materialised on first request
 * after each build). */
arc_status arc_lbvh_reference_views(arc_lbvh* bvh, ArcBvhParam* bvh_param, ArcAvplBvhNodeDataParam* node_data);

/* ---------------------------------------------------------------------------------------- */
/* Cut gather (kernel_bvh and its tile-level successors)                                    */
/* ---------------------------------------------------------------------------------------- */

typedef enum arc_cut_kind {
    ARC_CUT_SOLID_ANGLE = 0, /* per-pixel DFS with the solid-angle test of kernel_bvh (cudaGather.cu:316-444) */
    ARC_CUT_ERROR_BOUND = 1, /* per 8x8 tile cut: refine while the node's error bound > eps * tile estimate */
    ARC_CUT_LEARNED = 2      /* per 8x8 tile cut: refine decision from the MLP, error bound as fallback */
} arc_cut_kind;

typedef struct arc_mlp arc_mlp;

typedef struct ArcCutParams {
    int32_t kind;                /* arc_cut_kind */
    float solid_angle_threshold; /* ClusterRefinementThreshold, default pi/10 (CConfigManager.cpp:37) */
    float error_bound;           /* relative error bound, default 0.01 */
    float ar_uncertain_factor;   /* antiradiance bound multiplier for nodes whose cone test may differ
                                    between pairs (default 16); 1 treats them like certain nodes */
    int32_t max_cut_nodes;       /* per-tile cut capacity, default 2^20 (ARC_DEVERR_CUT_OVERFLOW beyond it) */
    int64_t cut_pool_entries;    /* total cut entries over all tiles; 0 = 32768 per tile (the learned cut also keeps
                                  * an 8-byte accepted-pair list of the same capacity) */
    const arc_mlp* model;        /* LEARNED only */
    float mlp_threshold;         /* LEARNED: refine when the predicted probability >= this (BCE model), or
                                    when the predicted relative node error >= this (squared-loss model
                                    regressing log2 of the error) */
    float mlp_band;              /* LEARNED: nodes whose error bound exceeds mlp_band times the tile's error
                                    budget are refined without the network (default 4096; 0 = no limit) */
    int32_t debug_pixel_x;       /* SOLID_ANGLE scene probe (cudaGather.cu:338, 392-396); -1 = off */
    int32_t debug_pixel_y;
    int32_t* used_nodes;         /* optional device array[2N-1]: set to 1 for nodes the probe pixel used */
} ArcCutParams;

void arc_cut_params_default(ArcCutParams* p);

/* avpls: the AVPL arrays the tree was built from; needed only by ARC_CUT_SOLID_ANGLE with an
 * antiradiance mode (its antiradiance is the brute-force pass, as in run()), else may be NULL. */
arc_status arc_gather_cut(arc_context* ctx, const arc_lbvh* bvh, const ArcAvplsGpuParam* avpls,
                          const ArcGBufferView* gbuffer, ArcFloat3 camera_position, const ArcGatherParams* params,
                          const ArcCutParams* cut, const ArcOutputView* out);

/* Per-tile cut lists of the last ERROR_BOUND / LEARNED gather on this context (device pointers).
 * Tile t (row-major 8x8 tiles) holds counts[t] nodes in the node-record index space (leaf i -> i,
 * inner k -> N + k); entry j of tile t is pool[tables[t * max_chunks + j / chunk_size] *
 * chunk_size + j % chunk_size]. */
typedef struct ArcCutLists {
    int32_t num_tiles;
    int32_t chunk_size;
    int32_t max_chunks;
    int32_t pool_chunks_used;
    const int32_t* counts;
    const int32_t* tables;
    const int32_t* pool;
} ArcCutLists;
arc_status arc_last_cut(arc_context* ctx, ArcCutLists* out);

/* ---------------------------------------------------------------------------------------- */
/* Cut-refinement MLP (no counterpart in the reference)                                      */
/* ---------------------------------------------------------------------------------------- */

/* 16 -> 64 -> 64 -> 64 -> 1 multilayer perceptron (GELU or ReLU activations, a property of the
 * model): BF16 weights and activations on the tensor cores (tcgen05), FP32 accumulation, FP32
 * master parameters
 * (layout: W1[64][16], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], w4[64], b4).  Features
 * are BF16 rows of 16 values (16-byte aligned).  What the output means follows the model's loss:
 * ARC_MLP_LOSS_BCE (default): the logit of "refine this node" (labels 0 / 1);
 * ARC_MLP_LOSS_SQUARED: a regression of the label value, for the learned cut log2 of the node's
 * error relative to the tile value. */
typedef enum arc_mlp_loss {
    ARC_MLP_LOSS_BCE = 0,    /* weighted binary cross-entropy on the logit */
    ARC_MLP_LOSS_SQUARED = 1 /* weighted squared error */
} arc_mlp_loss;
int32_t arc_mlp_num_params(void);
arc_status arc_mlp_create(arc_context* ctx, uint64_t seed, arc_mlp** out);
arc_status arc_mlp_destroy(arc_mlp* mlp);
arc_status arc_mlp_set_params(arc_mlp* mlp, const float* host_params, int32_t num);
arc_status arc_mlp_get_params(arc_mlp* mlp, float* host_params, int32_t num);
/* logits[rows] = MLP(features[rows][16]) (device pointers, enqueued on the context's stream). */
arc_status arc_mlp_forward(arc_mlp* mlp, const void* features_bf16, int64_t rows, float* logits);
/* Gradient of the whole batch's weighted loss (sum(w * loss) / weight_sum) into
 * host_grads[num params] and host_loss; waits for the stream.  labels / weights: device arrays
 * (weights may be NULL = 1). */
arc_status arc_mlp_gradients(arc_mlp* mlp, const void* features_bf16, const float* labels, const float* weights,
                             int64_t rows, float weight_sum, float* host_grads, float* host_loss);
/* Loss used by arc_mlp_gradients / arc_mlp_train_step, and the meaning of the output (above). */
arc_status arc_mlp_set_loss(arc_mlp* mlp, int32_t kind);
int32_t arc_mlp_get_loss(const arc_mlp* mlp);
/* Hidden-layer activation of the model (default GELU); applies to forward, gradients, training
 * and the learned cut's selection alike. */
typedef enum arc_mlp_activation {
    ARC_MLP_ACT_GELU = 0, /* x sigma(1.702 x) = x/2 (1 + tanh(0.851 x)) (sigmoid form of GELU) */
    ARC_MLP_ACT_RELU = 1  /* max(x, 0) */
} arc_mlp_activation;
arc_status arc_mlp_set_activation(arc_mlp* mlp, int32_t kind);
int32_t arc_mlp_get_activation(const arc_mlp* mlp);
/* One Adam step (beta 0.9 / 0.999) on the batch's gradient; device_loss_accum (optional, device
 * float) accumulates the batch loss.  Enqueued only. */
arc_status arc_mlp_train_step(arc_mlp* mlp, const void* features_bf16, const float* labels, const float* weights,
                              int64_t rows, float weight_sum, float lr, float* device_loss_accum);

/* Training samples of the learned cut (no counterpart in the reference): walks every 8x8 tile's
 * tree with the exact decision "refine iff the RMS over the tile's pixels of |exact node
 * contribution - node estimate| > delta * mean |exact tile value|" (exact contributions from FP64
 * prefix sums over the sorted leaves) and writes, for each visited node that the learned selection
 * with `cut` would score (its bound above cut->error_bound times the estimate and not above
 * cut->mlp_band times that), its 16 BF16 features, its 0/1 label and its error relative to the
 * tile value.  Device output arrays of `capacity` rows; keys (optional, 2 ints per row) receives
 * each row's (tile, node): the tile index in row-major 8x8 tiles of `gbuffer`, the node in record
 * index space (inner k at num_leaves + k).  Rows come in no particular order across tiles.
 * *count receives the rows written.  Waits for the stream. */
arc_status arc_cut_training_samples(arc_context* ctx, const arc_lbvh* bvh, const ArcGBufferView* gbuffer,
                                    ArcFloat3 camera_position, const ArcGatherParams* params, const ArcCutParams* cut,
                                    float delta, void* features_bf16, float* labels, float* errors, int32_t* keys,
                                    int32_t capacity, int32_t* count);

/* ---------------------------------------------------------------------------------------- */
/* CudaGather::run                                                                           */
/* ---------------------------------------------------------------------------------------- */

/* The CONF_VARS flags that select hot-path variants (CConfigManager.h:6-52). */
typedef struct ArcRunConfig {
    int32_t useLightCuts;             /* 1: LBVH + cut gather for radiance; 0: brute force */
    int32_t cut_kind;                 /* arc_cut_kind used when useLightCuts */
    float clusterRefinementThreshold; /* solid-angle threshold (pi/10) */
    float error_bound;                /* for ERROR_BOUND / LEARNED */
    float photonRadiusScale;          /* DISK radius = scale * sceneExtent / 100 (cudaGather.cu:949) */
    int32_t ar_kind;                  /* arc_ar_kind */
    float cone_half_angle;
    float dist_clamp;
    int32_t precision;
    int32_t considerNormals;
    const arc_mlp* model;
    int32_t profile; /* print per-stage CUDA-event timings, as run(..., profile) */
    /* cut details (ArcCutParams fields of the same names) */
    float ar_uncertain_factor;
    float mlp_threshold;
    float mlp_band;
    int64_t cut_pool_entries;
    /* useClusteredDeferred (cudaGather.cu:948-1031): the disk antiradiance through screen clusters
     * (arc_antiradiance_clustered) instead of brute force; with ar_kind ARC_AR_DISK only */
    int32_t useClusteredDeferred;
    float cluster_z_near; /* ArcClusterParams.z_near */
    float cluster_theta;  /* ArcClusterParams.theta */
} ArcRunConfig;

void arc_run_config_default(ArcRunConfig* c);

/* CudaGather::run(avpls, cameraPosition, sceneProbe, sceneExtent, profile) (cudaGather.cu:836-1051):
 * uploads the AVPLs, gathers radiance (brute force or cut) and antiradiance and writes
 * result = radiance - antiradiance. */
arc_status arc_run(arc_context* ctx, const ArcAvplHost* avpls, int32_t num, ArcFloat3 camera_position,
                   float scene_extent, const ArcRunConfig* config, const ArcGBufferView* gbuffer,
                   const ArcOutputView* out);

/* ---------------------------------------------------------------------------------------- */
/* Batched multi-view rendering and the brute-force tile-shape autotuner (no counterpart in  */
/* the reference, whose CudaGather::run renders one view per call with fixed launch shapes)  */
/* ---------------------------------------------------------------------------------------- */

/* One view of a batch: its own AVPL set (device arrays), G-buffer, camera and output planes. */
typedef struct ArcBatchView {
    ArcAvplsGpuParam avpls;
    ArcGBufferView gbuffer;
    ArcFloat3 camera_position;
    ArcOutputView out;
} ArcBatchView;

typedef struct arc_batch arc_batch;

/* A batch renderer on `ctx`.  It owns four lanes -- sub-contexts on the same device, each with its
 * own stream, scratch arena, LBVH and error word -- that render their share of a batch's views
 * concurrently, so that views of uneven sizes share the GPU.  The lanes copy `ctx`'s material
 * table before each render. */
arc_status arc_batch_create(arc_context* ctx, arc_batch** out);
arc_status arc_batch_destroy(arc_batch* batch);
/* Per view, the LBVH build of its AVPLs (`lbvh`, default wait limit) and the cut gather (`cut`;
 * SOLID_ANGLE, ERROR_BOUND or LEARNED) into its outputs.  The views are dealt to the lanes longest
 * first (estimated work: pixels x log2 AVPLs); the lanes fork from the context's stream and join
 * back into it, folding their device error words into the context's.  Enqueued only. */
arc_status arc_batch_render(arc_batch* batch, const ArcBatchView* views, int32_t num_views, const ArcLbvhParams* lbvh,
                            const ArcGatherParams* gather, const ArcCutParams* cut);
/* Records arc_batch_render of these views into one CUDA graph: it first renders them once eagerly
 * (sizing every library buffer), then captures the same work -- every lane, the fork and the join --
 * from the context's stream.  The views' buffers must stay valid and in place while the graph is
 * used.  ERROR_BOUND and LEARNED cuts.  Replaces any previously recorded graph. */
arc_status arc_batch_capture(arc_batch* batch, const ArcBatchView* views, int32_t num_views,
                             const ArcLbvhParams* lbvh, const ArcGatherParams* gather, const ArcCutParams* cut);
/* Replays the recorded graph on the context's stream: the whole batch in one launch.  Enqueued
 * only; the device error word collects the views' device errors. */
arc_status arc_batch_launch(arc_batch* batch);

/* Times every brute-force launch shape (pixel tile 16 x 16 PX, PX in {1, 2, 4}, AVPL chunk 64 ...
 * 1024, ArcGatherParams.tile_config index) on this workload and makes the fastest the context's
 * default for tile_config = -1.  times_ms[num_shapes] (optional) receives each shape's time
 * (< 0 where it does not apply); *best the chosen index.  Waits for the stream; writes `out`. */
int32_t arc_bruteforce_num_tile_shapes(void);
/* Sets the context's default launch shape for tile_config = -1 (-1: the library's built-in one),
 * e.g. to apply a shape tuned earlier. */
arc_status arc_context_set_tile_config(arc_context* ctx, int32_t tile_config);
arc_status arc_autotune_bruteforce(arc_context* ctx, const ArcAvplsGpuParam* avpls, const ArcGBufferView* gbuffer,
                                   ArcFloat3 camera_position, const ArcGatherParams* params, const ArcOutputView* out,
                                   int32_t* best, float* times_ms, int32_t num_shapes);

/* ---------------------------------------------------------------------------------------- */
/* Clustered deferred antiradiance (the reference's accelerator for the disk antiradiance)   */
/* ---------------------------------------------------------------------------------------- */

/* Screen clusters (VisiblePointsBvh, bvh.cu:986-1179): 16 x 16 pixel tiles split by depth slice
 * k = floor(log(d / z_near) / log(1 + 2 tan(theta) / 16)), d the distance to the camera. */
typedef struct ArcClusterParams {
    float z_near; /* the camera's near plane distance */
    float theta;  /* cameraTheta: half the vertical field of view, radians */
} ArcClusterParams;

/* Device arrays of the last arc_antiradiance_clustered call on the context (valid until the
 * next call): pixel_cluster[height * width] (cluster slot or -1: no surface); box[slot][8]
 * ({min, 0}, {max, 0}); tile_count[tile] (clusters of the tile, in slots tile * slots_per_tile
 * ...); counts[slot] (AVPLs in the cluster's list) and lists (every list in slot order, each in
 * AVPL order: the list of slot s starts at the sum of counts[0 .. s-1]). */
typedef struct ArcClusterInfo {
    const int32_t* pixel_cluster;
    const float* box;
    const int32_t* tile_count;
    const int32_t* counts;
    const int32_t* lists;
    int32_t num_tiles;
    int32_t slots_per_tile;
    int64_t list_entries;
} ArcClusterInfo;

/* Disk antiradiance through screen clusters and their light lists (kernel_gather_cluster_lights +
 * kernel_antiradiance_clusterred, cudaGather.cu:605-748): the AVPLs of a pixel's cluster are
 * those whose ray (position, incDirection) meets the cluster box grown by twice the disk radius,
 * which holds every AVPL whose disk antiradiance reaches the cluster's pixels, so the result is
 * the brute-force disk antiradiance up to summation order.  Writes out->antiradiance (float4,
 * w = 1) and, when set, out->result_fp64 (3 doubles per pixel: the antiradiance in FP64); other
 * planes are untouched.  params: ar_kind ARC_AR_DISK with disk_radius > 0.  info may be NULL. */
arc_status arc_antiradiance_clustered(arc_context* ctx, const ArcAvplsGpuParam* avpls, const ArcGBufferView* gbuffer,
                                      ArcFloat3 camera_position, const ArcClusterParams* cparams,
                                      const ArcGatherParams* params, const ArcOutputView* out, ArcClusterInfo* info);

/* ---------------------------------------------------------------------------------------- */
/* After the gather: accumulation, normalisation, image error, export                        */
/* ---------------------------------------------------------------------------------------- */

/* FP64 running sums of the three output planes over frames (Renderer::Add, Render.cpp:298-301):
 * sum holds 9 doubles per pixel (result, radiance, antiradiance; r, g, b each), row pitch in
 * pixels.  Caller-owned device memory. */
typedef struct ArcAccumView {
    double* sum;
    int32_t width;
    int32_t height;
    int64_t pitch;
} ArcAccumView;

/* acc += the frame's planes (planes that are NULL in `frame` are skipped). */
arc_status arc_accumulate(arc_context* ctx, const ArcOutputView* frame, const ArcAccumView* acc);
/* acc = 0. */
arc_status arc_accum_clear(arc_context* ctx, const ArcAccumView* acc);
/* out = acc / num_paths (Renderer::Normalize, Render.cpp:639-664: 0 when num_paths is 0), rounded
 * to float once; w = 1; out->result_fp64, when set, receives the FP64 quotient of the result. */
arc_status arc_accum_normalize(arc_context* ctx, const ArcAccumView* acc, int64_t num_paths,
                               const ArcOutputView* out);

typedef enum arc_error_metric {
    ARC_ERROR_REFERENCE = 0, /* CReferenceImage::GetError as written: (e_r * e_g + e_b) / 3 */
    ARC_ERROR_RMSE = 1       /* the mean it was meant to be: (e_r + e_g + e_b) / 3 */
} arc_error_metric;

/* Error of device RGBA plane `image` against `reference` (CReferenceImage.cpp:28-51): per channel
 * e_c = sqrt(mean over pixels of min(100, d_c^2)), d = reference - image in FP32, summed in FP64;
 * *error per `metric`; channel_rmse (3 doubles, may be NULL) receives e. */
arc_status arc_image_error(arc_context* ctx, const float* reference, const float* image, int32_t width,
                           int32_t height, int64_t pitch, int32_t metric, double* error, double* channel_rmse);

/* Host RGBA float plane (row 0 = top, pitch in pixels) to a file: PFM as CExport::ExportPFM
 * (Utils/CExport.cpp:22-58: "PF", little-endian scale -1.0, RGB rows bottom to top), or Radiance
 * RGBE .hdr as CExport::ExportHDR (top to bottom, run-length scanlines for widths 8..32767). */
arc_status arc_export_pfm(const char* path, const float* rgba, int32_t width, int32_t height, int64_t pitch);
arc_status arc_export_hdr(const char* path, const float* rgba, int32_t width, int32_t height, int64_t pitch);

/* ---------------------------------------------------------------------------------------- */
/* Synthetic scenes (CPU): inputs for tests and benchmarks                                   */
/* ---------------------------------------------------------------------------------------- */

#define ARC_SCENE_MAX_BOXES 32

typedef struct ArcBox {
    ArcFloat3 lo;
    ArcFloat3 hi;
    int32_t material;
} ArcBox;

typedef struct ArcSceneDesc {
    int32_t num_boxes;
    ArcBox boxes[ARC_SCENE_MAX_BOXES];
    int32_t num_materials;
    ArcMaterial materials[ARC_MAX_MATERIALS];
    ArcFloat3 light_center;   /* area light quad centre (faces -y) */
    float light_half_size;    /* half edge length of the square light */
    ArcFloat3 light_radiance; /* emitted radiance */
    int32_t light_material;
    ArcFloat3 camera_position;
    ArcFloat3 camera_target;
    float camera_fov_deg; /* vertical field of view */
    ArcFloat3 scene_min;
    ArcFloat3 scene_max;
} ArcSceneDesc;

typedef enum arc_scene_preset {
    ARC_SCENE_ROOM = 0,         /* open-front room, red/green side walls, gray 0.7 elsewhere */
    ARC_SCENE_ROOM_2BOXES = 1,  /* room + two boxes */
    ARC_SCENE_ROOM_RANDOM = 2,  /* room + `num_boxes` random boxes (seeded) */
    ARC_SCENE_TRAIN_VARIANT = 3 /* room + 0..16 random boxes, random albedo and light position (seeded) */
} arc_scene_preset;

arc_status arc_scene_preset_desc(int32_t preset, uint64_t seed, int32_t num_boxes, ArcSceneDesc* out);

/* Light tracer with the AVPL semantics of AvplShooter::createPath (AvplShooter.h:77-142):
 * PCG32 stream per path, cosine-weighted bounces, Russian roulette 0.8, at most max_bounces
 * bounces.  Writes exactly num_avpls indirect (bounce >= 1) AVPLs; *num_paths receives the
 * number of light paths they came from. */
arc_status arc_scene_trace_avpls(const ArcSceneDesc* scene, uint64_t seed, int32_t max_bounces,
                                 int32_t explicit_direct_illum, int32_t num_avpls, ArcAvplHost* out,
                                 int64_t* num_paths);

/* One primary ray per pixel centre from the scene's pinhole camera.  Writes float4 planes
 * (position (x,y,z,1), normal (n, float(material))); misses are all zero (material 0).
 * Row 0 is the top of the image. */
arc_status arc_scene_gbuffer(const ArcSceneDesc* scene, int32_t width, int32_t height, float* position,
                             float* normal);

/* The same two generators on the GPU (csrc/scene_gpu.cu), on the context's stream: the same
 * G-buffer bits, and the same AVPLs in the same order up to the rounding of the azimuth's
 * cos / sin (device vs host math library).  arc_scene_gbuffer_device writes the
 * caller's device planes `out` (out->width x out->height, row pitch out->pitch float4s; the view's
 * planes are written).  arc_scene_trace_avpls_device writes out->numAvpls AVPLs into the caller's
 * device SoA arrays `out` (AvplsGpuParam layout), in the CPU tracer's order; returns after the
 * tracer has produced them (it reads the running count back between batches of paths). */
arc_status arc_scene_gbuffer_device(arc_context* ctx, const ArcSceneDesc* scene, const ArcGBufferView* out);
arc_status arc_scene_trace_avpls_device(arc_context* ctx, const ArcSceneDesc* scene, uint64_t seed,
                                        int32_t max_bounces, int32_t explicit_direct_illum,
                                        const ArcAvplsGpuParam* out, int64_t* num_paths);

/* Views of a multi-view batch in `scene`: camera inside the room (outside every box) looking at a
 * point of the room at least 0.3 away, resolution drawn uniformly from {256x256, 512x512,
 * 1280x720, 1920x1080}, AVPL count log-uniform in [8192, 262144], and a seed for the view's own
 * AVPL set; all drawn from the PCG32 stream (seed, 0). */
typedef struct ArcBatchViewDesc {
    int32_t width;
    int32_t height;
    int32_t num_avpls;
    uint64_t avpl_seed;
    ArcFloat3 camera_position;
    ArcFloat3 camera_target;
} ArcBatchViewDesc;
arc_status arc_scene_batch_views(const ArcSceneDesc* scene, uint64_t seed, int32_t count, ArcBatchViewDesc* out);

#ifdef __cplusplus
}
#endif

#endif /* ARC_API_H_ */
