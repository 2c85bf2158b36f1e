// Batched multi-view rendering.  No counterpart in the reference: its CudaGather::run renders one
// view per call (cudaGather.cu:836-1051), and Renderer::Render loops over frames on the host
// (Render.cpp:230-389).
//
// A batch renders many views, each with its own AVPL set, G-buffer and outputs: per view an LBVH
// build and a cut gather.  Views of uneven sizes share the GPU through kLanes lanes that run
// concurrently: each lane is a sub-context with its own stream, scratch arena, LBVH and device
// error word, and takes a share of the views chosen longest-first (the view with the most
// estimated work goes to the lane with the least work so far), so that the small views fill the
// machine around the large ones instead of running alone one after another.  The lanes fork from
// the batch's stream with an event and join back into it; at the join each lane folds its error
// word into the owner context's.
//
// arc_batch_capture records the whole batch -- every lane, every view, the fork and the join --
// into one CUDA graph after an eager pass has sized every buffer, so that arc_batch_launch
// replays all views' kernels with a single launch and no host work per view.  Every cut kind
// records: the learned selection launches a fixed number of levels and reads nothing back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "arc_internal.h"

namespace {

constexpr int kLanes = 4;

struct Lane {
    arc_context* ctx = nullptr;
    arc_lbvh* bvh = nullptr;
    cudaEvent_t done = nullptr;
};

}  // namespace

struct arc_batch {
    arc_context* ctx = nullptr;  // owner: the batch runs on its stream and reports into its error word
    std::vector<Lane> lanes;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

// Folds a lane's device error word into the owner's and clears the lane's.
__global__ void fold_error_word(uint32_t* lane_err, uint32_t* owner_err) {
    const uint32_t w = *lane_err;
    if (w) {
        atomicOr(owner_err, w);
        *lane_err = 0u;
    }
}

arc_status check_views(const ArcBatchView* views, int32_t n, const ArcLbvhParams* lbvh, const ArcGatherParams* gather,
                       const ArcCutParams* cut) {
    ARC_CHECK_ARG(views && lbvh && gather && cut, "NULL argument");
    ARC_CHECK_ARG(n > 0, "empty batch");
    for (int32_t v = 0; v < n; ++v) ARC_CHECK_ARG(views[v].avpls.numAvpls >= 2, "every view needs >= 2 AVPLs");
    return ARC_OK;
}

// Estimated work of a view: its pixels times the log of its AVPL count (a cut's size grows about
// logarithmically with the AVPLs) plus its LBVH build.
double view_work(const ArcBatchView& v) {
    const double px = (double)v.gbuffer.width * v.gbuffer.height;
    return px * std::log2((double)v.avpls.numAvpls + 2.0) + 4.0 * v.avpls.numAvpls;
}

// View indices per lane, longest first onto the least-loaded lane (stable for equal work).
std::vector<std::vector<int>> assign(const ArcBatchView* views, int32_t n, int lanes) {
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return view_work(views[a]) > view_work(views[b]); });
    std::vector<std::vector<int>> out(lanes);
    std::vector<double> load(lanes, 0.0);
    for (int v : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        out[l].push_back(v);
        load[l] += view_work(views[v]);
    }
    return out;
}

// The lanes' material tables follow the owner's (uploaded only when they differ, so the pass that
// is recorded into a graph uploads nothing).
arc_status sync_materials(arc_batch* b) {
    const auto& m = b->ctx->host_materials;
    ARC_CHECK_ARG(!m.empty(), "materials not uploaded");
    for (Lane& l : b->lanes) {
        const auto& lm = l.ctx->host_materials;
        if (lm.size() == m.size() && std::memcmp(lm.data(), m.data(), sizeof(ArcMaterial) * m.size()) == 0) continue;
        ARC_TRY(arc_materials_upload(l.ctx, m.data(), (int32_t)m.size()));
    }
    return ARC_OK;
}

arc_status render(arc_batch* b, const ArcBatchView* views, int32_t n, const ArcLbvhParams* lbvh,
                  const ArcGatherParams* gather, const ArcCutParams* cut) {
    arc_context* ctx = b->ctx;
    const auto plan = assign(views, n, (int)b->lanes.size());
    ARC_TRY_CUDA(cudaEventRecord(b->fork, ctx->stream));
    for (Lane& l : b->lanes) ARC_TRY_CUDA(cudaStreamWaitEvent(l.ctx->stream, b->fork, 0));
    arc_status s = ARC_OK;
    for (size_t li = 0; li < b->lanes.size() && s == ARC_OK; ++li) {
        Lane& l = b->lanes[li];
        const uint64_t launches0 = l.ctx->launches;
        for (int v : plan[li]) {
            const ArcBatchView& view = views[v];
            s = arc_lbvh_build(l.bvh, &view.avpls, lbvh);
            if (s == ARC_OK)
                s = arc_gather_cut(l.ctx, l.bvh, &view.avpls, &view.gbuffer, view.camera_position, gather, cut,
                                   &view.out);
            if (s != ARC_OK) break;
        }
        ctx->launches += l.ctx->launches - launches0;
    }
    // the join is enqueued even after a failure, so that no lane stream is left forked
    for (Lane& l : b->lanes) {
        fold_error_word<<<1, 1, 0, l.ctx->stream>>>(l.ctx->d_error, ctx->d_error);
        ctx->launches += 1;
        const cudaError_t e1 = cudaEventRecord(l.done, l.ctx->stream);
        const cudaError_t e2 = cudaStreamWaitEvent(ctx->stream, l.done, 0);
        if (s == ARC_OK && (e1 != cudaSuccess || e2 != cudaSuccess)) {
            arc::set_last_error(std::string("batch join: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            s = ARC_ERR_CUDA;
        }
    }
    return s;
}

void release_graph(arc_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

void destroy_lanes(arc_batch* b) {
    for (Lane& l : b->lanes) {
        if (l.bvh) arc_lbvh_destroy(l.bvh);
        if (l.done) cudaEventDestroy(l.done);
        if (l.ctx) arc_context_destroy(l.ctx);
    }
    b->lanes.clear();
}

}  // namespace

extern "C" arc_status arc_batch_create(arc_context* ctx, arc_batch** out) {
    ARC_CHECK_ARG(ctx && out, "NULL argument");
    *out = nullptr;
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    arc_batch* b = new arc_batch();
    b->ctx = ctx;
    arc_status s = ARC_OK;
    cudaError_t e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int i = 0; i < kLanes && s == ARC_OK && e == cudaSuccess; ++i) {
        Lane l;
        s = arc_context_create(ctx->device, nullptr, &l.ctx);
        if (s == ARC_OK) s = arc_lbvh_create(l.ctx, &l.bvh);
        if (s == ARC_OK) e = cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming);
        b->lanes.push_back(l);
    }
    if (s == ARC_OK && e != cudaSuccess) {
        arc::set_last_error(std::string("arc_batch_create: ") + cudaGetErrorString(e));
        s = ARC_ERR_CUDA;
    }
    if (s != ARC_OK) {
        destroy_lanes(b);
        if (b->fork) cudaEventDestroy(b->fork);
        delete b;
        return s;
    }
    *out = b;
    return ARC_OK;
}

extern "C" arc_status arc_batch_destroy(arc_batch* b) {
    if (!b) return ARC_OK;
    if (b->ctx) cudaSetDevice(b->ctx->device);
    if (b->ctx && b->ctx->stream) cudaStreamSynchronize(b->ctx->stream);
    release_graph(b);
    destroy_lanes(b);
    if (b->fork) cudaEventDestroy(b->fork);
    delete b;
    return ARC_OK;
}

extern "C" arc_status arc_batch_render(arc_batch* b, const ArcBatchView* views, int32_t num_views,
                                       const ArcLbvhParams* lbvh, const ArcGatherParams* gather,
                                       const ArcCutParams* cut) {
    ARC_CHECK_ARG(b, "NULL batch");
    ARC_TRY(check_views(views, num_views, lbvh, gather, cut));
    ARC_CHECK_ARG(lbvh->wait_limit == 0, "a batch builds with the default wait limit");
    ARC_TRY_CUDA(cudaSetDevice(b->ctx->device));
    ARC_TRY(sync_materials(b));
    return render(b, views, num_views, lbvh, gather, cut);
}

extern "C" arc_status arc_batch_capture(arc_batch* b, const ArcBatchView* views, int32_t num_views,
                                        const ArcLbvhParams* lbvh, const ArcGatherParams* gather,
                                        const ArcCutParams* cut) {
    ARC_CHECK_ARG(b, "NULL batch");
    ARC_TRY(check_views(views, num_views, lbvh, gather, cut));
    ARC_CHECK_ARG(lbvh->wait_limit == 0, "a batch builds with the default wait limit");
    ARC_CHECK_ARG(cut->kind == ARC_CUT_ERROR_BOUND || cut->kind == ARC_CUT_LEARNED,
                  "error-bound and learned cuts can be recorded into a graph");
    arc_context* ctx = b->ctx;
    ARC_CHECK_ARG(!ctx->timer.enabled, "disable stage profiling before recording a batch");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    release_graph(b);
    ARC_TRY(sync_materials(b));
    // eager pass: every scratch buffer reaches its largest size, so recording allocates nothing
    ARC_TRY(render(b, views, num_views, lbvh, gather, cut));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    const uint64_t launches0 = ctx->launches;
    ARC_TRY_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    const arc_status s = render(b, views, num_views, lbvh, gather, cut);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);  // always ends the capture
    ctx->launches = launches0;  // recorded, not launched
    if (s != ARC_OK) {
        if (graph) cudaGraphDestroy(graph);
        return s;
    }
    ARC_TRY_CUDA(e);
    b->graph = graph;
    ARC_TRY_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return ARC_OK;
}

extern "C" arc_status arc_batch_launch(arc_batch* b) {
    ARC_CHECK_ARG(b, "NULL batch");
    ARC_CHECK_ARG(b->exec, "no recorded batch (arc_batch_capture)");
    ARC_TRY_CUDA(cudaSetDevice(b->ctx->device));
    ARC_TRY_CUDA(cudaGraphLaunch(b->exec, b->ctx->stream));
    return ARC_OK;
}
