// Batched multi-view rendering.  No counterpart in the reference: its CudaGather::run renders one
// view per call (cudaGather.cu:836-1051).
//
// A batch renders many views, each with its own AVPL set, G-buffer and outputs: per view an LBVH
// build and a cut gather, enqueued in view order on the context's stream.  One LBVH object serves
// every view in turn (the stream orders each view's build after the previous view's gather), and
// the context's scratch buffers grow to the largest view on the first pass.  arc_batch_capture
// records the whole batch into one CUDA graph after an eager pass has sized every buffer, so
// that arc_batch_launch replays all views' kernels with a single launch and no host work per view.
#include <cuda_runtime.h>

#include "arc_internal.h"

struct arc_batch {
    arc_context* ctx = nullptr;
    arc_lbvh* bvh = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

arc_status check_views(const ArcBatchView* views, int32_t n, const ArcLbvhParams* lbvh, const ArcGatherParams* gather,
                       const ArcCutParams* cut) {
    ARC_CHECK_ARG(views && lbvh && gather && cut, "NULL argument");
    ARC_CHECK_ARG(n > 0, "empty batch");
    for (int32_t v = 0; v < n; ++v) ARC_CHECK_ARG(views[v].avpls.numAvpls >= 2, "every view needs >= 2 AVPLs");
    return ARC_OK;
}

arc_status render(arc_batch* b, const ArcBatchView* views, int32_t n, const ArcLbvhParams* lbvh,
                  const ArcGatherParams* gather, const ArcCutParams* cut) {
    for (int32_t v = 0; v < n; ++v) {
        const ArcBatchView& view = views[v];
        ARC_TRY(arc_lbvh_build(b->bvh, &view.avpls, lbvh));
        ARC_TRY(arc_gather_cut(b->ctx, b->bvh, &view.avpls, &view.gbuffer, view.camera_position, gather, cut,
                               &view.out));
    }
    return ARC_OK;
}

void release_graph(arc_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

}  // namespace

extern "C" arc_status arc_batch_create(arc_context* ctx, arc_batch** out) {
    ARC_CHECK_ARG(ctx && out, "NULL argument");
    *out = nullptr;
    arc_batch* b = new arc_batch();
    b->ctx = ctx;
    const arc_status s = arc_lbvh_create(ctx, &b->bvh);
    if (s != ARC_OK) {
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
    if (b->bvh) arc_lbvh_destroy(b->bvh);
    delete b;
    return ARC_OK;
}

extern "C" arc_status arc_batch_render(arc_batch* b, const ArcBatchView* views, int32_t num_views,
                                       const ArcLbvhParams* lbvh, const ArcGatherParams* gather,
                                       const ArcCutParams* cut) {
    ARC_CHECK_ARG(b, "NULL batch");
    ARC_TRY(check_views(views, num_views, lbvh, gather, cut));
    ARC_TRY_CUDA(cudaSetDevice(b->ctx->device));
    return render(b, views, num_views, lbvh, gather, cut);
}

extern "C" arc_status arc_batch_capture(arc_batch* b, const ArcBatchView* views, int32_t num_views,
                                        const ArcLbvhParams* lbvh, const ArcGatherParams* gather,
                                        const ArcCutParams* cut) {
    ARC_CHECK_ARG(b, "NULL batch");
    ARC_TRY(check_views(views, num_views, lbvh, gather, cut));
    ARC_CHECK_ARG(cut->kind == ARC_CUT_ERROR_BOUND, "only error-bound cuts can be recorded into a graph");
    arc_context* ctx = b->ctx;
    ARC_CHECK_ARG(!ctx->timer.enabled, "disable stage profiling before recording a batch");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    release_graph(b);
    // eager pass: every scratch buffer reaches its largest size, so recording allocates nothing
    ARC_TRY(render(b, views, num_views, lbvh, gather, cut));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    ARC_TRY_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    const arc_status s = render(b, views, num_views, lbvh, gather, cut);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);  // always ends the capture
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
