// Learned cut selection (placeholder until the MLP kernels land).
#include "arc_internal.h"

namespace arc {

arc_status launch_cut_select_learned(arc_context*, const arc_lbvh*, const ArcGatherParams*, const ArcCutParams*,
                                     const float4*, int, int, const CutPool&) {
    set_last_error("learned cut not available");
    return ARC_ERR_UNSUPPORTED;
}

}  // namespace arc
