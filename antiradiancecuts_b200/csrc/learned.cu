// Learned cut selection (placeholder until the MLP kernels land).
#include "arc_internal.h"

namespace arc {

arc_status launch_cut_select_learned(arc_context*, const arc_lbvh*, const ArcCutParams*, const float4*, int, int,
                                     int32_t*, int32_t*, int) {
    set_last_error("learned cut not available");
    return ARC_ERR_UNSUPPORTED;
}

}  // namespace arc
