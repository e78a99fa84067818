// Device BVH builder (filled in below).
#include "rtb_internal.h"

namespace rtb {

rtb_status build_bvh(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                     rtb_scene** out, rtb_bvh_stats* stats) {
  (void)desc;
  (void)cfg;
  (void)out;
  (void)stats;
  return fail(ctx, RTB_ERR_UNSUPPORTED, "device builder not built");
}

}  // namespace rtb
