// tvg_walk_group.cu -- the group form of the walk (one warp per PH group,
// FP32 on integer-offset positions).
#include "tvg_internal.cuh"

int tvg_impl_walk_group(tvg_context *ctx, int use_bh, uint32_t parts, int ewald_kind)
{
	(void) use_bh; (void) parts; (void) ewald_kind;
	return tvg_fail(ctx, TVG_E_STATE, "group walk not available in this build");
}
