// tvg_step.cu -- one tree-force evaluation on device-resident particles, with
// per-phase CUDA-event timing on the context stream.
#include "tvg_internal.cuh"

extern "C" int tvg_force_step(tvg_context *ctx, int32_t form, int32_t use_bh, uint32_t parts,
                              int32_t ewald_kind)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_domain) return tvg_fail(ctx, TVG_E_STATE, "force_step: domain not set");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	cudaEvent_t *ev = ctx->ev;
	TVG_CUDA(ctx, cudaEventRecord(ev[8], s));
	TVG_CHECK(tvg_impl_keys(ctx, false));
	ctx->keys_std = true;
	TVG_CUDA(ctx, cudaEventRecord(ev[9], s));
	TVG_CHECK(tvg_impl_sort(ctx, nullptr));
	ctx->sorted = true;
	ctx->use_active = false;
	TVG_CUDA(ctx, cudaEventRecord(ev[10], s));
	TVG_CHECK(tvg_impl_top_nodes(ctx));
	ctx->have_top = true;
	TVG_CUDA(ctx, cudaEventRecord(ev[11], s));
	const uint32_t bflags = form == TVG_FORM_PLAIN ? TVG_BUILD_EXACT_MOMENTS : 0;
	TVG_CHECK(tvg_impl_tree_build(ctx, bflags));
	ctx->have_tree = true;
	ctx->have_walktree = false;
	TVG_CUDA(ctx, cudaEventRecord(ev[12], s));
	if ((parts & TVG_WALK_EWALD) && !ctx->have_ewald) {
		TVG_CHECK(tvg_impl_ewald_init(ctx));
		ctx->have_ewald = true;
	}
	TVG_CHECK(tvg_impl_zero_accel(ctx));
	if (form == TVG_FORM_PLAIN)
		TVG_CHECK(tvg_impl_walk_plain(ctx, use_bh, parts));
	else
		TVG_CHECK(tvg_impl_walk_group(ctx, use_bh, parts, ewald_kind));
	TVG_CUDA(ctx, cudaEventRecord(ev[13], s));
	TVG_CUDA(ctx, cudaEventSynchronize(ev[13]));
	float ms[5];
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[0], ev[8], ev[9]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[1], ev[9], ev[10]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[2], ev[10], ev[11]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[3], ev[11], ev[12]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[4], ev[8], ev[13]));
	ctx->phase_ms[0] = ms[0];
	ctx->phase_ms[1] = ms[1];
	ctx->phase_ms[2] = ms[2];
	ctx->phase_ms[3] = ms[3];
	ctx->phase_ms[6] = ms[4];
	return tvg_sync_status(ctx, "force_step");
}
