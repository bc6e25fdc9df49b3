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

// Compute_Acceleration (accel.c:15-71) after the single-rank domain
// decomposition: keys, sort, active list, top nodes, build, walks.
extern "C" int tvg_compute_acceleration(tvg_context *ctx, int32_t form, uint32_t parts,
                                        int32_t ewald_kind, int32_t prepare)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_domain) return tvg_fail(ctx, TVG_E_STATE, "compute_acceleration: domain not set");
	if (form != TVG_FORM_PLAIN && form != TVG_FORM_GROUP)
		return tvg_fail(ctx, TVG_E_BADINPUT, "unknown form %d", form);
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	cudaEvent_t *ev = ctx->ev;
	TVG_CUDA(ctx, cudaEventRecord(ev[8], s));
	TVG_CHECK(tvg_impl_keys(ctx, false));
	ctx->keys_std = true;
	TVG_CUDA(ctx, cudaEventRecord(ev[9], s));
	TVG_CHECK(tvg_impl_sort(ctx, nullptr));
	ctx->sorted = true;
	// Sort_Particles_By_Peano_Key ends with Make_Active_Particle_List (peano.c:42)
	if (ctx->have_timeline) {
		TVG_CHECK(tvg_impl_active_from_bins(ctx));
	} else {
		ctx->use_active = false;
	}
	TVG_CUDA(ctx, cudaEventRecord(ev[10], s));
	TVG_CHECK(tvg_impl_top_nodes(ctx));
	ctx->have_top = true;
	TVG_CUDA(ctx, cudaEventRecord(ev[11], s));
	TVG_CHECK(tvg_impl_tree_build(ctx, form == TVG_FORM_PLAIN ? TVG_BUILD_EXACT_MOMENTS : 0));
	ctx->have_tree = true;
	ctx->have_walktree = false;
	TVG_CUDA(ctx, cudaEventRecord(ev[12], s));
	if ((parts & TVG_WALK_EWALD) && !ctx->have_ewald) {
		TVG_CHECK(tvg_impl_ewald_init(ctx));
		ctx->have_ewald = true;
	}
	// safe_last_accel, accel.c:28-43 (the active particles)
	TVG_CHECK(tvg_impl_save_last_accel(ctx));
	if (prepare) {
		// accel.c:56-65: a Barnes-Hut pass gives |a_old| for the relative criterion
		if (ctx->have_timeline) ctx->tl.state.prepare_step = 1;
		if (form == TVG_FORM_PLAIN) TVG_CHECK(tvg_impl_walk_plain(ctx, 1, parts));
		else TVG_CHECK(tvg_impl_walk_group(ctx, 1, parts, ewald_kind));
		TVG_CHECK(tvg_impl_save_last_accel(ctx));
	}
	if (form == TVG_FORM_PLAIN) TVG_CHECK(tvg_impl_walk_plain(ctx, 0, parts));
	else TVG_CHECK(tvg_impl_walk_group(ctx, 0, parts, ewald_kind));
	if (ctx->have_timeline) ctx->tl.state.prepare_step = 0;
	TVG_CUDA(ctx, cudaEventRecord(ev[13], s));
	TVG_CUDA(ctx, cudaEventSynchronize(ev[13]));
	float ms[5];
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[0], ev[8], ev[9]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[1], ev[9], ev[10]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[2], ev[10], ev[11]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[3], ev[11], ev[12]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[4], ev[8], ev[13]));
	for (int i = 0; i < 4; i++) ctx->phase_ms[i] = ms[i];
	ctx->phase_ms[6] = ms[4];
	return tvg_sync_status(ctx, "compute_acceleration");
}
