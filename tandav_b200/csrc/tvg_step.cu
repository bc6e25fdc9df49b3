// tvg_step.cu -- one tree-force evaluation on device-resident particles, with
// per-phase CUDA-event timing on the context stream; the same evaluation from
// and to host buffers with the copies overlapped (tvg_force_step_host); and
// the evaluation captured as a CUDA graph (tvg_step_graph).
#include <string.h>

#include "tvg_internal.cuh"

// set_computational_domain at every decomposition (TVG_CFG_FIND_DOMAIN, isolated)
static bool find_domain_each_step(const tvg_context *ctx)
{
	return (ctx->cfg.flags & TVG_CFG_FIND_DOMAIN) && !ctx->cfg.periodic;
}

// keys, sort, top nodes, tree build and walks of one force step, enqueued on
// the context stream between the phase events ev[8..13]; `sorted`, when set,
// is recorded right after the sort
static int force_phases(tvg_context *ctx, int32_t form, int32_t use_bh, uint32_t parts, int32_t ewald_kind,
                        cudaEvent_t sorted)
{
	cudaStream_t s = ctx->stream;
	cudaEvent_t *ev = ctx->ev;
	if (find_domain_each_step(ctx)) {
		double o[3], sz;
		TVG_CHECK(tvg_find_domain(ctx, o, &sz));
	}
	TVG_CUDA(ctx, cudaEventRecord(ev[8], s));
	TVG_CHECK(tvg_impl_keys(ctx, false));
	ctx->keys_std = true;
	TVG_CUDA(ctx, cudaEventRecord(ev[9], s));
	TVG_CHECK(tvg_impl_sort(ctx, nullptr));
	ctx->sorted = true;
	ctx->use_active = false;
	if (sorted) TVG_CUDA(ctx, cudaEventRecord(sorted, s));
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
	return TVG_OK;
}

// the phase times of the last force step, once ev[13] has completed
static int force_times(tvg_context *ctx)
{
	cudaEvent_t *ev = ctx->ev;
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
	return TVG_OK;
}

extern "C" int tvg_force_step(tvg_context *ctx, int32_t form, int32_t use_bh, uint32_t parts,
                              int32_t ewald_kind)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_domain && !find_domain_each_step(ctx))
		return tvg_fail(ctx, TVG_E_STATE, "force_step: domain not set");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(force_phases(ctx, form, use_bh, parts, ewald_kind, nullptr));
	TVG_CUDA(ctx, cudaEventSynchronize(ctx->ev[13]));
	TVG_CHECK(force_times(ctx));
	return tvg_sync_status(ctx, "force_step");
}

// Fields that the steps after the sort never write: a force step from host
// buffers downloads them while the walks run.
static const uint32_t kWrittenByStep = TVG_F_ACC | TVG_F_GRAV_ACC | TVG_F_COST | TVG_F_TREE_PARENT
                                     | TVG_F_GRAV_POT;

extern "C" int tvg_force_step_host(tvg_context *ctx, int64_t n, const tvg_particles *in, uint32_t in_fields,
                                   tvg_particles *out, uint32_t out_fields, int32_t form, int32_t use_bh,
                                   uint32_t parts, int32_t ewald_kind)
{
	if (!ctx || !in || !out) return TVG_E_BADINPUT;
	if (n < 0 || n > ctx->cap)
		return tvg_fail(ctx, TVG_E_BADINPUT, "force_step_host: n=%lld > capacity %lld", (long long) n,
		                (long long) ctx->cap);
	if (!(in_fields & TVG_F_POS)) return tvg_fail(ctx, TVG_E_BADINPUT, "force_step_host: positions are an input");
	if ((in_fields | out_fields) & TVG_F_KEY)
		return tvg_fail(ctx, TVG_E_BADINPUT, "force_step_host: keys are no field of this call");
	if (!ctx->have_domain && !find_domain_each_step(ctx))
		return tvg_fail(ctx, TVG_E_STATE, "force_step_host: domain not set");
	for (int f = 0; f < FS_NFIELDS; f++) {
		if ((in_fields & tvg_slot_bit(f)) && !tvg_host_field(in, f))
			return tvg_fail(ctx, TVG_E_BADINPUT, "force_step_host: input field slot %d is NULL", f);
		if ((out_fields & tvg_slot_bit(f)) && !tvg_host_field(out, f))
			return tvg_fail(ctx, TVG_E_BADINPUT, "force_step_host: output field slot %d is NULL", f);
		if (((in_fields | out_fields) & tvg_slot_bit(f)) && !ctx->f[f])
			return tvg_fail(ctx, TVG_E_STATE, "force_step_host: field slot %d is not kept by this context", f);
	}
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (!ctx->copy_stream) TVG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
	for (int i = 0; i < 3; i++)
		if (!ctx->xev[i]) TVG_CUDA(ctx, cudaEventCreateWithFlags(&ctx->xev[i], cudaEventDisableTiming));
	cudaStream_t s = ctx->stream, cs = ctx->copy_stream;
	ctx->n = n;
	ctx->sorted = false;
	ctx->have_tree = false;
	ctx->have_top = false;
	ctx->use_active = false;
	// positions first, on the context stream: the keys need them
	for (int f = FS_POS0; f <= FS_POS2; f++)
		TVG_CUDA(ctx, cudaMemcpyAsync(ctx->f[f], tvg_host_field(in, f), tvg_field_bytes(ctx, f) * n,
		                              cudaMemcpyHostToDevice, s));
	// then the other inputs on the copy stream, while the keys and the radix
	// passes run; the field gather of the sort waits for them
	TVG_CUDA(ctx, cudaEventRecord(ctx->xev[0], s));
	TVG_CUDA(ctx, cudaStreamWaitEvent(cs, ctx->xev[0], 0));
	for (int f = 0; f < FS_NFIELDS; f++) {
		if (f >= FS_POS0 && f <= FS_POS2) continue;
		if (!(in_fields & tvg_slot_bit(f))) continue;
		TVG_CUDA(ctx, cudaMemcpyAsync(ctx->f[f], tvg_host_field(in, f), tvg_field_bytes(ctx, f) * n,
		                              cudaMemcpyHostToDevice, cs));
	}
	TVG_CUDA(ctx, cudaEventRecord(ctx->xev[1], cs));
	// the isolated domain search reads the particles before the sort
	if (find_domain_each_step(ctx)) TVG_CUDA(ctx, cudaStreamWaitEvent(s, ctx->xev[1], 0));
	ctx->gather_wait = ctx->xev[1];
	const int rc = force_phases(ctx, form, use_bh, parts, ewald_kind, ctx->xev[2]);
	ctx->gather_wait = nullptr;
	if (rc != TVG_OK) {
		cudaStreamSynchronize(cs);
		return rc;
	}
	// outputs the walks do not write leave as soon as the sort is done, the
	// others after the walks
	TVG_CUDA(ctx, cudaStreamWaitEvent(cs, ctx->xev[2], 0));
	for (int f = 0; f < FS_NFIELDS; f++) {
		const uint32_t bit = tvg_slot_bit(f);
		if (!(out_fields & bit)) continue;
		TVG_CUDA(ctx, cudaMemcpyAsync(tvg_host_field(out, f), ctx->f[f], tvg_field_bytes(ctx, f) * n,
		                              cudaMemcpyDeviceToHost, (bit & kWrittenByStep) ? s : cs));
	}
	TVG_CUDA(ctx, cudaStreamSynchronize(cs));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	TVG_CHECK(force_times(ctx));
	return tvg_sync_status(ctx, "force_step_host");
}

// The launches of Compute_Acceleration (accel.c:15-71) after the single-rank
// domain decomposition: keys, sort, active list, top nodes, build, walks,
// bracketed by the phase events ev[8..13]. No host synchronisation while a
// capture is in progress.
static int accel_phases(tvg_context *ctx, int32_t form, uint32_t parts, int32_t ewald_kind,
                        int32_t prepare)
{
	cudaEvent_t *ev = ctx->ev;
	// without a due domain update the kept tree is walked (accel.c:53, main.c:73-78)
	const bool keep_tree = tvg_tree_update_due(ctx);
	if (keep_tree) TVG_CHECK(tvg_tree_update_check(ctx, "compute_acceleration"));
	TVG_CUDA(ctx, tvg_record(ctx, ev[8]));
	if (keep_tree) {
		TVG_CUDA(ctx, tvg_record(ctx, ev[9]));
		TVG_CUDA(ctx, tvg_record(ctx, ev[10]));
		TVG_CUDA(ctx, tvg_record(ctx, ev[11]));
		ctx->have_walktree = false;
	} else {
		// set_computational_domain (domain.c:67-71), on the current order
		if (find_domain_each_step(ctx)) {
			if (ctx->capturing) return tvg_fail(ctx, TVG_E_STATE, "find_domain cannot be captured");
			double o[3], sz;
			TVG_CHECK(tvg_find_domain(ctx, o, &sz));
		}
		TVG_CHECK(tvg_impl_keys(ctx, false));
		ctx->keys_std = true;
		TVG_CUDA(ctx, tvg_record(ctx, ev[9]));
		TVG_CHECK(tvg_impl_sort(ctx, nullptr));
		ctx->sorted = true;
		// Sort_Particles_By_Peano_Key ends with Make_Active_Particle_List (peano.c:42)
		if (ctx->have_timeline) {
			TVG_CHECK(tvg_impl_active_from_bins(ctx));
		} else {
			ctx->use_active = false;
		}
		TVG_CUDA(ctx, tvg_record(ctx, ev[10]));
		TVG_CHECK(tvg_impl_top_nodes(ctx));
		ctx->have_top = true;
		TVG_CUDA(ctx, tvg_record(ctx, ev[11]));
		TVG_CHECK(tvg_impl_tree_build(ctx, form == TVG_FORM_PLAIN ? TVG_BUILD_EXACT_MOMENTS : 0));
		ctx->have_tree = true;
		ctx->have_walktree = false;
	}
	TVG_CUDA(ctx, tvg_record(ctx, ev[12]));
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
	TVG_CUDA(ctx, tvg_record(ctx, ev[13]));
	return TVG_OK;
}

// phase times from the events of the last step (synchronises)
static int accel_times(tvg_context *ctx)
{
	cudaEvent_t *ev = ctx->ev;
	TVG_CUDA(ctx, cudaEventSynchronize(ev[13]));
	float ms[5];
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[0], ev[8], ev[9]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[1], ev[9], ev[10]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[2], ev[10], ev[11]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[3], ev[11], ev[12]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms[4], ev[8], ev[13]));
	for (int i = 0; i < 4; i++) ctx->phase_ms[i] = ms[i];
	ctx->phase_ms[6] = ms[4];
	return TVG_OK;
}

static int accel_check(tvg_context *ctx, int32_t form)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_domain && !find_domain_each_step(ctx))
		return tvg_fail(ctx, TVG_E_STATE, "compute_acceleration: domain not set");
	if (form != TVG_FORM_PLAIN && form != TVG_FORM_GROUP)
		return tvg_fail(ctx, TVG_E_BADINPUT, "unknown form %d", form);
	return TVG_OK;
}

extern "C" int tvg_compute_acceleration(tvg_context *ctx, int32_t form, uint32_t parts,
                                        int32_t ewald_kind, int32_t prepare)
{
	TVG_CHECK(accel_check(ctx, form));
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if ((parts & TVG_WALK_EWALD) && !ctx->have_ewald) {
		TVG_CHECK(tvg_impl_ewald_init(ctx));
		ctx->have_ewald = true;
	}
	TVG_CHECK(accel_phases(ctx, form, parts, ewald_kind, prepare));
	TVG_CHECK(accel_times(ctx));
	return tvg_sync_status(ctx, "compute_acceleration");
}

// ------------------------------------------------------------- CUDA graph
//
// The step's launch sequence has no host round trip (every count stays on the
// device), so it is captured once and replayed. Captured kernels keep the
// buffer pointers they were given; the sort leaves the particle fields, the
// low key words and the permutation in the other buffer of their pair (and
// the radix passes, always eight, leave the high words where they were), so
// the buffers alternate between two states from step to step. One graph is
// kept per state, with the pointer set it starts from and the one it leaves.

enum { GP_KEY_HI, GP_KEY_LO, GP_KEY_TMP, GP_PERM, GP_PERM_TMP, GP_FIELDS };
#define GP_N (GP_FIELDS + 2 * FS_NFIELDS)

struct tvg_graph_entry {
	cudaGraphExec_t exec = nullptr;
	uint64_t key = 0;
	void *start[GP_N];
	void *end[GP_N];
	int64_t launches = 0;
};

static void snap_ptrs(const tvg_context *ctx, void **p)
{
	p[GP_KEY_HI] = ctx->key_hi;
	p[GP_KEY_LO] = ctx->key_lo;
	p[GP_KEY_TMP] = ctx->key_tmp;
	p[GP_PERM] = ctx->perm;
	p[GP_PERM_TMP] = ctx->perm_tmp;
	for (int f = 0; f < FS_NFIELDS; f++) {
		p[GP_FIELDS + f] = ctx->f[f];
		p[GP_FIELDS + FS_NFIELDS + f] = ctx->falt[f];
	}
}

static void set_ptrs(tvg_context *ctx, void *const *p)
{
	ctx->key_hi = (uint64_t *) p[GP_KEY_HI];
	ctx->key_lo = (uint64_t *) p[GP_KEY_LO];
	ctx->key_tmp = (uint64_t *) p[GP_KEY_TMP];
	ctx->perm = (uint32_t *) p[GP_PERM];
	ctx->perm_tmp = (uint32_t *) p[GP_PERM_TMP];
	for (int f = 0; f < FS_NFIELDS; f++) {
		ctx->f[f] = p[GP_FIELDS + f];
		ctx->falt[f] = p[GP_FIELDS + FS_NFIELDS + f];
	}
}

static bool same_ptrs(void *const *a, void *const *b)
{
	for (int i = 0; i < GP_N; i++)
		if (a[i] != b[i]) return false;
	return true;
}

void tvg_graph_release(tvg_context *ctx)
{
	for (int i = 0; i < 2; i++) {
		if (!ctx->graphs[i]) continue;
		if (ctx->graphs[i]->exec) cudaGraphExecDestroy(ctx->graphs[i]->exec);
		delete ctx->graphs[i];
		ctx->graphs[i] = nullptr;
	}
	ctx->graph_warm_key = 0;
}

static uint64_t mix(uint64_t k, uint64_t v)
{
	k ^= v + 0x9E3779B97F4A7C15ull + (k << 6) + (k >> 2);
	return k;
}

static uint64_t mix_d(uint64_t k, double v)
{
	uint64_t b;
	memcpy(&b, &v, 8);
	return mix(k, b);
}

// the configuration a graph is valid for: everything the captured launches
// were given by value (a change forces a direct step and new captures)
static uint64_t graph_key(const tvg_context *ctx, uint32_t parts, int32_t ewald_kind)
{
	const tvg_config &c = ctx->cfg;
	uint64_t k = 1;
	k = mix(k, parts);
	k = mix(k, (uint32_t) ewald_kind);
	k = mix(k, (uint32_t) ctx->group_tpl);
	k = mix(k, ctx->have_timeline ? 1u : 0u);
	k = mix(k, (uint64_t) ctx->n);
	k = mix(k, ctx->mlp_ok ? 1u : 0u);
	k = mix(k, (uint64_t) c.flags);
	k = mix(k, (uint64_t) c.vector_size);
	k = mix_d(k, c.open_rel);
	k = mix_d(k, c.open_bh);
	k = mix_d(k, c.gravity);
	k = mix_d(k, c.softening);
	k = mix_d(k, c.boxsize);
	k = mix_d(k, ctx->ewald_open_rel);
	k = mix_d(k, ctx->ewald_open_bh);
	k = mix(k, (uint32_t) ctx->walk_limit);
	k = mix_d(k, ctx->dsize);
	for (int d = 0; d < 3; d++) k = mix_d(k, ctx->origin[d]);
	return k ? k : 1;
}

static int capture(tvg_context *ctx, uint32_t parts, int32_t ewald_kind, uint64_t key,
                   tvg_graph_entry **out)
{
	cudaStream_t s = ctx->stream;
	tvg_graph_entry *e = new tvg_graph_entry;
	e->key = key;
	snap_ptrs(ctx, e->start);
	const int64_t l0 = ctx->launches;
	cudaError_t ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
	if (ce != cudaSuccess) {
		delete e;
		return tvg_fail(ctx, TVG_E_CUDA, "step graph: begin capture: %s", cudaGetErrorString(ce));
	}
	ctx->capturing = true;
	int rc = accel_phases(ctx, TVG_FORM_GROUP, parts, ewald_kind, 0);
	ctx->capturing = false;
	cudaGraph_t g = nullptr;
	ce = cudaStreamEndCapture(s, &g);
	snap_ptrs(ctx, e->end);
	e->launches = ctx->launches - l0;
	// nothing ran yet: the buffers are where the capture started
	set_ptrs(ctx, e->start);
	ctx->launches = l0;
	if (rc == TVG_OK && ce != cudaSuccess)
		rc = tvg_fail(ctx, TVG_E_CUDA, "step graph: capture failed: %s", cudaGetErrorString(ce));
	if (rc == TVG_OK) {
		ce = cudaGraphInstantiate(&e->exec, g, 0);
		if (ce != cudaSuccess)
			rc = tvg_fail(ctx, TVG_E_CUDA, "step graph: instantiation failed: %s", cudaGetErrorString(ce));
	}
	if (g) cudaGraphDestroy(g);
	if (rc != TVG_OK) {
		cudaGetLastError();
		if (e->exec) cudaGraphExecDestroy(e->exec);
		delete e;
		return rc;
	}
	*out = e;
	return TVG_OK;
}

extern "C" int tvg_step_graph(tvg_context *ctx, uint32_t parts, int32_t ewald_kind)
{
	TVG_CHECK(accel_check(ctx, TVG_FORM_GROUP));
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	// a step on the kept tree (no keys, sort or build), or one that finds its
	// domain first or balances its top nodes over several targets (host
	// synchronisations), runs directly
	const bool balanced = ctx->dd_ntask > 1 && ctx->dd_ntask < 65;
	if (tvg_tree_update_due(ctx) || find_domain_each_step(ctx) || balanced)
		return tvg_compute_acceleration(ctx, TVG_FORM_GROUP, parts, ewald_kind, 0);
	const uint64_t key = graph_key(ctx, parts, ewald_kind);
	if (key != ctx->graph_warm_key) {
		// a new configuration: one direct step, which also makes every
		// allocation, table and kernel attribute the captured step relies on
		tvg_graph_release(ctx);
		TVG_CHECK(tvg_compute_acceleration(ctx, TVG_FORM_GROUP, parts, ewald_kind, 0));
		ctx->graph_warm_key = key;
		return TVG_OK;
	}
	void *cur[GP_N];
	snap_ptrs(ctx, cur);
	tvg_graph_entry *e = nullptr;
	int slot = -1;
	for (int i = 0; i < 2; i++) {
		if (ctx->graphs[i] && ctx->graphs[i]->key == key && same_ptrs(ctx->graphs[i]->start, cur)) {
			e = ctx->graphs[i];
			break;
		}
		if (slot < 0 && !ctx->graphs[i]) slot = i;
	}
	if (!e) {
		if (slot < 0) {             // buffers moved: start over
			tvg_graph_release(ctx);
			ctx->graph_warm_key = key;
			slot = 0;
		}
		TVG_CHECK(capture(ctx, parts, ewald_kind, key, &e));
		ctx->graphs[slot] = e;
	}
	if (ctx->have_timeline) TVG_CHECK(tvg_set_device_max_bin(ctx));
	TVG_CUDA(ctx, cudaGraphLaunch(e->exec, ctx->stream));
	ctx->launches += e->launches;
	set_ptrs(ctx, e->end);
	ctx->keys_std = ctx->sorted = ctx->have_top = ctx->have_tree = ctx->have_walktree = true;
	ctx->use_active = ctx->have_timeline;
	// host mirrors of the step's counts and times (one synchronisation)
	TVG_CHECK(accel_times(ctx));
	TVG_CHECK(tvg_walk_group_results(ctx));
	TVG_CHECK(tvg_read_counts(ctx));
	if (ctx->have_timeline) {
		int64_t na = 0;
		TVG_CUDA(ctx, cudaMemcpy(&na, &ctx->dc->n_active, 8, cudaMemcpyDeviceToHost));
		ctx->n_active = na;
		ctx->tl.state.n_active = na;
	}
	return tvg_sync_status(ctx, "step_graph");
}

extern "C" int tvg_step_graph_reset(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	tvg_graph_release(ctx);
	return TVG_OK;
}
