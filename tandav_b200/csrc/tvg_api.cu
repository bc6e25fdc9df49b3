// tvg_api.cu -- context lifecycle, host<->device transfers, status handling
// and the extern "C" entry points declared in include/tandav_gpu.h.
#include <stdarg.h>
#include <stdlib.h>

#include "tvg_internal.cuh"

#define TVG_VERSION "tandav-b200 0.1 (sm_100a)"

int tvg_fail(tvg_context *ctx, int code, const char *fmt, ...)
{
	if (ctx) {
		va_list ap;
		va_start(ap, fmt);
		vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
		va_end(ap);
	}
	return code;
}

// Reads the device status word after a phase and maps it to an error code.
int tvg_sync_status(tvg_context *ctx, const char *phase)
{
	TVG_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->status, sizeof(int), cudaMemcpyDeviceToHost,
	                              ctx->stream));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	int st = *ctx->h_status;
	if (!st) return TVG_OK;
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->stream));
	if (st & TVG_ST_COINCIDENT)
		return tvg_fail(ctx, TVG_E_COINCIDENT, "%s: particles coincide to 41 key levels", phase);
	if (st & TVG_ST_BADPOS)
		return tvg_fail(ctx, TVG_E_BADINPUT, "%s: non-finite or out-of-domain position", phase);
	if (st & TVG_ST_TREE_FULL)
		return tvg_fail(ctx, TVG_E_TREE_FULL, "%s: node capacity exceeded", phase);
	if (st & TVG_ST_TIMEOUT)
		return tvg_fail(ctx, TVG_E_TIMEOUT, "%s: bounded device wait expired", phase);
	if (st & TVG_ST_LIST_OVERFLOW)
		return tvg_fail(ctx, TVG_E_TREE_FULL, "%s: interaction list overflow", phase);
	if (st & TVG_ST_TREE_STALE)
		return tvg_fail(ctx, TVG_E_STATE, "%s: the kept tree does not fit the particles", phase);
	if (st & TVG_ST_OFF_GRID)
		return tvg_fail(ctx, TVG_E_BADINPUT, "%s: a particle lies more than half a domain size "
		                "outside the domain of the last decomposition (the group form's integer grid); "
		                "a domain update is due", phase);
	if (st & TVG_ST_TIMESTEP)
		return tvg_fail(ctx, TVG_E_BADINPUT, "%s: time step below the integer timeline's resolution "
		                "or not finite (timestep.c:219-222)", phase);
	return tvg_fail(ctx, TVG_E_CUDA, "%s: device status 0x%x", phase, st);
}

static int dalloc(tvg_context *ctx, void **p, size_t bytes)
{
	if (bytes == 0) bytes = 16;
	cudaError_t e = cudaMalloc(p, bytes);
	if (e != cudaSuccess) {
		cudaGetLastError();
		return tvg_fail(ctx, TVG_E_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
	}
	return TVG_OK;
}

extern "C" const char *tvg_version(void) { return TVG_VERSION; }

extern "C" const char *tvg_last_error(const tvg_context *ctx)
{
	return ctx ? ctx->err : "no context";
}

extern "C" int tvg_init(int device, const tvg_config *cfg, tvg_context **out)
{
	if (!out || !cfg) return TVG_E_BADINPUT;
	*out = nullptr;
	if (cfg->float_bytes != 4 && cfg->float_bytes != 8) return TVG_E_BADINPUT;
	// node and particle indices are 32-bit: the uncollapsed-node capacity
	// 2 max_particles + 4096 must stay below 2^31
	if (cfg->max_particles <= 0 || cfg->max_particles > TVG_MAX_PARTICLES) return TVG_E_BADINPUT;
	if (cfg->periodic && !(cfg->boxsize > 0)) return TVG_E_BADINPUT;
	if (cfg->vector_size <= 0 || cfg->vector_size > 64) return TVG_E_BADINPUT;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
		cudaGetLastError();
		return TVG_E_CUDA;
	}
	tvg_context *ctx = new tvg_context();
	ctx->device = device;
	ctx->cfg = *cfg;
	ctx->cap = cfg->max_particles;
	*out = ctx;
	TVG_CUDA(ctx, cudaSetDevice(device));
	TVG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
	for (int i = 0; i < 16; i++) TVG_CUDA(ctx, cudaEventCreate(&ctx->ev[i]));
	const int64_t cap = ctx->cap;
	for (int s = 0; s < FS_NFIELDS; s++) {
		size_t b = tvg_field_bytes(ctx, s) * (size_t) cap;
		TVG_CHECK(dalloc(ctx, &ctx->f[s], b));
		TVG_CHECK(dalloc(ctx, &ctx->falt[s], b));
		TVG_CUDA(ctx, cudaMemset(ctx->f[s], 0, b));
	}
	TVG_CHECK(dalloc(ctx, (void **) &ctx->key_hi, 8 * cap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->key_lo, 8 * cap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->key_tmp, 8 * cap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->perm, 4 * cap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->perm_tmp, 4 * cap));
	const int64_t ntiles = (cap + 4095) / 4096;
	TVG_CHECK(dalloc(ctx, (void **) &ctx->sort_hist, 4 * 256 * (ntiles + 1)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->sort_off, 4 * 256 * (ntiles + 1)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->digit_count, 4 * 8 * 256));
	ctx->scan_tmp_bytes = 8 * ((cap * 3) / 512 + 4096);
	TVG_CHECK(dalloc(ctx, &ctx->scan_tmp, ctx->scan_tmp_bytes));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->status, sizeof(int)));
	TVG_CUDA(ctx, cudaMemset(ctx->status, 0, sizeof(int)));
	TVG_CUDA(ctx, cudaMallocHost((void **) &ctx->h_status, sizeof(int)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->d_top, sizeof(tvg_topnode) * TVG_MAX_TOP));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->top_first, 4 * TVG_MAX_TOP));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->top_count, 4 * TVG_MAX_TOP));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->lvl, cap + 64));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->lvl_min64, cap / 64 + 64));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->ncnt, 4 * (cap + 1)));
	// uncollapsed nodes: at most ~2 per particle for non-degenerate inputs;
	// the build checks the bound and fails with TVG_E_TREE_FULL otherwise
	ctx->ucap = 2 * cap + 4096;
	TVG_CHECK(dalloc(ctx, (void **) &ctx->u_start, 4 * ctx->ucap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->u_count, 4 * ctx->ucap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->u_endu, 4 * ctx->ucap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->u_diff, 4 * (ctx->ucap + 1)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->u_final, 4 * (ctx->ucap + 1)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->u_level, ctx->ucap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->u_flag, ctx->ucap));
	ctx->tcap = cap + 2 * TVG_MAX_TOP + 4096;
	size_t node_bytes = 16 + 10 * tvg_fsize(ctx);
	TVG_CHECK(dalloc(ctx, &ctx->tree, node_bytes * ctx->tcap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->tree_u, 4 * ctx->tcap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->pref, 8 * 4 * (cap + 1)));
	for (int k = 0; k < 3; k++) TVG_CHECK(dalloc(ctx, (void **) &ctx->ipos[k], 4 * cap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->wtree, sizeof(tvg_wnode) * ctx->tcap));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->big_list, 4 * (ctx->tcap + 1)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->group_first, 4 * (cap / 8 + 1024)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->work_counter, 64));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->counters, 8 * 8));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->dc, sizeof(tvg_devcount)));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->d_toptab, 4 * sizeof(int32_t) * TVG_MAX_TOP));
	TVG_CUDA(ctx, cudaMemset(ctx->d_toptab, 0, 4 * sizeof(int32_t) * TVG_MAX_TOP));
	TVG_CHECK(dalloc(ctx, (void **) &ctx->top_of, 4 * cap));
	TVG_CUDA(ctx, cudaMemset(ctx->dc, 0, sizeof(tvg_devcount)));
	return TVG_OK;
}

// the device counts of the last step into the host mirrors
int tvg_read_counts(tvg_context *ctx)
{
	tvg_devcount h;
	cudaStream_t s = ctx->stream;
	TVG_CUDA(ctx, cudaMemcpyAsync(&h, ctx->dc, sizeof(h), cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	ctx->ntop = h.ntop;
	ctx->nu = h.nu;
	ctx->nnodes = h.nnodes;
	if (ctx->ntop > 0)
		TVG_CUDA(ctx, cudaMemcpyAsync(ctx->h_top, ctx->d_top, sizeof(tvg_topnode) * ctx->ntop,
		                              cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	return TVG_OK;
}

extern "C" void tvg_finalize(tvg_context *ctx)
{
	if (!ctx) return;
	cudaSetDevice(ctx->device);
	if (ctx->stream) cudaStreamSynchronize(ctx->stream);
	tvg_graph_release(ctx);
	for (int s = 0; s < FS_NFIELDS; s++) { cudaFree(ctx->f[s]); cudaFree(ctx->falt[s]); }
	void *bufs[] = { ctx->key_hi, ctx->key_lo, ctx->key_tmp, ctx->perm, ctx->perm_tmp,
	                 ctx->sort_hist, ctx->sort_off, ctx->digit_count, ctx->scan_tmp, ctx->status,
	                 ctx->d_top, ctx->top_first, ctx->top_count, ctx->lvl, ctx->lvl_min64,
	                 ctx->ncnt, ctx->u_start, ctx->u_count, ctx->u_endu, ctx->u_diff,
	                 ctx->u_final, ctx->u_level, ctx->u_flag, ctx->tree, ctx->tree_u, ctx->pref,
	                 ctx->ipos[0], ctx->ipos[1], ctx->ipos[2], ctx->wtree, ctx->group_first,
	                 ctx->work_counter, ctx->counters, ctx->ewald_f[0], ctx->ewald_f[1],
	                 ctx->ewald_f[2], ctx->ewald_f[3], ctx->ewald_raw, ctx->ewald32,
	                 ctx->ewald_ext, ctx->active, ctx->kd_x, ctx->kd_kick, ctx->kd_drift,
	                 ctx->kd_m2k, ctx->kd_m2d, ctx->kd_work, ctx->tl_scratch, ctx->act_flag,
	                 ctx->act_off, ctx->mlp_prm, ctx->mlp_bf16, ctx->ewald_taylor, ctx->dc,
	                 ctx->d_toptab, ctx->top_of, ctx->dd_scratch, ctx->tu_first, ctx->tu_dp,
	                 ctx->tu_big, ctx->big_list, ctx->tune_active, ctx->wquad, ctx->wrange };
	for (void *b : bufs) if (b) cudaFree(b);
	if (ctx->h_status) cudaFreeHost(ctx->h_status);
	for (int i = 0; i < 16; i++) if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
	for (int i = 0; i < 3; i++) if (ctx->xev[i]) cudaEventDestroy(ctx->xev[i]);
	if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
	if (ctx->stream) cudaStreamDestroy(ctx->stream);
	delete ctx;
}

// host field pointer for a slot
void *tvg_host_field(const tvg_particles *p, int slot)
{
	switch (slot) {
	case FS_TYPE: return p->type;
	case FS_TIME_BIN: return p->time_bin;
	case FS_IT_DRIFT: return p->it_drift_pos;
	case FS_IT_KICK: return p->it_kick_pos;
	case FS_ID: return p->id;
	case FS_COST: return p->cost;
	case FS_POS0: case FS_POS1: case FS_POS2: return p->pos[slot - FS_POS0];
	case FS_VEL0: case FS_VEL1: case FS_VEL2: return p->vel[slot - FS_VEL0];
	case FS_ACC0: case FS_ACC1: case FS_ACC2: return p->acc[slot - FS_ACC0];
	case FS_MASS: return p->mass;
	case FS_GACC0: case FS_GACC1: case FS_GACC2: return p->grav_acc[slot - FS_GACC0];
	case FS_LAST_ACC: return p->last_acc_mag;
	case FS_TREE_PARENT: return p->tree_parent;
	case FS_GRAV_POT: return p->grav_pot;
	}
	return nullptr;
}

uint32_t tvg_slot_bit(int slot)
{
	switch (slot) {
	case FS_TYPE: return TVG_F_TYPE;
	case FS_TIME_BIN: return TVG_F_TIME_BIN;
	case FS_IT_DRIFT: return TVG_F_IT_DRIFT;
	case FS_IT_KICK: return TVG_F_IT_KICK;
	case FS_ID: return TVG_F_ID;
	case FS_COST: return TVG_F_COST;
	case FS_POS0: case FS_POS1: case FS_POS2: return TVG_F_POS;
	case FS_VEL0: case FS_VEL1: case FS_VEL2: return TVG_F_VEL;
	case FS_ACC0: case FS_ACC1: case FS_ACC2: return TVG_F_ACC;
	case FS_MASS: return TVG_F_MASS;
	case FS_GACC0: case FS_GACC1: case FS_GACC2: return TVG_F_GRAV_ACC;
	case FS_LAST_ACC: return TVG_F_LAST_ACC;
	case FS_TREE_PARENT: return TVG_F_TREE_PARENT;
	case FS_GRAV_POT: return TVG_F_GRAV_POT;
	}
	return 0;
}

__global__ void k_split_keys(int64_t n, const uint64_t *key16, uint64_t *hi, uint64_t *lo)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) { lo[i] = key16[2 * i]; hi[i] = key16[2 * i + 1]; }
}

__global__ void k_join_keys(int64_t n, const uint64_t *hi, const uint64_t *lo, uint64_t *key16)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) { key16[2 * i] = lo[i]; key16[2 * i + 1] = hi[i]; }
}

extern "C" int tvg_upload(tvg_context *ctx, int64_t n, const tvg_particles *p, uint32_t fields)
{
	if (!ctx || !p) return TVG_E_BADINPUT;
	if (n < 0 || n > ctx->cap) return tvg_fail(ctx, TVG_E_BADINPUT, "n=%lld > capacity %lld",
	                                           (long long) n, (long long) ctx->cap);
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	ctx->n = n;
	for (int s = 0; s < FS_NFIELDS; s++) {
		if (!(fields & tvg_slot_bit(s))) continue;
		const void *h = tvg_host_field(p, s);
		if (!h) return tvg_fail(ctx, TVG_E_BADINPUT, "upload: field slot %d is NULL", s);
		TVG_CUDA(ctx, cudaMemcpyAsync(ctx->f[s], h, tvg_field_bytes(ctx, s) * n,
		                              cudaMemcpyHostToDevice, ctx->stream));
	}
	if (fields & TVG_F_KEY) {
		if (!p->key) return tvg_fail(ctx, TVG_E_BADINPUT, "upload: key is NULL");
		// stage the 16-byte keys in the prefix-sum buffer (32 * (cap + 1) bytes)
		uint64_t *k16 = (uint64_t *) ctx->pref;
		TVG_CUDA(ctx, cudaMemcpyAsync(k16, p->key, 16 * n, cudaMemcpyHostToDevice, ctx->stream));
		k_split_keys<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, ctx->stream>>>(n, k16, ctx->key_hi, ctx->key_lo);
	}
	if (fields & TVG_F_POS) {
		ctx->sorted = false;
		ctx->have_tree = false;
		ctx->have_top = false;
		ctx->use_active = false;
	}
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	return TVG_OK;
}

extern "C" int tvg_download(tvg_context *ctx, tvg_particles *p, uint32_t fields)
{
	if (!ctx || !p) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	const int64_t n = ctx->n;
	for (int s = 0; s < FS_NFIELDS; s++) {
		if (!(fields & tvg_slot_bit(s))) continue;
		void *h = tvg_host_field(p, s);
		if (!h) return tvg_fail(ctx, TVG_E_BADINPUT, "download: field slot %d is NULL", s);
		TVG_CUDA(ctx, cudaMemcpyAsync(h, ctx->f[s], tvg_field_bytes(ctx, s) * n,
		                              cudaMemcpyDeviceToHost, ctx->stream));
	}
	if (fields & TVG_F_KEY) {
		if (!p->key) return tvg_fail(ctx, TVG_E_BADINPUT, "download: key is NULL");
		uint64_t *k16 = (uint64_t *) ctx->pref;   // 32*(cap+1) bytes >= 16*n
		k_join_keys<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, ctx->stream>>>(n, ctx->key_hi, ctx->key_lo, k16);
		TVG_CUDA(ctx, cudaMemcpyAsync(p->key, k16, 16 * n, cudaMemcpyDeviceToHost, ctx->stream));
	}
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	return TVG_OK;
}

extern "C" int tvg_set_domain(tvg_context *ctx, const double origin[3], double size)
{
	if (!ctx || !origin || !(size > 0)) return TVG_E_BADINPUT;
	for (int k = 0; k < 3; k++) ctx->origin[k] = origin[k];
	ctx->dsize = size;
	ctx->have_domain = true;
	return TVG_OK;
}

extern "C" int tvg_peano_keys(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_domain) return tvg_fail(ctx, TVG_E_STATE, "peano_keys: domain not set");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_keys(ctx, false));
	ctx->keys_std = true;
	return tvg_sync_status(ctx, "peano_keys");
}

extern "C" int tvg_reverse_keys(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_domain) return tvg_fail(ctx, TVG_E_STATE, "reverse_keys: domain not set");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_keys(ctx, true));
	ctx->keys_std = false;
	return tvg_sync_status(ctx, "reverse_keys");
}

extern "C" int tvg_sort_particles(tvg_context *ctx, uint32_t *perm)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->keys_std) return tvg_fail(ctx, TVG_E_STATE, "sort: standard keys not computed");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_sort(ctx, perm));
	ctx->sorted = true;
	ctx->use_active = false;
	ctx->have_tree = false;
	return tvg_sync_status(ctx, "sort");
}

extern "C" int tvg_top_nodes(tvg_context *ctx, int32_t *ntop)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->sorted || !ctx->keys_std)
		return tvg_fail(ctx, TVG_E_STATE, "top_nodes: particles not sorted by standard keys");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_top_nodes(ctx));
	ctx->have_top = true;
	if (ntop) *ntop = ctx->ntop;
	return TVG_OK;
}

extern "C" int tvg_tree_build(tvg_context *ctx, uint32_t flags)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_top) return tvg_fail(ctx, TVG_E_STATE, "tree_build: no top nodes");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_tree_build(ctx, flags));
	ctx->have_tree = true;
	ctx->have_walktree = false;
	return TVG_OK;
}

extern "C" int tvg_download_tree(tvg_context *ctx, void *tree, int64_t tree_cap, int64_t *nnodes,
                                 tvg_topnode *top, int32_t top_cap, int32_t *ntop)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_tree) return tvg_fail(ctx, TVG_E_STATE, "download_tree: no tree");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (tree) TVG_CHECK(tvg_impl_download_tree(ctx, tree, tree_cap, nnodes));
	else if (nnodes) *nnodes = ctx->nnodes;
	if (top) {
		if (top_cap < ctx->ntop) return tvg_fail(ctx, TVG_E_BADINPUT, "top_cap too small");
		TVG_CUDA(ctx, cudaMemcpy(top, ctx->d_top, sizeof(tvg_topnode) * ctx->ntop,
		                         cudaMemcpyDeviceToHost));
	}
	if (ntop) *ntop = ctx->ntop;
	return TVG_OK;
}

extern "C" int tvg_ewald_init(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->cfg.periodic) return tvg_fail(ctx, TVG_E_STATE, "ewald_init: not periodic");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_ewald_init(ctx));
	ctx->have_ewald = true;
	return TVG_OK;
}

extern "C" int tvg_download_ewald_table(tvg_context *ctx, void *fx, void *fy, void *fz, void *fp);

extern "C" int tvg_walk(tvg_context *ctx, int32_t form, int32_t use_bh, uint32_t parts,
                        int32_t ewald_kind)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_tree) return tvg_fail(ctx, TVG_E_STATE, "walk: no tree");
	if ((parts & TVG_WALK_EWALD) && !ctx->cfg.periodic)
		return tvg_fail(ctx, TVG_E_STATE, "walk: Ewald part needs a periodic box");
	if ((parts & TVG_WALK_EWALD) && !ctx->have_ewald)
		return tvg_fail(ctx, TVG_E_STATE, "walk: Ewald table not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (form == TVG_FORM_PLAIN) {
		if (ewald_kind != TVG_EWALD_TABLE)
			return tvg_fail(ctx, TVG_E_BADINPUT, "plain form uses the Ewald table");
		TVG_CHECK(tvg_impl_walk_plain(ctx, use_bh, parts));
	} else if (form == TVG_FORM_GROUP) {
		TVG_CHECK(tvg_impl_walk_group(ctx, use_bh, parts, ewald_kind));
	} else {
		return tvg_fail(ctx, TVG_E_BADINPUT, "unknown form %d", form);
	}
	return tvg_sync_status(ctx, "walk");
}

extern "C" int tvg_save_last_accel(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_save_last_accel(ctx));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	return TVG_OK;
}

extern "C" int tvg_zero_accel(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CHECK(tvg_impl_zero_accel(ctx));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	return TVG_OK;
}

extern "C" int tvg_phase_times(tvg_context *ctx, double *ms, int32_t n)
{
	if (!ctx || !ms) return TVG_E_BADINPUT;
	for (int i = 0; i < n && i < 8; i++) ms[i] = ctx->phase_ms[i];
	return TVG_OK;
}

extern "C" int tvg_walk_counters(tvg_context *ctx, double *g, double *e)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (g) *g = ctx->last_counts[0];
	if (e) *e = ctx->last_counts[1];
	return TVG_OK;
}

extern "C" int tvg_walk_quad_interactions(tvg_context *ctx, double *q)
{
	if (!ctx || !q) return TVG_E_BADINPUT;
	*q = ctx->last_counts[2];
	return TVG_OK;
}

__global__ void k_ffma_peak(float *out, int iters, float a, float b)
{
	// 8 independent FMA chains per thread keep every FP32 lane busy
	float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5,
	      x6 = x0 + 6, x7 = x0 + 7;
	for (int i = 0; i < iters; i++) {
#pragma unroll 16
		for (int j = 0; j < 16; j++) {
			x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
			x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
		}
	}
	const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
	if (s == 1234.5f) out[blockIdx.x] = s;     // keeps the chains alive
}

extern "C" int tvg_fp32_peak(tvg_context *ctx, double ms_target, double *tflops)
{
	if (!ctx || !tflops) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	int nsm = 0;
	TVG_CUDA(ctx, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
	const int blocks = nsm * 8, threads = 256;
	float *out = (float *) ctx->scan_tmp;
	int iters = 256;
	double best = 0;
	int measured = 0;
	for (int rep = 0; rep < 40 && measured < 3; rep++) {
		TVG_CUDA(ctx, cudaEventRecord(ctx->ev[14], ctx->stream));
		k_ffma_peak<<<TVG_CNT(ctx, blocks), threads, 0, ctx->stream>>>(out, iters, 0.999999f, 1e-7f);
		TVG_CUDA(ctx, cudaGetLastError());
		TVG_CUDA(ctx, cudaEventRecord(ctx->ev[15], ctx->stream));
		TVG_CUDA(ctx, cudaEventSynchronize(ctx->ev[15]));
		float ms = 0;
		TVG_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[14], ctx->ev[15]));
		const double flop = 2.0 * 8 * 16 * (double) iters * blocks * threads;
		if (ms > 0.5 * ms_target) {
			best = fmax(best, flop / (ms * 1e-3) / 1e12);
			measured++;
		} else {
			iters = (int) fmin(iters * 2.0, 1 << 26);
		}
	}
	*tflops = best;
	return TVG_OK;
}

extern "C" int tvg_set_opening(tvg_context *ctx, double open_bh, double open_rel)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!(open_bh > 0) || !(open_rel > 0))
		return tvg_fail(ctx, TVG_E_BADINPUT, "set_opening: parameters must be > 0");
	ctx->cfg.open_bh = open_bh;
	ctx->cfg.open_rel = open_rel;
	return TVG_OK;
}

extern "C" int tvg_set_ewald_opening(tvg_context *ctx, double rel_alpha, double bh_factor)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!(rel_alpha > 0) || !(bh_factor > 0))
		return tvg_fail(ctx, TVG_E_BADINPUT, "set_ewald_opening: parameters must be > 0");
	ctx->ewald_open_rel = rel_alpha;
	ctx->ewald_open_bh = bh_factor;
	return TVG_OK;
}

extern "C" int tvg_set_walk_limit(tvg_context *ctx, int64_t max_iterations)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (max_iterations < 1 || max_iterations > 0x7FFFFFFF)
		return tvg_fail(ctx, TVG_E_BADINPUT, "set_walk_limit: %lld outside 1 .. 2^31 - 1",
		                (long long) max_iterations);
	ctx->walk_limit = (int32_t) max_iterations;
	return TVG_OK;
}

extern "C" int tvg_set_active(tvg_context *ctx, const int32_t *list, int64_t n_active)
{
	if (!ctx) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (!list) {
		ctx->use_active = false;
		ctx->n_active = ctx->n;
		return TVG_OK;
	}
	if (n_active < 0 || n_active > ctx->n) return tvg_fail(ctx, TVG_E_BADINPUT, "n_active out of range");
	if (!ctx->active) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->active, 4 * (size_t) ctx->cap));
	if (!ctx->act_flag) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->act_flag, 4 * (size_t) ctx->cap));
	if (!ctx->act_off) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->act_off, 4 * (size_t) ctx->cap));
	TVG_CUDA(ctx, cudaMemcpyAsync(ctx->active, list, 4 * (size_t) n_active, cudaMemcpyHostToDevice,
	                              ctx->stream));
	// the walks read the list's length on the device
	TVG_CUDA(ctx, cudaMemcpyAsync(&ctx->dc->n_active, &n_active, 8, cudaMemcpyHostToDevice, ctx->stream));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	ctx->use_active = true;
	ctx->n_active = n_active;
	return TVG_OK;
}

extern "C" int tvg_launch_count(tvg_context *ctx, int64_t *count)
{
	if (!ctx || !count) return TVG_E_BADINPUT;
	*count = ctx->launches;
	return TVG_OK;
}

extern "C" int tvg_host_alloc(size_t bytes, void **ptr)
{
	if (!ptr) return TVG_E_BADINPUT;
	cudaError_t e = cudaMallocHost(ptr, bytes ? bytes : 16);
	if (e != cudaSuccess) { cudaGetLastError(); *ptr = nullptr; return TVG_E_NOMEM; }
	return TVG_OK;
}

extern "C" int tvg_host_register(void *ptr, size_t bytes)
{
	if (!ptr || !bytes) return TVG_E_BADINPUT;
	const cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
	if (e == cudaSuccess) return TVG_OK;
	cudaGetLastError();
	return e == cudaErrorHostMemoryAlreadyRegistered ? TVG_E_STATE : TVG_E_CUDA;
}

extern "C" int tvg_host_unregister(void *ptr)
{
	if (!ptr) return TVG_E_BADINPUT;
	const cudaError_t e = cudaHostUnregister(ptr);
	if (e == cudaSuccess) return TVG_OK;
	cudaGetLastError();
	return e == cudaErrorHostMemoryNotRegistered ? TVG_E_STATE : TVG_E_CUDA;
}

extern "C" int tvg_host_free(void *ptr)
{
	return cudaFreeHost(ptr) == cudaSuccess ? TVG_OK : TVG_E_CUDA;
}

extern "C" int tvg_timer(tvg_context *ctx, int32_t stop, double *ms)
{
	if (!ctx) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (!stop) {
		TVG_CUDA(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
		return TVG_OK;
	}
	TVG_CUDA(ctx, cudaEventRecord(ctx->ev[7], ctx->stream));
	TVG_CUDA(ctx, cudaEventSynchronize(ctx->ev[7]));
	float f = 0;
	TVG_CUDA(ctx, cudaEventElapsedTime(&f, ctx->ev[6], ctx->ev[7]));
	if (ms) *ms = f;
	return TVG_OK;
}
