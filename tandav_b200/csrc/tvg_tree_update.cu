// tvg_tree_update.cu -- the reference's tree updates between rebuilds.
//
// Time_For_Domain_Update (src/signal.c:85-116) decides when the particles
// are decomposed, sorted and given a new tree: at a sync point, or once the
// active particles of the steps since the last decomposition exceed
// DOMAIN_UPDATE_PARAM * N. In between, the tree is kept: every kick adds the
// particles' momentum change to the nodes above them
// (Gravity_Tree_Update_Kicks, tree_update.c:12-54, from kick.c:31-32,61-62),
// every drift moves the kicked nodes (Gravity_Tree_Update_Drift,
// tree_update.c:62-101, from drift.c:41-42), and the force walks run on that
// tree (accel.c:53). A context enters this mode with its first
// tvg_time_for_domain_update call; until then every force computation
// rebuilds.
//
// Kernels (the arithmetic in tvg_tree_update.cuh): the first particle of
// every node, the node kicks, the top-node kicks, the node and top-node
// drifts. A node's kick is a serial sum over its active particles in slot
// order (the reference's order); a node with more than TU_WARP_MIN of them,
// and every top node, is summed by a warp: the lanes divide a chunk of dp by
// the node mass in parallel, and lanes 0..2 add the quotients in slot order,
// one component each, so every partial sum is the serial loop's. (One
// thread per top node summed 262k particles a node in a full step at 256^3:
// ~290 ms for the kick.) Roofline: a kick reads each active particle's dp
// once per tree level above it; a drift reads and writes the 48 B (FP32) node
// records.
#include "tvg_internal.cuh"
#include "tvg_tree_update.cuh"

template <typename F>
__global__ void k_node_first(const tvg_devcount *__restrict__ dc, int64_t tcap,
                             const TuNode<F> *__restrict__ tree, int32_t *__restrict__ first)
{
	const int64_t nn = dc->nnodes < tcap ? dc->nnodes : tcap;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nn; i += (int64_t) gridDim.x * blockDim.x)
		first[i] = tu_node_first(tree, nn, i);
}

// nodes with more active particles than this are left to a warp each
#define TU_WARP_MIN 128
// slots a warp divides per round, then adds in order; a row of quotients
// per component, padded so that the three adding lanes use different banks
#define TU_CHUNK 128
#define TU_QROW (TU_CHUNK + 1)
#define TU_WARPS 4

template <typename F>
__global__ void k_kick_nodes(const tvg_devcount *__restrict__ dc, int64_t tcap, TuNode<F> *tree,
                             const int32_t *__restrict__ first, const int32_t *__restrict__ act_off, int64_t n,
                             int64_t na, const F *__restrict__ dp0, const F *__restrict__ dp1,
                             const F *__restrict__ dp2, int32_t *big, int *status)
{
	const int64_t nn = dc->nnodes < tcap ? dc->nnodes : tcap;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nn; i += (int64_t) gridDim.x * blockDim.x) {
		const int64_t lo = first[i];
		if (lo < 0) continue;
		const int64_t hi = lo + tree[i].Npart;
		if (tree[i].Npart <= 0 || hi > n) {
			atomicOr(status, TVG_ST_TREE_STALE);
			continue;
		}
		int64_t a0, a1;
		tu_active_slots(act_off, n, na, lo, hi, &a0, &a1);
		if (a1 - a0 > TU_WARP_MIN) big[1 + atomicAdd(&big[0], 1)] = (int32_t) i;   // each node once: < tcap
		else tu_kick_node(tree[i], dp0, dp1, dp2, a0, a1);
	}
}

// Adds dp_c[k] / m for the slots k in [a0, a1), in slot order, to d by one
// warp: lane c < 3 carries component c (the result is in lane c). A chunk's
// quotients are formed by all lanes into q; the next chunk's dp is loaded
// into registers while lanes 0..2 add this one's, so that its memory latency
// overlaps the serial additions. add(d, quotient) is the node's or the top
// node's rounding of a step.
template <typename F, typename A, typename Add>
__device__ __forceinline__ A tu_warp_sum(const F *__restrict__ dp0, const F *__restrict__ dp1,
                                         const F *__restrict__ dp2, int64_t a0, int64_t a1, F m, A d,
                                         F (*q)[TU_QROW], Add add)
{
	constexpr int PER = TU_CHUNK / 32;
	const int lane = threadIdx.x & 31;
	F r0[PER], r1[PER], r2[PER];
	int cnt = (int) (a1 - a0 < TU_CHUNK ? a1 - a0 : TU_CHUNK);
#pragma unroll
	for (int u = 0; u < PER; u++) {
		const int j = lane + 32 * u;
		if (j < cnt) {
			r0[u] = dp0[a0 + j];
			r1[u] = dp1[a0 + j];
			r2[u] = dp2[a0 + j];
		}
	}
	for (int64_t b = a0; b < a1; b += TU_CHUNK) {
		cnt = (int) (a1 - b < TU_CHUNK ? a1 - b : TU_CHUNK);
#pragma unroll
		for (int u = 0; u < PER; u++) {
			const int j = lane + 32 * u;
			if (j < cnt) {
				q[0][j] = r0[u] / m;
				q[1][j] = r1[u] / m;
				q[2][j] = r2[u] / m;
			}
		}
		__syncwarp();
		const int64_t nb = b + TU_CHUNK;
		const int ncnt = (int) (a1 - nb < TU_CHUNK ? a1 - nb : TU_CHUNK);   // <= 0 after the last chunk
#pragma unroll
		for (int u = 0; u < PER; u++) {
			const int j = lane + 32 * u;
			if (j < ncnt) {
				r0[u] = dp0[nb + j];
				r1[u] = dp1[nb + j];
				r2[u] = dp2[nb + j];
			}
		}
		if (lane < 3) {
#pragma unroll 8
			for (int j = 0; j < cnt; j++) d = add(d, q[lane][j]);
		}
		__syncwarp();
	}
	return d;
}

// tu_kick_node by one warp
template <typename F>
__device__ void tu_kick_node_warp(TuNode<F> &nd, const F *__restrict__ dp0, const F *__restrict__ dp1,
                                  const F *__restrict__ dp2, int64_t a0, int64_t a1, F (*q)[TU_QROW])
{
	const int lane = threadIdx.x & 31;
	F d = lane < 3 ? nd.Dp[lane] : (F) 0;
	d = tu_warp_sum(dp0, dp1, dp2, a0, a1, nd.Mass, d, q, [](F s, F x) { return s + x; });
	if (lane < 3) nd.Dp[lane] = d;
	if (lane == 0) nd.Bitfield |= TVG_NODE_UPDATED;
	__syncwarp();
}

template <typename F>
__global__ void __launch_bounds__(TU_WARPS * 32) k_kick_big(TuNode<F> *tree, const int32_t *__restrict__ first,
                                                          const int32_t *__restrict__ act_off, int64_t n, int64_t na,
                                                          const F *__restrict__ dp0, const F *__restrict__ dp1,
                                                          const F *__restrict__ dp2, const int32_t *__restrict__ big)
{
	__shared__ F q[TU_WARPS][3][TU_QROW];
	const int w = threadIdx.x >> 5;
	const int nbig = big[0];
	for (int k = blockIdx.x * TU_WARPS + w; k < nbig; k += gridDim.x * TU_WARPS) {
		const int32_t i = big[1 + k];
		const int64_t lo = first[i], hi = lo + tree[i].Npart;    // checked by k_kick_nodes
		int64_t a0, a1;
		tu_active_slots(act_off, n, na, lo, hi, &a0, &a1);
		tu_kick_node_warp(tree[i], dp0, dp1, dp2, a0, a1, q[w]);
	}
}

// tu_kick_top by one warp per top node
template <typename F>
__global__ void __launch_bounds__(TU_WARPS * 32) k_kick_top(const tvg_devcount *__restrict__ dc, tvg_topnode *top,
                                                          const int32_t *__restrict__ act_off, int64_t n, int64_t na,
                                                          const F *__restrict__ dp0, const F *__restrict__ dp1,
                                                          const F *__restrict__ dp2, int *status)
{
	__shared__ F q[TU_WARPS][3][TU_QROW];
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int ntop = dc->ntop < TVG_MAX_TOP ? dc->ntop : TVG_MAX_TOP;
	for (int t = blockIdx.x * TU_WARPS + w; t < ntop; t += gridDim.x * TU_WARPS) {
		const int64_t lo = top[t].first_part, hi = lo + top[t].npart;
		if (lo < 0 || top[t].npart < 0 || hi > n) {
			if (lane == 0) atomicOr(status, TVG_ST_TREE_STALE);
			continue;
		}
		int64_t a0, a1;
		tu_active_slots(act_off, n, na, lo, hi, &a0, &a1);
		if (a0 >= a1) continue;
		float d = lane < 3 ? top[t].dp[lane] : 0.f;
		d = tu_warp_sum(dp0, dp1, dp2, a0, a1, (F) top[t].mass, d, q[w],
		                [](float s, F x) { return (float) ((F) s + x); });
		if (lane < 3) top[t].dp[lane] = d;
		if (lane == 0 && top[t].level > 0) top[t].level = -top[t].level;
		__syncwarp();
	}
}

template <typename F>
__global__ void k_drift_nodes(const tvg_devcount *__restrict__ dc, int64_t tcap, TuNode<F> *tree, double dt)
{
	const int64_t nn = dc->nnodes < tcap ? dc->nnodes : tcap;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nn; i += (int64_t) gridDim.x * blockDim.x)
		tu_drift_node(tree[i], dt);
}

__global__ void k_drift_top(const tvg_devcount *__restrict__ dc, tvg_topnode *top, double dt)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= dc->ntop || t >= TVG_MAX_TOP) return;
	tu_drift_top(top[t], dt);
}

// flag[active[k]] = 1 (indices outside [0, n) are reported, not written)
__global__ void k_flag_list(int64_t na, const int32_t *__restrict__ active, int64_t n, int32_t *flag, int *status)
{
	const int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (k >= na) return;
	const int32_t i = active[k];
	if (i < 0 || i >= n) {
		atomicOr(status, TVG_ST_TREE_STALE);
		return;
	}
	flag[i] = 1;
}

__global__ void k_fill_i32(int64_t n, int32_t v, int32_t *a)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) a[i] = v;
}

static int alloc_once(tvg_context *ctx, void **p, size_t bytes)
{
	if (*p) return TVG_OK;
	if (cudaMalloc(p, bytes) != cudaSuccess) {
		cudaGetLastError();
		*p = nullptr;
		return tvg_fail(ctx, TVG_E_NOMEM, "tree update: cannot allocate %zu bytes", bytes);
	}
	return TVG_OK;
}

bool tvg_tree_update_due(const tvg_context *ctx)
{
	return ctx->tree_updates && !ctx->domain_update;
}

int tvg_tree_update_check(tvg_context *ctx, const char *what)
{
	if (!ctx->have_tree || !ctx->have_top)
		return tvg_fail(ctx, TVG_E_STATE, "%s: no tree to update (the tree of the last domain update "
		                "is kept until the next one)", what);
	return TVG_OK;
}

int tvg_impl_active_slots(tvg_context *ctx, int64_t *na_out)
{
	const int64_t n = ctx->n, cap = ctx->cap;
	cudaStream_t s = ctx->stream;
	TVG_CHECK(alloc_once(ctx, (void **) &ctx->act_flag, 4 * (size_t) cap));
	TVG_CHECK(alloc_once(ctx, (void **) &ctx->act_off, 4 * (size_t) cap));
	const int64_t na = ctx->use_active ? ctx->n_active : n;
	if (ctx->use_active) {
		TVG_CUDA(ctx, cudaMemsetAsync(ctx->act_flag, 0, 4 * (size_t) n, s));
		if (na > 0)
			k_flag_list<<<TVG_CNT(ctx, tvg_blocks(na, 256)), 256, 0, s>>>(na, ctx->active, n, ctx->act_flag,
			                                                              ctx->status);
	} else {
		k_fill_i32<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, 1, ctx->act_flag);
	}
	TVG_CUDA(ctx, cudaGetLastError());
	int64_t total = 0;
	TVG_CHECK(tvg_device_scan_i32(ctx, ctx->act_flag, ctx->act_off, n, &total));
	TVG_CHECK(tvg_sync_status(ctx, "tree update: active list"));
	if (total != na)
		return tvg_fail(ctx, TVG_E_BADINPUT, "tree update: the active list repeats particles (%lld of %lld distinct)",
		                (long long) total, (long long) na);
	*na_out = na;
	return TVG_OK;
}

template <typename F>
static int tree_kick_typed(tvg_context *ctx, int64_t na, const F *dp)
{
	const int64_t n = ctx->n, cap = ctx->cap, tcap = ctx->tcap;
	cudaStream_t s = ctx->stream;
	TVG_CHECK(alloc_once(ctx, (void **) &ctx->tu_first, 4 * (size_t) tcap));
	TVG_CHECK(alloc_once(ctx, (void **) &ctx->tu_big, 4 * ((size_t) tcap + 1)));
	TuNode<F> *tree = (TuNode<F> *) ctx->tree;
	const int grid = (int) (tvg_blocks(tcap, 256) < 148 * 16 ? tvg_blocks(tcap, 256) : 148 * 16);
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->tu_big, 0, 4, s));
	k_node_first<F><<<TVG_CNT(ctx, grid), 256, 0, s>>>(ctx->dc, tcap, tree, ctx->tu_first);
	k_kick_nodes<F><<<TVG_CNT(ctx, grid), 256, 0, s>>>(ctx->dc, tcap, tree, ctx->tu_first, ctx->act_off, n, na,
	                                                   dp, dp + cap, dp + 2 * cap, ctx->tu_big, ctx->status);
	k_kick_big<F><<<TVG_CNT(ctx, 148 * 8), TU_WARPS * 32, 0, s>>>(tree, ctx->tu_first, ctx->act_off, n, na, dp,
	                                                              dp + cap, dp + 2 * cap, ctx->tu_big);
	k_kick_top<F><<<TVG_CNT(ctx, TVG_MAX_TOP / TU_WARPS), TU_WARPS * 32, 0, s>>>(
	    ctx->dc, ctx->d_top, ctx->act_off, n, na, dp, dp + cap, dp + 2 * cap, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	return tvg_sync_status(ctx, "tree update: kicks");
}

int tvg_impl_tree_kick(tvg_context *ctx, int64_t na)
{
	if (ctx->cfg.float_bytes == 4) return tree_kick_typed<float>(ctx, na, (const float *) ctx->tu_dp);
	return tree_kick_typed<double>(ctx, na, (const double *) ctx->tu_dp);
}

int tvg_impl_tree_dp_buffer(tvg_context *ctx, void **dp)
{
	TVG_CHECK(alloc_once(ctx, &ctx->tu_dp, 3 * (size_t) ctx->cap * tvg_fsize(ctx)));
	*dp = ctx->tu_dp;
	return TVG_OK;
}

template <typename F>
static int tree_drift_typed(tvg_context *ctx, double dt)
{
	cudaStream_t s = ctx->stream;
	const int64_t tcap = ctx->tcap;
	const int grid = (int) (tvg_blocks(tcap, 256) < 148 * 16 ? tvg_blocks(tcap, 256) : 148 * 16);
	k_drift_nodes<F><<<TVG_CNT(ctx, grid), 256, 0, s>>>(ctx->dc, tcap, (TuNode<F> *) ctx->tree, dt);
	k_drift_top<<<TVG_CNT(ctx, TVG_MAX_TOP / 128), 128, 0, s>>>(ctx->dc, ctx->d_top, dt);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

int tvg_impl_tree_drift(tvg_context *ctx, double dt)
{
	if (ctx->cfg.float_bytes == 4) return tree_drift_typed<float>(ctx, dt);
	return tree_drift_typed<double>(ctx, dt);
}

extern "C" int tvg_time_for_domain_update(tvg_context *ctx, double domain_update_param, int32_t *domain_update)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!(domain_update_param >= 0)) return tvg_fail(ctx, TVG_E_BADINPUT, "domain_update_param must be >= 0");
	ctx->tree_updates = true;
	// signal.c:89-113 (one rank: the global count is the local one)
	ctx->domain_update = false;
	ctx->npart_updates += ctx->have_timeline ? ctx->tl.state.n_active : ctx->n;
	const double max_updates = domain_update_param * (double) ctx->n;
	const bool sync = ctx->have_timeline && ctx->tl.state.sync_point;
	if (sync || (double) ctx->npart_updates > max_updates) {
		ctx->npart_updates = 0;
		ctx->domain_update = true;
	}
	if (domain_update) *domain_update = ctx->domain_update ? 1 : 0;
	return TVG_OK;
}
