// tvg_tree.cu -- top nodes and the octree, built in parallel from PH-sorted
// keys, bit-exact with Gravity_Tree_Build (src/Gravity/tree_build.c:47-572).
//
// The reference inserts particles one by one (build_subtree) and collapses
// finished branches into bundles of <= VECTOR_SIZE particles
// (collapse_last_branch). Its result has a closed form, which this file
// evaluates with one thread per particle / node:
//
//   l_i   = level of the deepest common cell of sorted particles i-1 and i
//           (leading equal key triplets); at a top node's first particle l
//           is 0, a boundary below every level, whatever the top node's
//           level L (>= 2; all 64 level-2 cells on one target, deeper cells
//           where Domain_Decomposition balances several).
//   nodes = the top cell, and every cell whose parent cell holds >= 2
//           particles. The cells that start at particle i are levels
//           lo_i .. max(l_i, l_{i+1})+1, lo_i = L at a top node's first
//           particle and l_i+1 elsewhere; pre-order = (first particle, level).
//   event = particle e with l_e < l_{e-1}: the reference sees it as a new
//           branch. At e the cell A (level l_e+1, holding e-1) becomes a
//           bundle if it has <= VECTOR_SIZE particles, else the cell B (level
//           l_{e-1}, holding e-1) if B has <= VECTOR_SIZE particles.
//           Nothing else collapses (the last branch of a top node stays).
//   a node survives unless a strict ancestor became a bundle; DNext of an
//           internal node is the distance to the next surviving node after
//           its subtree (or to the terminator), of a bundle/leaf -(first)-1.
// Particles equal to 41 levels ("dumped" by the reference,
// tree_build.c:337-342) are reported as TVG_E_COINCIDENT.
//
// Node centres (Pos) repeat the reference's float arithmetic down the chain
// of ancestors (tree_build.c:542-550). Mass/CoM: bundles, leaves and, in
// exact mode, every node are summed sequentially in particle order in Float
// (tree_build.c:561-572), which reproduces the reference bit for bit; the fast
// mode sums internal nodes in FP64 with one warp per node.
// Roofline: HBM/L2 bound (1 B level + 16 B key per particle, ~O(nodes)).
#include "tvg_internal.cuh"

#define TOP_LEVEL 2         // MIN_LEVEL (domain.c:3): the top level on one target
#define LVL_START 0         // l at a top node's first particle
#define LVL_SMALL 0xFF      // particle of a top node without subtree

template <typename F> struct TNode {
	int32_t DNext;
	uint32_t Bitfield;
	int32_t DUp;
	int32_t Npart;
	F Pos[3];
	F Mass;
	F CoM[3];
	F Dp[3];
};

// ------------------------------------------------------------ top nodes

__global__ void k_top_first(int64_t n, const uint64_t *__restrict__ key_hi, int32_t *first)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	int c = (int) (key_hi[i] >> 58);
	if (i == 0 || (int) (key_hi[i - 1] >> 58) != c) first[c] = (int32_t) i;
}

// one thread: top nodes in descending key order (compare_bunches_by_key,
// domain.c:678-684), centre from the first particle (domain.c:237-246)
template <typename F>
__global__ void k_make_top(int64_t n, const int32_t *first, const F *x, const F *y, const F *z,
                           double ox, double oy, double oz, double size, tvg_topnode *top,
                           int32_t *count, tvg_devcount *dc)
{
	if (threadIdx.x || blockIdx.x) return;
	int nt = 0;
	for (int c = 63; c >= 0; c--) {
		if (first[c] < 0) { count[c] = 0; continue; }
		int64_t e = n;
		for (int d = c + 1; d < 64; d++)
			if (first[d] >= 0) { e = first[d]; break; }
		count[c] = (int32_t) (e - first[c]);
		tvg_topnode t;
		t.key = ((uint64_t) c << 58) | (0xFFFFFFFFFFFFFFFFULL >> 6);
		t.target = -1;
		t.level = TOP_LEVEL;
		t.first_part = first[c];
		t.npart = (int32_t) (e - first[c]);
		int64_t ip = first[c];
		const double sz = size / (double) (1ULL << TOP_LEVEL);
		const double px = (double) x[ip] - ox, py = (double) y[ip] - oy, pz = (double) z[ip] - oz;
		t.pos[0] = (float) __dadd_rn(__dmul_rn(floor(px / sz) + 0.5, sz), ox);
		t.pos[1] = (float) __dadd_rn(__dmul_rn(floor(py / sz) + 0.5, sz), oy);
		t.pos[2] = (float) __dadd_rn(__dmul_rn(floor(pz / sz) + 0.5, sz), oz);
		t.mass = 0;
		for (int k = 0; k < 3; k++) { t.com[k] = 0; t.dp[k] = 0; }
		top[nt++] = t;
	}
	dc->ntop = nt;
}

// top node of every particle: block b takes top nodes b, b + grid, ...
__global__ void k_top_of(const tvg_devcount *__restrict__ dc, const tvg_topnode *__restrict__ top,
                         int32_t *__restrict__ top_of)
{
	const int ntop = dc->ntop;
	for (int t = blockIdx.x; t < ntop; t += gridDim.x) {
		const int64_t f = top[t].first_part, e = f + top[t].npart;
		for (int64_t i = f + threadIdx.x; i < e; i += blockDim.x) top_of[i] = t;
	}
}

int tvg_impl_top_of(tvg_context *ctx)
{
	k_top_of<<<TVG_CNT(ctx, 148 * 4), 256, 0, ctx->stream>>>(ctx->dc, ctx->d_top, ctx->top_of);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

// One target (NTask = 1, or >= 65 tasks on one rank, domain.c:151-156): the
// reference's loop stops at once with every non-empty level-2 cell as a top
// node, which needs no host round trip (the step graph captures it). More
// targets: the cost-balanced refinement of tvg_decompose.cu.
int tvg_impl_top_nodes(tvg_context *ctx)
{
	if (ctx->dd_ntask > 1 && ctx->dd_ntask < 65) return tvg_impl_top_nodes_balanced(ctx);
	const int64_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->top_first, 0xFF, 4 * 64, s));
	k_top_first<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, ctx->key_hi, ctx->top_first);
	if (ctx->cfg.float_bytes == 4)
		k_make_top<float><<<TVG_CNT(ctx, 1), 1, 0, s>>>(n, ctx->top_first, (const float *) ctx->f[FS_POS0],
		                                  (const float *) ctx->f[FS_POS1], (const float *) ctx->f[FS_POS2],
		                                  ctx->origin[0], ctx->origin[1], ctx->origin[2], ctx->dsize,
		                                  ctx->d_top, ctx->top_count, ctx->dc);
	else
		k_make_top<double><<<TVG_CNT(ctx, 1), 1, 0, s>>>(n, ctx->top_first, (const double *) ctx->f[FS_POS0],
		                                   (const double *) ctx->f[FS_POS1], (const double *) ctx->f[FS_POS2],
		                                   ctx->origin[0], ctx->origin[1], ctx->origin[2], ctx->dsize,
		                                   ctx->d_top, ctx->top_count, ctx->dc);
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CHECK(tvg_impl_top_of(ctx));
	if (ctx->capturing) return TVG_OK;
	return tvg_read_counts(ctx);
}

// ----------------------------------------------------- build: levels


__device__ __forceinline__ int lca_level(const uint64_t *hi, const uint64_t *lo, int64_t a, int64_t b)
{
	int l = tvg_clz128(hi[a] ^ hi[b], lo[a] ^ lo[b]) / 3;
	return l > TVG_MAX_LEVEL ? TVG_MAX_LEVEL : l;
}

__global__ void k_levels(int64_t n, const uint64_t *__restrict__ hi, const uint64_t *__restrict__ lo,
                         const tvg_topnode *__restrict__ top, const int32_t *__restrict__ top_of,
                         int vsize, uint8_t *__restrict__ lvl, int32_t *__restrict__ ncnt,
                         uint8_t *__restrict__ lvl_min64, int *status)
{
	__shared__ uint8_t s_min[256 / 32];
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	unsigned my = 0xFF;
	if (i < n) {
		const tvg_topnode &tn = top[top_of[i]];
		const int64_t f = tn.first_part, e = f + tn.npart;
		const bool big = tn.npart > vsize;
		int l, cnt = 0;
		if (i == f) {
			l = LVL_START;
		} else if (!big) {
			l = LVL_SMALL;
		} else {
			l = lca_level(hi, lo, i - 1, i);
			if (l >= TVG_MAX_LEVEL - 1) atomicOr(status, TVG_ST_COINCIDENT);
		}
		if (big) {
			int lnext = (i + 1 < e) ? lca_level(hi, lo, i, i + 1) : -1;
			int lo_l = i == f ? tn.level : l + 1;
			int hi_l = (l > lnext ? l : lnext) + 1;
			cnt = hi_l - lo_l + 1;
		}
		lvl[i] = (uint8_t) l;
		ncnt[i] = cnt;
		my = (unsigned) l;
	}
	// min over each 64-particle block (two warps)
	unsigned wmin = __reduce_min_sync(0xFFFFFFFFu, my);
	const int w = threadIdx.x >> 5;
	if ((threadIdx.x & 31) == 0) s_min[w] = (uint8_t) wmin;
	__syncthreads();
	if (threadIdx.x < blockDim.x / 64) {
		int64_t b = (blockIdx.x * (int64_t) blockDim.x) / 64 + threadIdx.x;
		if (b * 64 < n) {
			uint8_t a = s_min[2 * threadIdx.x], bb = s_min[2 * threadIdx.x + 1];
			lvl_min64[b] = a < bb ? a : bb;
		}
	}
	if (i == n - 1) ncnt[n] = 0;
}

// first j > s with lvl[j] < l, or n
__device__ int64_t next_smaller(const uint8_t *__restrict__ lvl, const uint8_t *__restrict__ m64,
                                int64_t n, int64_t s, int l)
{
	int64_t j = s + 1;
	while (j < n && (j & 63)) {
		if (lvl[j] < l) return j;
		j++;
	}
	if (j >= n) return n;
	int64_t b = j >> 6;
	const int64_t nb = (n + 63) >> 6;
	while (b < nb && m64[b] >= l) b++;
	if (b >= nb) return n;
	j = b << 6;
	while (j < n && lvl[j] >= l) j++;
	return j;
}

// last j < s with lvl[j] < l (exists: a top node's first particle has lvl 1)
__device__ int64_t prev_smaller(const uint8_t *__restrict__ lvl, const uint8_t *__restrict__ m64,
                                int64_t s, int l)
{
	int64_t j = s - 1;
	while (j >= 0 && ((j + 1) & 63)) {
		if (lvl[j] < l) return j;
		j--;
	}
	if (j < 0) return -1;
	int64_t b = j >> 6;
	while (b >= 0 && m64[b] >= l) b--;
	if (b < 0) return -1;
	j = (b << 6) + 63;
	while (lvl[j] >= l) j--;
	return j;
}

enum { UF_COLLAPSED = 1, UF_LEAF = 2, UF_ROOT = 4 };

// every uncollapsed node: range, collapse decision, removal marks
// first level of the nodes that start at particle s (the top node's level at
// its first particle, whose l is LVL_START)
__device__ __forceinline__ int first_level(const uint8_t *__restrict__ lvl,
                                           const tvg_topnode *__restrict__ top,
                                           const int32_t *__restrict__ top_of, int64_t s)
{
	const int ls = lvl[s];
	return ls == LVL_START ? top[top_of[s]].level : ls + 1;
}

__global__ void k_nodes(int64_t n, const uint8_t *__restrict__ lvl, const uint8_t *__restrict__ m64,
                        const int32_t *__restrict__ base, const tvg_topnode *__restrict__ top,
                        const int32_t *__restrict__ top_of, int vsize, int32_t *__restrict__ u_start,
                        uint8_t *__restrict__ u_level, int32_t *__restrict__ u_count,
                        int32_t *__restrict__ u_endu, uint8_t *__restrict__ u_flag,
                        int32_t *__restrict__ u_diff, int64_t ucap, int *status)
{
	const int64_t s = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (s >= n) return;
	const int32_t b0 = base[s], nc = base[s + 1] - b0;
	if (nc == 0) return;
	const bool top_start = lvl[s] == LVL_START;
	const int lo_l = first_level(lvl, top, top_of, s);
	for (int k = 0; k < nc; k++) {
		const int l = lo_l + k;
		const int64_t u = b0 + k;
		const int64_t e = next_smaller(lvl, m64, n, s, l);
		const int32_t cnt = (int32_t) (e - s);
		uint8_t flag = 0;
		if (top_start && k == 0) flag |= UF_ROOT;
		if (cnt == 1) flag |= UF_LEAF;
		if (cnt <= vsize && e < n && cnt > 1) {
			const int le = lvl[e], lp = lvl[e - 1];
			// e is an event: not a top node start and l_e < l_{e-1}
			if (le != LVL_START && le < lp) {
				if (l == le + 1) {
					flag |= UF_COLLAPSED;
				} else if (l == lp) {
					// cell A (level l_e+1 holding e-1) must hold > vsize particles
					int64_t a0 = e - vsize;
					if (a0 < 0) a0 = 0;
					bool a_small = false;
					for (int64_t j = a0; j < e; j++)
						if (lvl[j] <= le) { a_small = true; break; }
					if (!a_small) flag |= UF_COLLAPSED;
				}
			}
		}
		const int32_t endu = base[e];
		if (u >= ucap || endu > ucap) {      // u_diff holds ucap + 1 entries
			atomicOr(status, TVG_ST_TREE_FULL);
			return;
		}
		u_start[u] = (int32_t) s;
		u_level[u] = (uint8_t) l;
		u_count[u] = cnt;
		u_endu[u] = endu;
		u_flag[u] = flag;
		if (flag & UF_COLLAPSED) {
			atomicAdd(&u_diff[u + 1], 1);
			atomicAdd(&u_diff[endu], -1);
		}
	}
}

// survivor flag from the scanned removal marks: surv[u] = (marks(u) == 0),
// for u <= nu (nu from the device, at most ucap)
__global__ void k_survivors(const tvg_devcount *__restrict__ dc, int64_t ucap,
                            const int32_t *__restrict__ excl, int32_t *__restrict__ surv)
{
	const int64_t nu = min(dc->nu, ucap);
	int64_t u = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (u > nu) return;
	surv[u] = (u < nu && excl[u + 1] == 0) ? 1 : 0;
}

// one thread: subtree placement in top-node order (tree_build.c:59-96); the
// placement table for the emission and the node count, on the device
__global__ void k_place_subtrees(tvg_devcount *dc, tvg_topnode *top, const int32_t *__restrict__ base,
                                 const int32_t *__restrict__ F, int vsize, TopTables tp, int64_t ucap,
                                 int64_t tcap, int *status)
{
	if (threadIdx.x || blockIdx.x) return;
	const int ntop = dc->ntop;
	int64_t run = 0;
	for (int t = 0; t < ntop; t++) {
		top[t].target = (int32_t) run;       // also for small top nodes (quirk Q3)
		tp.target[t] = (int32_t) run;
		tp.end[t] = top[t].first_part + top[t].npart;
		tp.nsurv[t] = tp.toff[t] = 0;
		if (top[t].npart > vsize) {
			int64_t f = top[t].first_part, e = f + top[t].npart;
			// base <= nu; past the capacity the build has failed (status set)
			int32_t fs = F[min((int64_t) base[f], ucap)], fe = F[min((int64_t) base[e], ucap)];
			tp.nsurv[t] = fe - fs;
			tp.toff[t] = (int32_t) (run - fs);
			run += (fe - fs) + 1;             // + terminator
		}
	}
	if (run > tcap) atomicOr(status, TVG_ST_TREE_FULL);
	dc->nnodes = run;
}


__device__ __forceinline__ int32_t triplet_at(const uint64_t *hi, const uint64_t *lo, int64_t i, int l)
{
	return tvg_std_triplet(hi[i], lo[i], l);
}

template <typename F>
__global__ void k_emit_nodes(const tvg_devcount *__restrict__ dc, int64_t ucap, int64_t n,
                             const uint8_t *__restrict__ lvl,
                             const uint8_t *__restrict__ m64, const int32_t *__restrict__ base,
                             const int32_t *__restrict__ u_start, const uint8_t *__restrict__ u_level,
                             const int32_t *__restrict__ u_count, const int32_t *__restrict__ u_endu,
                             const uint8_t *__restrict__ u_flag, const int32_t *__restrict__ surv,
                             const int32_t *__restrict__ Fidx, const uint64_t *__restrict__ hi,
                             const uint64_t *__restrict__ lo, const tvg_topnode *__restrict__ top,
                             const int32_t *__restrict__ top_of, TopTables tp,
                             TNode<F> *tree, int32_t *__restrict__ tree_u,
                             int32_t *__restrict__ tree_parent, int64_t tcap, int *status)
{
	const int64_t nu = min(dc->nu, ucap);
	const int64_t u = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (u >= nu || !surv[u]) return;
	const int32_t s = u_start[u];
	const int l = u_level[u];
	const int32_t cnt = u_count[u];
	const uint8_t flag = u_flag[u];
	const int t = top_of[s];
	const int64_t G = (int64_t) tp.toff[t] + Fidx[u];
	if (G < 0 || G >= tcap) { atomicOr(status, TVG_ST_TREE_FULL); return; }
	TNode<F> nd;
	nd.Npart = cnt;
	nd.Bitfield = (uint32_t) l | ((uint32_t) triplet_at(hi, lo, s, l) << 6) | (1u << 9)
	            | ((flag & UF_ROOT) ? (1u << 10) : 0u);
	if (flag & (UF_COLLAPSED | UF_LEAF)) {
		nd.DNext = -s - 1;
	} else {
		const bool at_end = (int64_t) s + cnt >= tp.end[t];
		const int64_t nxt = at_end ? (int64_t) tp.target[t] + tp.nsurv[t]
		                           : (int64_t) tp.toff[t] + Fidx[u_endu[u]];
		nd.DNext = (int32_t) (nxt - G);
	}
	if (flag & UF_ROOT) {
		nd.DUp = t;
	} else {
		int64_t pu;
		if (u > base[s]) {
			pu = u - 1;
		} else {
			const int ls = lvl[s];
			const int64_t p = prev_smaller(lvl, m64, s, ls);
			pu = base[p] + (ls - first_level(lvl, top, top_of, p));
		}
		nd.DUp = (int32_t) (G - ((int64_t) tp.toff[t] + Fidx[pu]));
	}
	for (int k = 0; k < 3; k++) { nd.Pos[k] = 0; nd.CoM[k] = 0; nd.Dp[k] = 0; }
	nd.Mass = 0;
	tree[G] = nd;
	tree_u[G] = (int32_t) u;
	if (flag & (UF_COLLAPSED | UF_LEAF))
		for (int32_t j = s; j < s + cnt; j++) tree_parent[j] = (int32_t) G;
}

// particles of top nodes without subtree point to their top node (-t-1),
// set_tree_parent_pointers, tree_build.c:226-242
__global__ void k_small_parent(int64_t n, const tvg_topnode *__restrict__ top,
                               const int32_t *__restrict__ top_of, int vsize,
                               int32_t *__restrict__ tree_parent)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int t = top_of[i];
	if (top[t].npart <= vsize) tree_parent[i] = -t - 1;
}

// reference arithmetic for a child centre (tree_build.c:542-550)
template <typename F>
__device__ __forceinline__ F child_pos(F ppos, F ppart, double dsize, int l)
{
	const int sign = -1 + 2 * (ppart > ppos);
	const int32_t div = (int32_t) (1u << (l & 31));
	const F size = (F) (dsize / (double) div);
	const F ss = (F) sign * size;
	return (F) __dadd_rn((double) ppos, __dmul_rn((double) ss, 0.5));
}

// centre of node G down its chain of ancestors
template <typename F>
__device__ void node_pos_one(int64_t G, TNode<F> *tree, const int32_t *__restrict__ tree_u,
                             const int32_t *__restrict__ u_start, const F *__restrict__ x,
                             const F *__restrict__ y, const F *__restrict__ z,
                             const tvg_topnode *__restrict__ top, double dsize)
{
	const uint32_t bf = tree[G].Bitfield;
	if (!(bf & (1u << 9))) return;              // terminator
	int64_t chain[TVG_MAX_LEVEL + 1];
	int depth = 0;
	int64_t g = G;
	while (!(tree[g].Bitfield & (1u << 10))) {  // up to the root (TOP bit)
		chain[depth++] = g;
		g = g - tree[g].DUp;
		if (depth > TVG_MAX_LEVEL) return;
	}
	const int t = tree[g].DUp;
	F p[3] = { (F) top[t].pos[0], (F) top[t].pos[1], (F) top[t].pos[2] };
	for (int d = depth - 1; d >= 0; d--) {
		const int64_t gg = chain[d];
		const int l = (int) (tree[gg].Bitfield & 0x3F);
		const int32_t s = u_start[tree_u[gg]];
		p[0] = child_pos<F>(p[0], x[s], dsize, l);
		p[1] = child_pos<F>(p[1], y[s], dsize, l);
		p[2] = child_pos<F>(p[2], z[s], dsize, l);
	}
	tree[G].Pos[0] = p[0];
	tree[G].Pos[1] = p[1];
	tree[G].Pos[2] = p[2];
}

// all nodes (count from the device), grid-stride
template <typename F>
__global__ void k_node_pos(const tvg_devcount *__restrict__ dc, int64_t tcap, TNode<F> *tree,
                           const int32_t *__restrict__ tree_u, const int32_t *__restrict__ u_start,
                           const F *__restrict__ x, const F *__restrict__ y, const F *__restrict__ z,
                           const tvg_topnode *__restrict__ top, double dsize)
{
	const int64_t nnodes = min(dc->nnodes, tcap);
	for (int64_t G = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; G < nnodes;
	     G += (int64_t) gridDim.x * blockDim.x)
		node_pos_one<F>(G, tree, tree_u, u_start, x, y, z, top, dsize);
}

// Float sums in particle order (add_particle_to_node), then CoM /= Mass
template <typename F>
__device__ __forceinline__ void seq_moments(int64_t s, int64_t cnt, const F *__restrict__ x,
                                            const F *__restrict__ y, const F *__restrict__ z,
                                            const F *__restrict__ m, F out[4])
{
	F cx = 0, cy = 0, cz = 0, mm = 0;
	for (int64_t j = s; j < s + cnt; j++) {
		const F mj = m[j];
		if (sizeof(F) == 4) {
			cx = __fadd_rn(cx, __fmul_rn(x[j], mj));
			cy = __fadd_rn(cy, __fmul_rn(y[j], mj));
			cz = __fadd_rn(cz, __fmul_rn(z[j], mj));
			mm = __fadd_rn(mm, mj);
		} else {
			cx = __dadd_rn(cx, __dmul_rn(x[j], mj));
			cy = __dadd_rn(cy, __dmul_rn(y[j], mj));
			cz = __dadd_rn(cz, __dmul_rn(z[j], mj));
			mm = __dadd_rn(mm, mj);
		}
	}
	out[0] = mm;
	out[1] = cx / mm;
	out[2] = cy / mm;
	out[3] = cz / mm;
}

template <typename F>
__global__ void k_moments_seq(const tvg_devcount *__restrict__ dc, int64_t tcap, TNode<F> *tree,
                              const int32_t *__restrict__ tree_u, const int32_t *__restrict__ u_start,
                              const F *__restrict__ x, const F *__restrict__ y, const F *__restrict__ z,
                              const F *__restrict__ m, int exact)
{
	const int64_t nnodes = min(dc->nnodes, tcap);
	for (int64_t G = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; G < nnodes;
	     G += (int64_t) gridDim.x * blockDim.x) {
		const TNode<F> &nd = tree[G];
		if (!(nd.Bitfield & (1u << 9))) continue;
		if (!exact && nd.DNext > 0) continue;       // internal node: fast path
		F o[4];
		seq_moments<F>(u_start[tree_u[G]], nd.Npart, x, y, z, m, o);
		tree[G].Mass = o[0];
		tree[G].CoM[0] = o[1];
		tree[G].CoM[1] = o[2];
		tree[G].CoM[2] = o[3];
	}
}

// fast mode: one warp per internal node, FP64 sums relative to the node
// centre; nodes of more than MOM_BLOCK_MIN particles are left to a block each
// (k_moments_block: the subtree roots below the top nodes hold about N / 64
// particles, and one warp over one of them set the kernel's length)
#define MOM_BLOCK_MIN 8192
template <typename F>
__device__ void moments_warp_one(int64_t G, int lane, TNode<F> *tree, const int32_t *__restrict__ tree_u,
                                 const int32_t *__restrict__ u_start, const F *__restrict__ x,
                                 const F *__restrict__ y, const F *__restrict__ z,
                                 const F *__restrict__ m)
{
	const TNode<F> &nd = tree[G];
	if (!(nd.Bitfield & (1u << 9)) || nd.DNext <= 0 || nd.Npart > MOM_BLOCK_MIN) return;
	const int64_t s = u_start[tree_u[G]], cnt = nd.Npart;
	const double c0 = (double) nd.Pos[0], c1 = (double) nd.Pos[1], c2 = (double) nd.Pos[2];
	double a0 = 0, a1 = 0, a2 = 0, am = 0;
	for (int64_t j = s + lane; j < s + cnt; j += 32) {
		const double mj = (double) m[j];
		am += mj;
		a0 += mj * ((double) x[j] - c0);
		a1 += mj * ((double) y[j] - c1);
		a2 += mj * ((double) z[j] - c2);
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		am += __shfl_xor_sync(0xFFFFFFFFu, am, o);
		a0 += __shfl_xor_sync(0xFFFFFFFFu, a0, o);
		a1 += __shfl_xor_sync(0xFFFFFFFFu, a1, o);
		a2 += __shfl_xor_sync(0xFFFFFFFFu, a2, o);
	}
	if (lane == 0) {
		tree[G].Mass = (F) am;
		tree[G].CoM[0] = (F) (c0 + a0 / am);
		tree[G].CoM[1] = (F) (c1 + a1 / am);
		tree[G].CoM[2] = (F) (c2 + a2 / am);
	}
}

// a warp per node, grid-stride over the device node count
template <typename F>
__global__ void k_moments_warp(const tvg_devcount *__restrict__ dc, int64_t tcap, TNode<F> *tree,
                               const int32_t *__restrict__ tree_u, const int32_t *__restrict__ u_start,
                               const F *__restrict__ x, const F *__restrict__ y, const F *__restrict__ z,
                               const F *__restrict__ m)
{
	const int64_t nnodes = min(dc->nnodes, tcap);
	const int lane = threadIdx.x & 31;
	for (int64_t G = (blockIdx.x * (int64_t) blockDim.x + threadIdx.x) >> 5; G < nnodes;
	     G += ((int64_t) gridDim.x * blockDim.x) >> 5)
		moments_warp_one<F>(G, lane, tree, tree_u, u_start, x, y, z, m);
}

// the internal nodes of more than MOM_BLOCK_MIN particles, listed for
// k_moments_block (list[0] counts them; at most one entry per node)
template <typename F>
__global__ void k_list_big_nodes(const tvg_devcount *__restrict__ dc, int64_t tcap, const TNode<F> *tree,
                                 int32_t *list)
{
	const int64_t nnodes = min(dc->nnodes, tcap);
	for (int64_t G = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; G < nnodes;
	     G += (int64_t) gridDim.x * blockDim.x) {
		const TNode<F> &nd = tree[G];
		if ((nd.Bitfield & (1u << 9)) && nd.DNext > 0 && nd.Npart > MOM_BLOCK_MIN)
			list[1 + atomicAdd(&list[0], 1)] = (int32_t) G;
	}
}

// the listed nodes, a block each, with the FP64 sums of moments_warp_one
#define MOM_BLOCK_THREADS 256
template <typename F>
__global__ void __launch_bounds__(MOM_BLOCK_THREADS) k_moments_block(TNode<F> *tree,
                                                                     const int32_t *__restrict__ tree_u,
                                                                     const int32_t *__restrict__ u_start,
                                                                     const F *__restrict__ x, const F *__restrict__ y,
                                                                     const F *__restrict__ z, const F *__restrict__ m,
                                                                     const int32_t *__restrict__ list)
{
	__shared__ double red[MOM_BLOCK_THREADS / 32][4];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int nl = list[0];
	for (int k = blockIdx.x; k < nl; k += gridDim.x) {
		const int64_t H = list[1 + k];
		const TNode<F> &nd = tree[H];
		const int64_t s = u_start[tree_u[H]], cnt = nd.Npart;
		const double c0x = (double) nd.Pos[0], c0y = (double) nd.Pos[1], c0z = (double) nd.Pos[2];
		double a0 = 0, a1 = 0, a2 = 0, am = 0;
		for (int64_t j = s + threadIdx.x; j < s + cnt; j += MOM_BLOCK_THREADS) {
			const double mj = (double) m[j];
			am += mj;
			a0 += mj * ((double) x[j] - c0x);
			a1 += mj * ((double) y[j] - c0y);
			a2 += mj * ((double) z[j] - c0z);
		}
#pragma unroll
		for (int o = 16; o; o >>= 1) {
			am += __shfl_xor_sync(0xFFFFFFFFu, am, o);
			a0 += __shfl_xor_sync(0xFFFFFFFFu, a0, o);
			a1 += __shfl_xor_sync(0xFFFFFFFFu, a1, o);
			a2 += __shfl_xor_sync(0xFFFFFFFFu, a2, o);
		}
		if (lane == 0) {
			red[w][0] = am;
			red[w][1] = a0;
			red[w][2] = a1;
			red[w][3] = a2;
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			for (int v = 1; v < MOM_BLOCK_THREADS / 32; v++) {
				am += red[v][0];
				a0 += red[v][1];
				a1 += red[v][2];
				a2 += red[v][3];
			}
			tree[H].Mass = (F) am;
			tree[H].CoM[0] = (F) (c0x + a0 / am);
			tree[H].CoM[1] = (F) (c0y + a1 / am);
			tree[H].CoM[2] = (F) (c0z + a2 / am);
		}
		__syncthreads();
	}
}

// top node Mass/CoM (finalise_subtree copies the subtree root, as float),
// terminators (tree_build.c:468-474); small top nodes sum their particles
template <typename F>
__global__ void k_finish_top(const tvg_devcount *__restrict__ dc, tvg_topnode *top, TNode<F> *tree,
                             TopTables tp, int64_t tcap, const F *__restrict__ x,
                             const F *__restrict__ y, const F *__restrict__ z, const F *__restrict__ m,
                             int vsize)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= dc->ntop) return;
	const int32_t *nsurv = tp.nsurv;
	F o[4];
	if (top[t].npart > vsize) {
		const TNode<F> &r = tree[top[t].target];
		o[0] = r.Mass; o[1] = r.CoM[0]; o[2] = r.CoM[1]; o[3] = r.CoM[2];
		TNode<F> term;
		term.DNext = 0; term.Bitfield = 1u << 10; term.DUp = 0; term.Npart = 0;
		for (int k = 0; k < 3; k++) { term.Pos[k] = 0; term.CoM[k] = 0; term.Dp[k] = 0; }
		term.Mass = 1;
		if ((int64_t) top[t].target + nsurv[t] < tcap) tree[(int64_t) top[t].target + nsurv[t]] = term;
	} else {
		seq_moments<F>(top[t].first_part, top[t].npart, x, y, z, m, o);
	}
	top[t].mass = (float) o[0];
	top[t].com[0] = (float) o[1];
	top[t].com[1] = (float) o[2];
	top[t].com[2] = (float) o[3];
}

// Every count (uncollapsed nodes, nodes, top nodes) stays on the device and
// the kernels read it, so the build needs no host round trip (and can be
// captured in a graph); launches are sized by the capacities. The host
// mirrors are read back at the end unless a capture is in progress.
template <typename F>
static int build_typed(tvg_context *ctx, uint32_t flags)
{
	const int64_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	const int vsize = ctx->cfg.vector_size;
	const F *x = (const F *) ctx->f[FS_POS0], *y = (const F *) ctx->f[FS_POS1],
	        *z = (const F *) ctx->f[FS_POS2], *m = (const F *) ctx->f[FS_MASS];
	int32_t *tree_parent = (int32_t *) ctx->f[FS_TREE_PARENT];
	const int64_t ucap = ctx->ucap, tcap = ctx->tcap;
	tvg_devcount *dc = ctx->dc;

	const TopTables tp = tvg_top_tables(ctx);
	k_levels<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, ctx->key_hi, ctx->key_lo, ctx->d_top,
	                                                          ctx->top_of, vsize, ctx->lvl, ctx->ncnt,
	                                                          ctx->lvl_min64, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	if (!ctx->capturing) TVG_CHECK(tvg_sync_status(ctx, "tree_build(levels)"));
	TVG_CHECK(tvg_device_scan_i32_dev(ctx, ctx->ncnt, ctx->ncnt, n + 1, &dc->nu));
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->u_diff, 0, 4 * (ucap + 1), s));
	k_nodes<<<TVG_CNT(ctx, tvg_blocks(n, 128)), 128, 0, s>>>(n, ctx->lvl, ctx->lvl_min64, ctx->ncnt,
	                                            ctx->d_top, ctx->top_of, vsize,
	                                            ctx->u_start, ctx->u_level, ctx->u_count, ctx->u_endu,
	                                            ctx->u_flag, ctx->u_diff, ucap, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	// removal marks -> survivor flags -> final (per top node) indices; entries
	// past nu are zero and do not change the prefix sums below them
	TVG_CHECK(tvg_device_scan_i32(ctx, ctx->u_diff, ctx->u_final, ucap + 1, nullptr));
	k_survivors<<<TVG_CNT(ctx, tvg_blocks(ucap + 1, 256)), 256, 0, s>>>(dc, ucap, ctx->u_final, ctx->u_diff);
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CHECK(tvg_device_scan_i32(ctx, ctx->u_diff, ctx->u_final, ucap + 1, nullptr));
	// placement of the subtrees
	k_place_subtrees<<<TVG_CNT(ctx, 1), 1, 0, s>>>(dc, ctx->d_top, ctx->ncnt, ctx->u_final, vsize, tp,
	                                               ucap, tcap, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	TNode<F> *tree = (TNode<F> *) ctx->tree;
	k_emit_nodes<F><<<TVG_CNT(ctx, tvg_blocks(ucap, 256)), 256, 0, s>>>(
	    dc, ucap, n, ctx->lvl, ctx->lvl_min64, ctx->ncnt, ctx->u_start, ctx->u_level, ctx->u_count,
	    ctx->u_endu, ctx->u_flag, ctx->u_diff, ctx->u_final, ctx->key_hi, ctx->key_lo, ctx->d_top,
	    ctx->top_of, tp, tree, ctx->tree_u, tree_parent, tcap, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	k_small_parent<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, ctx->d_top, ctx->top_of, vsize,
	                                                                tree_parent);
	TVG_CUDA(ctx, cudaGetLastError());
	const unsigned gs = 148 * 16;      // grid-stride launches over the node count
	k_node_pos<F><<<TVG_CNT(ctx, gs), 128, 0, s>>>(dc, tcap, tree, ctx->tree_u, ctx->u_start, x, y, z,
	                                              ctx->d_top, ctx->dsize);
	const int exact = (flags & TVG_BUILD_EXACT_MOMENTS) ? 1 : 0;
	k_moments_seq<F><<<TVG_CNT(ctx, gs), 128, 0, s>>>(dc, tcap, tree, ctx->tree_u, ctx->u_start, x, y, z, m,
	                                                 exact);
	if (!exact) {
		TVG_CUDA(ctx, cudaMemsetAsync(ctx->big_list, 0, 4, s));
		k_list_big_nodes<F><<<TVG_CNT(ctx, gs), 256, 0, s>>>(dc, tcap, tree, ctx->big_list);
		k_moments_warp<F><<<TVG_CNT(ctx, gs), 256, 0, s>>>(dc, tcap, tree, ctx->tree_u, ctx->u_start, x, y, z, m);
		k_moments_block<F><<<TVG_CNT(ctx, 148 * 4), MOM_BLOCK_THREADS, 0, s>>>(tree, ctx->tree_u, ctx->u_start,
		                                                                      x, y, z, m, ctx->big_list);
	}
	TVG_CUDA(ctx, cudaGetLastError());
	k_finish_top<F><<<TVG_CNT(ctx, TVG_MAX_TOP / 128), 128, 0, s>>>(dc, ctx->d_top, tree, tp, tcap, x, y,
	                                                                 z, m, vsize);
	TVG_CUDA(ctx, cudaGetLastError());
	if (ctx->capturing) return TVG_OK;
	TVG_CHECK(tvg_read_counts(ctx));
	if (ctx->nu + 1 > ucap)
		return tvg_fail(ctx, TVG_E_TREE_FULL, "tree_build: %lld uncollapsed nodes > capacity %lld",
		                (long long) ctx->nu, (long long) ucap);
	if (ctx->nnodes > tcap)
		return tvg_fail(ctx, TVG_E_TREE_FULL, "tree_build: %lld nodes > capacity %lld",
		                (long long) ctx->nnodes, (long long) tcap);
	return tvg_sync_status(ctx, "tree_build");
}

int tvg_impl_tree_build(tvg_context *ctx, uint32_t flags)
{
	if (ctx->cfg.float_bytes == 4) return build_typed<float>(ctx, flags);
	return build_typed<double>(ctx, flags);
}

int tvg_impl_download_tree(tvg_context *ctx, void *tree, int64_t cap, int64_t *nnodes)
{
	if (cap < ctx->nnodes)
		return tvg_fail(ctx, TVG_E_BADINPUT, "download_tree: capacity %lld < %lld nodes",
		                (long long) cap, (long long) ctx->nnodes);
	const size_t nb = 16 + 10 * tvg_fsize(ctx);
	TVG_CUDA(ctx, cudaMemcpy(tree, ctx->tree, nb * ctx->nnodes, cudaMemcpyDeviceToHost));
	if (nnodes) *nnodes = ctx->nnodes;
	return TVG_OK;
}
