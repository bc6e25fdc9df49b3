// tvg_walk_group.cu -- the group form of the tree walk.
//
// One warp per PH-contiguous group of 32 x TPL active particles (TPL targets
// per lane, TPL = 1 or 2), persistent blocks fed by an atomic work counter.
// The warp walks the tree once for the whole group with conservative
// (group-wide) opening tests: Barnes-Hut (size^2 > r_min^2 theta^2) or the
// relative criterion of the reference (M size^2 > r_min^4 |a_old|_min / G *
// alpha, tree_accel.c:167, 257) where r_min is the distance from the node's
// centre of mass to the group's bounding box, plus the reference's
// containment test against 0.6 node sizes (tree_accel.c:145-148, 270-281)
// widened by the box. Accepted nodes and the particles of opened bundles go
// into shared-memory interaction lists that all 32 lanes read by broadcast.
//
// Lists: sources whose distance to the group box exceeds the softening
// length go to the far list, whose pair kernel is the bare 1/r^2 law (one
// MUFU.RSQ and ~12 FP32 instructions); the group's own particles and sources
// inside the softening length go to the near list with the full softened
// kernel. Each list flush is summed in FP32 and carried in FP64: the net force
// at high redshift is a small remainder of partial sums hundreds of times
// larger, and a running FP32 sum over 1e5-1e6 interactions loses it.
//
// Precision: positions are 32-bit integer box coordinates (2^32 per box when
// periodic, so that integer wrap-around is the nearest image; 2^31 per
// domain when isolated). Each list entry is converted once to an FP32 offset
// from the group centre.
//
// Periodic images. With the Ewald part, every source is taken at its image
// nearest to the group centre, for all targets of the group, and the Ewald
// correction K (the force of the periodic lattice minus that image) is added
// for the same image: Newton + K is the lattice force, which is smooth across
// the half-box plane, so no target needs its own image. K is evaluated by a
// second, per-group traversal (k_ewald_group): at the centre of mass of each
// accepted node it evaluates K, its Jacobian J and Hessian H (tricubic
// interpolation of the lattice sum tabulated on the octant, with the
// analytic continuation one cell beyond L/2), sums them over the group's
// nodes, and each target adds the second-order Taylor expansion
// K - J t + H:tt/2 about the group centre. Nodes are opened for K by their
// own error estimate (the monopole error of K, G M h2 s^2 / (8 L^4) with h2 a
// bound of |d2K| in box units), except that a node whose extent reaches the
// half-box plane takes the gravity walk's decision, so that both parts always
// use the same image for the same particles. Without the Ewald part
// (parts = gravity only) sources within two group half-widths of the half-box
// plane go to the near list and take per-target nearest images, as the
// reference's gravity walk does (Periodic_Nearest, periodic.c:62-80).
//
// This replaces the reference's Ewald walk (tree_periodic.c:112-422), which
// accepts every node that does not straddle the half-box plane and is at most
// 0.2 L, even where the gravity criterion opens it, and interpolates the
// 65^3 table trilinearly (Gravity/periodic.c:35-113): both leave a force error
// (~3e-3 rms on the 256^3 box at z = 50) that no opening parameter removes.
//
// Roofline: FP32 pipe bound in the pair loop; 20 flop per interaction by
// convention.
#include <stdlib.h>

#include "tvg_internal.cuh"
#include "tvg_ewald_mlp.cuh"

// warps per block and far-list depth (sources per flush); compile-time
// choices, measured flat around these values
#ifndef GW_WARPS
#define GW_WARPS 4
#endif
#define GW_THREADS (GW_WARPS * 32)
// warps per block of the Ewald walk (its registers allow 9 warps per SM)
#ifndef GE_WARPS
#define GE_WARPS 4
#endif
#define GE_THREADS (GE_WARPS * 32)
#define GW_STACK 1024
#define GW_RESERVE (7 * (TVG_MAX_LEVEL - 2) + 8)
#ifndef GW_LIST
#define GW_LIST 256
#endif
#define GW_WLIST 64
#define GW_BQ 64
#define GW_ROOTS 256        // top nodes pushed at a time
#define GW_ELIST 64
#define GW_DEFAULT_TPL 2
// resident blocks per SM the table-evaluating Ewald walk is compiled for:
// 4 (128 registers, 8 B of spill: 15.2 against 15.8 ms per step at 256^3
// with 3 blocks of 168 registers, and 18.4 ms with 2 blocks of 206, since
// the uniform remainder is a polynomial). Before that,
// capping the registers had made it slower, with the tricubic lookup (1340,
// 1442 ms against 1252 ms per step) and with the Taylor table and the closed
// form (140.4 against 136.9 ms at 128^3). The learned correction's walk keeps
// 1 (its network needs the registers).
#ifndef GW_EWALD_MINB
#define GW_EWALD_MINB 4
#endif
// resident blocks per SM the gravity walk is compiled for (4: at most 128
// registers; unbounded it took 138 and ran 3 blocks, 8 % slower), and the
// unroll of its far-list loop (source pairs per iteration)
#ifndef GW_WALK_MINB
#define GW_WALK_MINB 4
#endif
#ifndef GW_FAR_UNROLL
#define GW_FAR_UNROLL 2
#endif
constexpr int kFarUnroll = GW_FAR_UNROLL;

// -------------------------------------------------- integer coordinates

// A coordinate off the integer grid (isolated runs: more than half a domain
// size below the domain of the last decomposition, or 1.5 sizes above it) is
// clamped to the grid's edge and reported (TVG_ST_OFF_GRID): the group form
// would misplace it, so the walk fails instead of returning wrong forces.
__device__ __forceinline__ uint32_t grid_coord(double v, int *bad)
{
	if (!(v >= 0.0)) { *bad = 1; return 0u; }
	if (v >= 4294967296.0) { *bad = 1; return 0xFFFFFFFFu; }
	return (uint32_t) (uint64_t) v;
}

template <typename F>
__global__ void k_int_pos(int64_t n, const F *__restrict__ x, const F *__restrict__ y,
                          const F *__restrict__ z, double ox, double oy, double oz, double fac,
                          uint32_t *__restrict__ ix, uint32_t *__restrict__ iy, uint32_t *__restrict__ iz,
                          int *status)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	int bad = 0;
	ix[i] = grid_coord(((double) x[i] - ox) * fac, &bad);
	iy[i] = grid_coord(((double) y[i] - oy) * fac, &bad);
	iz[i] = grid_coord(((double) z[i] - oz) * fac, &bad);
	if (bad) atomicOr(status, TVG_ST_OFF_GRID);
}

// ----------------------------------------------------- walk tree (CSR)

template <typename F> struct GNode {
	int32_t DNext;
	uint32_t Bitfield;
	int32_t DUp;
	int32_t Npart;
	F Pos[3];
	F Mass;
	F CoM[3];
	F Dp[3];
};

__device__ __forceinline__ bool is_local(uint32_t bf) { return bf & (1u << 9); }
__device__ __forceinline__ bool is_top(uint32_t bf) { return bf & (1u << 10); }

template <typename F>
__device__ __forceinline__ int wt_nchild_one(int64_t g, const GNode<F> *__restrict__ tree)
{
	const GNode<F> &nd = tree[g];
	int cnt = 0;
	if (is_local(nd.Bitfield) && nd.DNext > 0) {
		const int64_t end = g + nd.DNext;
		int64_t c = g + 1;
		while (c < end) {
			cnt++;
			const int32_t dn = tree[c].DNext;
			c += dn > 0 ? dn : 1;
		}
	}
	return cnt;
}

// children per node for the first min(nnodes, tcap) nodes, zeros up to
// lscan (the length of the scan that follows)
template <typename F>
__global__ void k_wt_nchild(const tvg_devcount *__restrict__ dc, int64_t tcap, int64_t lscan,
                            const GNode<F> *__restrict__ tree, int32_t *__restrict__ nch)
{
	const int64_t nn = min(dc->nnodes, tcap);
	for (int64_t g = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; g < lscan;
	     g += (int64_t) gridDim.x * blockDim.x)
		nch[g] = g < nn ? wt_nchild_one<F>(g, tree) : 0;
}

__device__ __forceinline__ uint32_t to_int(double v, double o, double fac)
{
	return (uint32_t) (uint64_t) ((v - o) * fac);
}

template <typename F>
__device__ __forceinline__ void wt_emit_one(int64_t g, int ntop, const GNode<F> *__restrict__ tree,
                                            const int32_t *__restrict__ nch,
                                            const int32_t *__restrict__ choff, double ox, double oy,
                                            double oz, double fac, double dsize,
                                            tvg_wnode *__restrict__ wt, int2 *__restrict__ wrange)
{
	const GNode<F> &nd = tree[g];
	if (!is_local(nd.Bitfield)) return;
	int64_t w;
	if (is_top(nd.Bitfield)) {
		w = nd.DUp;                                   // top node index
	} else {
		const int64_t p = g - nd.DUp;
		int rank = 0;
		int64_t c = p + 1;
		while (c < g) {
			rank++;
			const int32_t dn = tree[c].DNext;
			c += dn > 0 ? dn : 1;
		}
		w = ntop + (int64_t) choff[p] + rank;
	}
	tvg_wnode r;
	r.cx = to_int((double) nd.CoM[0], ox, fac);
	r.cy = to_int((double) nd.CoM[1], oy, fac);
	r.cz = to_int((double) nd.CoM[2], oz, fac);
	r.mass = (float) nd.Mass;
	r.gx = to_int((double) nd.Pos[0], ox, fac);
	r.gy = to_int((double) nd.Pos[1], oy, fac);
	r.gz = to_int((double) nd.Pos[2], oz, fac);
	const int lvl = (int) (nd.Bitfield & 0x3F);
	r.size = (float) (dsize / (double) (1ULL << lvl));
	r.size2 = r.size * r.size;
	r.level = lvl;
	if (nd.DNext > 0) {
		r.child = ntop + choff[g];
		r.nchild = nch[g];
	} else {
		r.child = -nd.DNext - 1;
		r.nchild = -nd.Npart;
	}
	wt[w] = r;
	if (wrange) {
		// particles of the node: Npart from its first particle, the first of
		// the first bundle or leaf below it (pre-order: a first child follows
		// its parent)
		int64_t f = g;
		while (tree[f].DNext > 0) f++;
		wrange[w] = make_int2(-tree[f].DNext - 1, nd.Npart);
	}
}

template <typename F>
__global__ void k_wt_emit(const tvg_devcount *__restrict__ dc, int64_t tcap,
                          const GNode<F> *__restrict__ tree, const int32_t *__restrict__ nch,
                          const int32_t *__restrict__ choff, double ox, double oy, double oz, double fac,
                          double dsize, tvg_wnode *__restrict__ wt, int2 *__restrict__ wrange)
{
	const int64_t nn = min(dc->nnodes, tcap);
	const int ntop = dc->ntop;
	for (int64_t g = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; g < nn;
	     g += (int64_t) gridDim.x * blockDim.x)
		wt_emit_one<F>(g, ntop, tree, nch, choff, ox, oy, oz, fac, dsize, wt, wrange);
}

// top nodes without subtree: one bundle record each (their First_Part; the
// reference's interact_with_topnode_particles reads from Target instead,
// quirk Q3, which the group form does not repeat)
__global__ void k_wt_small_top(const tvg_devcount *__restrict__ dc, const tvg_topnode *__restrict__ top,
                               int vsize, double ox, double oy, double oz, double fac, double dsize,
                               tvg_wnode *__restrict__ wt, int2 *__restrict__ wrange)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= dc->ntop || top[t].npart > vsize) return;
	tvg_wnode r;
	r.cx = to_int((double) top[t].com[0], ox, fac);
	r.cy = to_int((double) top[t].com[1], oy, fac);
	r.cz = to_int((double) top[t].com[2], oz, fac);
	r.mass = top[t].mass;
	r.gx = to_int((double) top[t].pos[0], ox, fac);
	r.gy = to_int((double) top[t].pos[1], oy, fac);
	r.gz = to_int((double) top[t].pos[2], oz, fac);
	r.size = (float) (dsize / (double) (1ULL << top[t].level));
	r.size2 = r.size * r.size;
	r.level = top[t].level;
	r.child = top[t].first_part;
	r.nchild = -top[t].npart;
	wt[t] = r;
	if (wrange) wrange[t] = make_int2(top[t].first_part, top[t].npart);
}

// TVG_CFG_QUADRUPOLE: G times the traceless quadrupole moment of every walk
// node about its centre of mass (the integer one of its record),
// Q_ab = sum m (3 y_a y_b - |y|^2 delta_ab), summed in FP64 over the node's
// particles, stored negated: wq[2w] = -(Qxx, Qyy, Qzz, Qxy),
// wq[2w + 1] = -(Qxz, Qyz, 0, 0).
struct QuadSums {
	double xx, yy, zz, xy, xz, yz;
};

__device__ __forceinline__ void quad_add(QuadSums &q, const uint32_t *__restrict__ ix,
                                         const uint32_t *__restrict__ iy, const uint32_t *__restrict__ iz,
                                         const float *__restrict__ mass_f, int64_t j, uint32_t cx,
                                         uint32_t cy, uint32_t cz, double scale)
{
	const double m = (double) mass_f[j];
	const double x = (double) (int) (ix[j] - cx) * scale, y = (double) (int) (iy[j] - cy) * scale,
	             z = (double) (int) (iz[j] - cz) * scale;
	q.xx += m * x * x;
	q.yy += m * y * y;
	q.zz += m * z * z;
	q.xy += m * x * y;
	q.xz += m * x * z;
	q.yz += m * y * z;
}

__device__ __forceinline__ void quad_store(const QuadSums &q, double gravity, float4 *__restrict__ wq,
                                           int64_t w)
{
	const double tr = q.xx + q.yy + q.zz, g = -gravity;
	wq[2 * w] = make_float4((float) (g * (3 * q.xx - tr)), (float) (g * (3 * q.yy - tr)),
	                        (float) (g * (3 * q.zz - tr)), (float) (g * 3 * q.xy));
	wq[2 * w + 1] = make_float4((float) (g * 3 * q.xz), (float) (g * 3 * q.yz), 0.f, 0.f);
}

// Every walk node (top nodes + the walk nodes below them, counted on the
// device), in two passes: a lane sums a node of at most GW_QUAD_LANE
// particles by itself (most nodes: bundles and the levels just above them),
// 32 consecutive nodes to a warp; then each larger node takes a warp of its
// own with a butterfly reduction. (Larger nodes come in runs, the top levels
// first, so a warp of 32 consecutive nodes summing its large ones in turn
// would leave one warp with the top nodes: 75 ms per 256^3 step.)
#define GW_QUAD_LANE 64
// nodes of more particles than this (the top nodes, about N / 64 each, and
// the levels just below them) are summed by a block each, k_wt_quad_block
#define GW_QUAD_BLOCK 8192
__global__ void k_wt_quad_dev(const tvg_devcount *__restrict__ dc, const tvg_wnode *__restrict__ wt,
                              const int2 *__restrict__ wrange, const uint32_t *__restrict__ ix,
                              const uint32_t *__restrict__ iy, const uint32_t *__restrict__ iz,
                              const float *__restrict__ mass_f, double scale, double gravity,
                              float4 *__restrict__ wq)
{
	const int64_t nw = (int64_t) dc->ntop + dc->nwchild;
	const int lane = threadIdx.x & 31;
	const int64_t warp = (blockIdx.x * (int64_t) blockDim.x + threadIdx.x) >> 5;
	const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
	for (int64_t w = warp * 32 + lane; w - lane < nw; w += nwarps * 32) {
		if (w >= nw) continue;
		const int2 r = wrange[w];
		if (r.y <= 0 || r.y > GW_QUAD_LANE) continue;
		QuadSums q = { 0, 0, 0, 0, 0, 0 };
		const uint32_t cx = wt[w].cx, cy = wt[w].cy, cz = wt[w].cz;
		for (int64_t j = r.x; j < (int64_t) r.x + r.y; j++) quad_add(q, ix, iy, iz, mass_f, j, cx, cy, cz, scale);
		quad_store(q, gravity, wq, w);
	}
	for (int64_t w = warp; w < nw; w += nwarps) {
		const int2 r = wrange[w];
		if (r.y <= GW_QUAD_LANE || r.y > GW_QUAD_BLOCK) continue;
		const uint32_t cx = wt[w].cx, cy = wt[w].cy, cz = wt[w].cz;
		QuadSums q = { 0, 0, 0, 0, 0, 0 };
		for (int64_t j = r.x + lane; j < (int64_t) r.x + r.y; j += 32)
			quad_add(q, ix, iy, iz, mass_f, j, cx, cy, cz, scale);
#pragma unroll
		for (int o = 16; o; o >>= 1) {
			q.xx += __shfl_xor_sync(0xFFFFFFFFu, q.xx, o);
			q.yy += __shfl_xor_sync(0xFFFFFFFFu, q.yy, o);
			q.zz += __shfl_xor_sync(0xFFFFFFFFu, q.zz, o);
			q.xy += __shfl_xor_sync(0xFFFFFFFFu, q.xy, o);
			q.xz += __shfl_xor_sync(0xFFFFFFFFu, q.xz, o);
			q.yz += __shfl_xor_sync(0xFFFFFFFFu, q.yz, o);
		}
		if (lane == 0) quad_store(q, gravity, wq, w);
	}
}

// the walk nodes of more than GW_QUAD_BLOCK particles, listed for
// k_wt_quad_block (list[0] counts them). The top nodes come first in the
// walk tree, so a block per chunk of consecutive nodes would leave one
// block with all of them.
__global__ void k_wt_list_big(const tvg_devcount *__restrict__ dc, const int2 *__restrict__ wrange, int32_t *list)
{
	const int64_t nw = (int64_t) dc->ntop + dc->nwchild;
	for (int64_t w = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; w < nw;
	     w += (int64_t) gridDim.x * blockDim.x)
		if (wrange[w].y > GW_QUAD_BLOCK) list[1 + atomicAdd(&list[0], 1)] = (int32_t) w;
}

// the listed walk nodes, a block each
#define GW_QUAD_BLOCK_THREADS 256
__global__ void __launch_bounds__(GW_QUAD_BLOCK_THREADS)
k_wt_quad_block(const tvg_wnode *__restrict__ wt, const int2 *__restrict__ wrange,
                const uint32_t *__restrict__ ix, const uint32_t *__restrict__ iy, const uint32_t *__restrict__ iz,
                const float *__restrict__ mass_f, double scale, double gravity, float4 *__restrict__ wq,
                const int32_t *__restrict__ list)
{
	__shared__ double red[GW_QUAD_BLOCK_THREADS / 32][6];
	const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
	const int nl = list[0];
	for (int k = blockIdx.x; k < nl; k += gridDim.x) {
		const int64_t v = list[1 + k];
		const int2 r = wrange[v];
		const uint32_t cx = wt[v].cx, cy = wt[v].cy, cz = wt[v].cz;
		QuadSums q = { 0, 0, 0, 0, 0, 0 };
		for (int64_t j = r.x + threadIdx.x; j < (int64_t) r.x + r.y; j += GW_QUAD_BLOCK_THREADS)
			quad_add(q, ix, iy, iz, mass_f, j, cx, cy, cz, scale);
#pragma unroll
		for (int o = 16; o; o >>= 1) {
			q.xx += __shfl_xor_sync(0xFFFFFFFFu, q.xx, o);
			q.yy += __shfl_xor_sync(0xFFFFFFFFu, q.yy, o);
			q.zz += __shfl_xor_sync(0xFFFFFFFFu, q.zz, o);
			q.xy += __shfl_xor_sync(0xFFFFFFFFu, q.xy, o);
			q.xz += __shfl_xor_sync(0xFFFFFFFFu, q.xz, o);
			q.yz += __shfl_xor_sync(0xFFFFFFFFu, q.yz, o);
		}
		if (lane == 0) {
			red[wp][0] = q.xx;
			red[wp][1] = q.yy;
			red[wp][2] = q.zz;
			red[wp][3] = q.xy;
			red[wp][4] = q.xz;
			red[wp][5] = q.yz;
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			for (int u = 1; u < GW_QUAD_BLOCK_THREADS / 32; u++) {
				q.xx += red[u][0];
				q.yy += red[u][1];
				q.zz += red[u][2];
				q.xy += red[u][3];
				q.xz += red[u][4];
				q.yz += red[u][5];
			}
			quad_store(q, gravity, wq, v);
		}
		__syncthreads();
	}
}


// ------------------------------------------------------------- the walk

// images the gravity walk uses
enum {
	GM_NEAREST = 0,     // per-target nearest image (isolated, or periodic without Ewald)
	GM_CENTRE = 1       // the image nearest to the group centre (periodic, with k_ewald_group)
};

struct GroupParams {
	int64_t n;                 // particles (groups of consecutive particles without an active list)
	const tvg_devcount *dc;    // device counts: top nodes, groups, total mass
	int gsize;
	int periodic;
	int use_bh;
	int open_bundles;   // TVG_CFG_OPEN_BUNDLES
	int max_iter;       // iteration limit of a group's traversal (tvg_set_walk_limit)
	int quad;           // TVG_CFG_QUADRUPOLE: node quadrupoles, octupole-order criterion
	float scale;        // length per integer unit
	float box, half_box;
	float theta2;       // TREE_OPEN_PARAM_BH
	float rel_fac;      // TREE_OPEN_PARAM_REL / G
	float gravity;
	float eps2, inv_eps2, c16;     // softening (h^2, 1/h^2, 1/(16 h^3))
	float near2;        // h^2 with a rounding margin: closer sources use the softened kernel
	float grid;         // Ewald table cells per length (2 * 64 / L)
	float inv_box;
	float ew_rel;       // Ewald opening: alpha_E / TREE_OPEN_PARAM_REL (relative mode)
	float ew_bh;        // Ewald opening: s^2 h2 limit in units of L^2 (Barnes-Hut mode)
	float taylor_h;     // groups with a larger half extent take per-target images (with Ewald)
	float tay_grid;     // Taylor-table node spacings per length (2 (TVG_TAYLOR_NODES - 1) / L)
	double uniform_g;   // G / L^2: times the total mass, the scale of the uniform-background remainder
};

// The far list keeps sources in pairs: entries 2q and 2q + 1 share the two
// float4 slots lxy[q] = (x0, x1, y0, y1) and lzw[q] = (z0, z1, w0, w1), so that
// each lane meets two sources with one packed f32x2 instruction per operation
// while its target's coordinates stay in registers as (t, t) pairs.
struct WarpSmem {
	int32_t stack[GW_STACK];
	float4 lxy[GW_LIST / 2];   // far sources (bare 1/r^2 kernel): x, y of a pair
	float4 lzw[GW_LIST / 2];   // far sources: z, G m of a pair
	float4 wlist[GW_WLIST];    // near sources (w > 0) and, per-target image, half-box-plane sources (w < 0)
	int2 bq[GW_BQ];
};

__device__ __forceinline__ void far_put(WarpSmem &S, int i, float4 e)
{
	float *a = (float *) &S.lxy[i >> 1], *b = (float *) &S.lzw[i >> 1];
	const int o = i & 1;
	a[o] = e.x;
	a[2 + o] = e.y;
	b[o] = e.z;
	b[2 + o] = e.w;
}


struct EwaldSmem {
	int32_t stack[GW_STACK];
	float4 list[GW_ELIST];     // accepted sources: offset from the group centre, G m
	int32_t lnode[GW_ELIST];   // TVG_CFG_QUADRUPOLE: their walk nodes (-1: a particle)
	int2 bq[GW_BQ];
};

// Per-warp stage of the Ewald walk's Taylor records (table evaluation),
// compiled in with GW_EWALD_STAGE=1: a full batch of 32 accepted sources has
// its 32 records (256 B each) copied from the table in global memory into
// shared memory by the bulk-copy (TMA) engine, cp.async.bulk completing on an
// mbarrier, while the warp goes on walking; the batch is evaluated from
// shared memory when the next one is issued. Two buffers: a new batch is
// issued before the pending one is evaluated. Sources are this GPU's own
// memory; no multicast. The results are those of the direct loads bit for
// bit, but the walk is slower (768 against 462 ms per 256^3 step): the
// records of neighbouring groups are reused through L1, which bulk copies
// bypass and the 92 KB stage per block shrinks. Off by default.
#ifndef GW_EWALD_STAGE
#define GW_EWALD_STAGE 0
#endif
struct EwaldStage {
	float4 rec[2][32][16];     // the batches' records
	float4 pend[2][32];        // the batches' sources
	uint64_t bar[2];           // completion barriers (arrival count 1 + transaction bytes)
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
	return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
	             : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
	uint32_t done;
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	             "selp.u32 %0, 1, 0, p;\n\t}"
	             : "=r"(done)
	             : "r"(smem_addr(bar)), "r"(parity)
	             : "memory");
	return done != 0;
}

// 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple
// of 16), completing `bytes` transactions on the mbarrier
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
	             ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
	             : "memory");
}

// per-lane sums over accepted sources of m K, m J and m H (about the group
// centre), FP32 (a few hundred terms per lane)
struct CorrSum {
	float k[3];
	float j[9];     // J[a][b] = dK_a / dd_b
	float h[18];    // H[a][xx, yy, zz, xy, xz, yz]
};

struct Target {
	float tx, ty, tz;       // offset from the group centre
	double ax, ay, az;      // FP32 sums of each list flush, carried in FP64
	float cost;
	float qcost;            // of which quadrupole interactions (TVG_CFG_QUADRUPOLE)
	bool valid;
};

struct GroupBox {
	uint32_t cx, cy, cz;    // centre, integer coordinates
	float hx, hy, hz;       // half extents (+ one unit)
	float fac;              // |a_old|_min * TREE_OPEN_PARAM_REL / G
};

// bounding box, centre and |a_old|_min of the group; target offsets
template <int TPL>
__device__ __forceinline__ void group_setup(const GroupParams &p, const uint32_t *__restrict__ ix,
                                            const uint32_t *__restrict__ iy,
                                            const uint32_t *__restrict__ iz,
                                            const float *__restrict__ last_acc,
                                            const int32_t *__restrict__ active, int64_t first,
                                            int cnt, Target (&t)[TPL], GroupBox &g)
{
	const int lane = threadIdx.x & 31;
	uint32_t px[TPL], py[TPL], pz[TPL];
	const int64_t me0 = active ? (int64_t) active[first] : first;
	const uint32_t rx = ix[me0], ry = iy[me0], rz = iz[me0];
	int minx = 0, maxx = 0, miny = 0, maxy = 0, minz = 0, maxz = 0;
	float amin = 3.0e38f;
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		const int slot = lane + 32 * k;
		t[k].valid = slot < cnt;
		const int64_t me = t[k].valid ? (active ? (int64_t) active[first + slot] : first + slot) : me0;
		px[k] = ix[me];
		py[k] = iy[me];
		pz[k] = iz[me];
		const int ox = (int) (px[k] - rx), oy = (int) (py[k] - ry), oz = (int) (pz[k] - rz);
		minx = min(minx, ox); maxx = max(maxx, ox);
		miny = min(miny, oy); maxy = max(maxy, oy);
		minz = min(minz, oz); maxz = max(maxz, oz);
		if (t[k].valid) amin = fminf(amin, last_acc[me]);
	}
	minx = __reduce_min_sync(0xFFFFFFFFu, minx); maxx = __reduce_max_sync(0xFFFFFFFFu, maxx);
	miny = __reduce_min_sync(0xFFFFFFFFu, miny); maxy = __reduce_max_sync(0xFFFFFFFFu, maxy);
	minz = __reduce_min_sync(0xFFFFFFFFu, minz); maxz = __reduce_max_sync(0xFFFFFFFFu, maxz);
	g.cx = rx + (uint32_t) (((int64_t) minx + maxx) >> 1);
	g.cy = ry + (uint32_t) (((int64_t) miny + maxy) >> 1);
	g.cz = rz + (uint32_t) (((int64_t) minz + maxz) >> 1);
	g.hx = ((float) ((int64_t) maxx - minx) * 0.5f + 1.f) * p.scale;
	g.hy = ((float) ((int64_t) maxy - miny) * 0.5f + 1.f) * p.scale;
	g.hz = ((float) ((int64_t) maxz - minz) * 0.5f + 1.f) * p.scale;
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		// rounded products (no FMA contraction into the later subtraction): a
		// particle's own list entry must sit at exactly zero separation, since
		// the reference's inner kernel (h < 0) turns any residue into a force
		t[k].tx = __fmul_rn((float) (int) (px[k] - g.cx), p.scale);
		t[k].ty = __fmul_rn((float) (int) (py[k] - g.cy), p.scale);
		t[k].tz = __fmul_rn((float) (int) (pz[k] - g.cz), p.scale);
		t[k].ax = t[k].ay = t[k].az = 0.0;
		t[k].cost = 0.f;
		t[k].qcost = 0.f;
	}
	// group-wide relative criterion: the smallest |a_old| opens the most
#pragma unroll
	for (int o = 16; o; o >>= 1) amin = fminf(amin, __shfl_xor_sync(0xFFFFFFFFu, amin, o));
	g.fac = amin * p.rel_fac;
}

// offset of an integer coordinate from the group centre (rounded product)
__device__ __forceinline__ float ioff(uint32_t v, uint32_t c, float scale)
{
	return __fmul_rn((float) (int) (v - c), scale);
}

// The gravity walk's opening decision for a node (shared by both walks, so
// that the Ewald walk can repeat it bit for bit). d: centre of mass offset,
// gx..: geometric centre offset. r2 receives the squared distance from the
// centre of mass to the group box. quad: the octupole-order criterion
// (TVG_CFG_QUADRUPOLE, groups without per-target images), except for a node
// within the softening length, which goes to the softened monopole list.
__device__ __forceinline__ bool gravity_opens(const GroupParams &p, const GroupBox &g,
                                              const tvg_wnode &nd, int node, float dx, float dy,
                                              float dz, float gx, float gy, float gz, float &r2,
                                              bool quad)
{
	const float qx = fmaxf(fabsf(dx) - g.hx, 0.f), qy = fmaxf(fabsf(dy) - g.hy, 0.f),
	            qz = fmaxf(fabsf(dz) - g.hz, 0.f);
	r2 = qx * qx + qy * qy + qz * qz;
	bool want;
	if (p.use_bh) want = nd.size2 > r2 * p.theta2;
	else if (quad && r2 >= p.near2) want = nd.mass * nd.size2 * nd.size > r2 * r2 * sqrtf(r2) * g.fac;
	else want = nd.mass * nd.size2 > r2 * r2 * g.fac;
	const float lim = 0.6f * nd.size;
	if (fabsf(gx) < lim + g.hx && fabsf(gy) < lim + g.hy && fabsf(gz) < lim + g.hz) want = true;
	// with TVG_CFG_OPEN_BUNDLES a bundle below the top level is never a
	// monopole: the reference interacts its particles whenever the walk
	// reaches it (tree_accel.c:221-243, tree_periodic.c:228-251)
	return want || (p.open_bundles && nd.nchild < 0 && node >= p.dc->ntop);
}

// Pops k <= 32 nodes of the stack (one per lane, -1 for idle lanes).
// Batches of up to 32 nodes may push 8 children each, so a batch of k keeps
// sp + 7k below GW_STACK - GW_RESERVE. Above that line the warp takes one
// node at a time: from there on the stack holds at most 7 siblings per level
// of the current path (<= 40 levels below the top nodes), which the reserve
// covers, so the stack cannot overflow.
__device__ __forceinline__ int pop_nodes(const int32_t *stack, int &sp, int *status, bool &stop)
{
	const int lane = threadIdx.x & 31;
	int k = min(32, sp);
	const int room = (GW_STACK - GW_RESERVE - sp) / 7;
	if (room < k) k = max(room, 1);
	stop = false;
	if (sp + 7 * k > GW_STACK) {
		atomicOr(status, TVG_ST_LIST_OVERFLOW);
		stop = true;
		return -1;
	}
	int node = -1;
	if (lane < k) node = stack[sp - 1 - lane];
	sp -= k;
	__syncwarp();
	return node;
}

// pushes the children of the lanes' opened internal nodes
__device__ __forceinline__ void push_children(int32_t *stack, int &sp, bool open_int, int nchild,
                                              int child)
{
	const int lane = threadIdx.x & 31;
	int c = open_int ? nchild : 0, incl = c;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int u = __shfl_up_sync(0xFFFFFFFFu, incl, o);
		if (lane >= o) incl += u;
	}
	const int tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
	for (int q = 0; q < c; q++) stack[sp + incl - c + q] = child + c - 1 - q;
	sp += tot;
}

// softened monopole, reference kernel (Dehnen K1 with h = -41/32 eps,
// tree_accel.c:362-394) in FP32 for a separation d; the r2 = 0 self term
// selects the inner branch and adds exactly zero
__device__ __forceinline__ void pair_full(const GroupParams &p, float dx, float dy, float dz,
                                          float gm, float &ax, float &ay, float &az)
{
	const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
	const float ri = rsqrtf(r2);
	const float fout = ri * ri * ri;
	const float u2 = r2 * p.inv_eps2;
	const float fin = fmaf(u2, fmaf(u2, 135.0f, -294.0f), 175.0f) * p.c16;
	const float f = gm * (r2 < p.eps2 ? fin : fout);
	ax = fmaf(f, dx, ax);
	ay = fmaf(f, dy, ay);
	az = fmaf(f, dz, az);
}

// Far-list flush: for every target of the lane, two sources per packed
// (f32x2) step -- 3 FADD2, FMUL2 + 2 FFMA2 for r^2, two MUFU.RSQ, 3 FMUL2 and
// 3 FFMA2 for two interactions, against 24 scalar FP32 instructions -- so the
// loop is bound by the FMA pipe rather than by instruction issue. The even
// and odd sources are summed separately and added at the end of the flush.
// An odd count is padded with a massless source far away (adds exactly 0).
template <int TPL>
__device__ __forceinline__ void flush_far(WarpSmem &S, int nl, Target (&t)[TPL])
{
	if (nl & 1) {
		if ((threadIdx.x & 31) == 0) far_put(S, nl, make_float4(1.0e15f, 0.f, 0.f, 0.f));
		__syncwarp();
	}
	const int np = (nl + 1) >> 1;
	float2 ax[TPL], ay[TPL], az[TPL], mx[TPL], my[TPL], mz[TPL];
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		ax[k] = ay[k] = az[k] = make_float2(0.f, 0.f);
		mx[k] = make_float2(-t[k].tx, -t[k].tx);
		my[k] = make_float2(-t[k].ty, -t[k].ty);
		mz[k] = make_float2(-t[k].tz, -t[k].tz);
	}
#pragma unroll kFarUnroll
	for (int q = 0; q < np; q++) {
		const float4 a = S.lxy[q], b = S.lzw[q];
		const float2 sx = make_float2(a.x, a.y), sy = make_float2(a.z, a.w),
		             sz = make_float2(b.x, b.y), sw = make_float2(b.z, b.w);
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			const float2 dx = __fadd2_rn(sx, mx[k]), dy = __fadd2_rn(sy, my[k]),
			             dz = __fadd2_rn(sz, mz[k]);
			const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
			const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
			const float2 f = __fmul2_rn(__fmul2_rn(sw, ri), __fmul2_rn(ri, ri));
			ax[k] = __ffma2_rn(f, dx, ax[k]);
			ay[k] = __ffma2_rn(f, dy, ay[k]);
			az[k] = __ffma2_rn(f, dz, az[k]);
		}
	}
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		t[k].ax += (double) ax[k].x + (double) ax[k].y;
		t[k].ay += (double) ay[k].x + (double) ay[k].y;
		t[k].az += (double) az[k].x + (double) az[k].y;
		t[k].cost += (float) nl;
	}
	__syncwarp();
}

// TVG_CFG_QUADRUPOLE: the accepted nodes with their quadrupoles (-G Q), in
// pairs like the far list; in shared memory after the warps' WarpSmem
#define GW_QLIST 64
struct QuadList {
	float4 xy[GW_QLIST / 2];   // x0 x1 y0 y1
	float4 zw[GW_QLIST / 2];   // z0 z1 w0 w1 (w = G m)
	float4 qa[GW_QLIST / 2];   // Qxx0 Qxx1 Qyy0 Qyy1
	float4 qb[GW_QLIST / 2];   // Qzz0 Qzz1 Qxy0 Qxy1
	float4 qc[GW_QLIST / 2];   // Qxz0 Qxz1 Qyz0 Qyz1
};

__device__ __forceinline__ void quad_put(QuadList &Q, int i, float4 e, float4 q0, float4 q1)
{
	const int h = i >> 1, o = i & 1;
	float *a = (float *) &Q.xy[h], *b = (float *) &Q.zw[h], *c = (float *) &Q.qa[h],
	      *d = (float *) &Q.qb[h], *f = (float *) &Q.qc[h];
	a[o] = e.x;
	a[2 + o] = e.y;
	b[o] = e.z;
	b[2 + o] = e.w;
	c[o] = q0.x;
	c[2 + o] = q0.y;
	d[o] = q0.z;
	d[2 + o] = q0.w;
	f[o] = q1.x;
	f[2 + o] = q1.y;
}

// Quadrupole flush: with d = source - target, r = |d| and the stored -G Q,
// a = G M d / r^3 + (-G Q) d / r^5 - 5/2 (d . (-G Q) d) d / r^7, two sources
// per packed step (31 f32x2 operations and two MUFU.RSQ per two
// interactions). An odd count is padded with a massless source far away.
template <int TPL>
__device__ __forceinline__ void flush_quad(QuadList &Q, int nq, Target (&t)[TPL])
{
	if (nq & 1) {
		if ((threadIdx.x & 31) == 0)
			quad_put(Q, nq, make_float4(1.0e15f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f),
			         make_float4(0.f, 0.f, 0.f, 0.f));
		__syncwarp();
	}
	const int np = (nq + 1) >> 1;
	const float2 m25 = make_float2(-2.5f, -2.5f);
	float2 ax[TPL], ay[TPL], az[TPL], mx[TPL], my[TPL], mz[TPL];
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		ax[k] = ay[k] = az[k] = make_float2(0.f, 0.f);
		mx[k] = make_float2(-t[k].tx, -t[k].tx);
		my[k] = make_float2(-t[k].ty, -t[k].ty);
		mz[k] = make_float2(-t[k].tz, -t[k].tz);
	}
	// two source pairs per iteration: four independent chains per lane
	// (150.7 against 152.7 ms per 256^3 step with one pair; three pairs:
	// 151.7 against 149.7 ms of walk)
#pragma unroll 2
	for (int q = 0; q < np; q++) {
		const float4 a = Q.xy[q], b = Q.zw[q], qa = Q.qa[q], qb = Q.qb[q], qc = Q.qc[q];
		const float2 sx = make_float2(a.x, a.y), sy = make_float2(a.z, a.w),
		             sz = make_float2(b.x, b.y), sw = make_float2(b.z, b.w);
		const float2 qxx = make_float2(qa.x, qa.y), qyy = make_float2(qa.z, qa.w),
		             qzz = make_float2(qb.x, qb.y), qxy = make_float2(qb.z, qb.w),
		             qxz = make_float2(qc.x, qc.y), qyz = make_float2(qc.z, qc.w);
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			const float2 dx = __fadd2_rn(sx, mx[k]), dy = __fadd2_rn(sy, my[k]),
			             dz = __fadd2_rn(sz, mz[k]);
			const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
			const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
			const float2 ri2 = __fmul2_rn(ri, ri), ri3 = __fmul2_rn(ri2, ri);
			const float2 fm = __fmul2_rn(sw, ri3);
			const float2 qdx = __ffma2_rn(qxx, dx, __ffma2_rn(qxy, dy, __fmul2_rn(qxz, dz)));
			const float2 qdy = __ffma2_rn(qxy, dx, __ffma2_rn(qyy, dy, __fmul2_rn(qyz, dz)));
			const float2 qdz = __ffma2_rn(qxz, dx, __ffma2_rn(qyz, dy, __fmul2_rn(qzz, dz)));
			const float2 dqd = __ffma2_rn(dx, qdx, __ffma2_rn(dy, qdy, __fmul2_rn(dz, qdz)));
			const float2 ri5 = __fmul2_rn(ri3, ri2), ri7 = __fmul2_rn(ri5, ri2);
			const float2 cd = __ffma2_rn(__fmul2_rn(dqd, ri7), m25, fm);
			ax[k] = __ffma2_rn(cd, dx, __ffma2_rn(qdx, ri5, ax[k]));
			ay[k] = __ffma2_rn(cd, dy, __ffma2_rn(qdy, ri5, ay[k]));
			az[k] = __ffma2_rn(cd, dz, __ffma2_rn(qdz, ri5, az[k]));
		}
	}
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		t[k].ax += (double) ax[k].x + (double) ax[k].y;
		t[k].ay += (double) ay[k].x + (double) ay[k].y;
		t[k].az += (double) az[k].x + (double) az[k].y;
		t[k].cost += (float) nq;
		t[k].qcost += (float) nq;
	}
	__syncwarp();
}


__device__ __forceinline__ float wrap_half(float d, float box, float half)
{
	d = d > half ? d - box : d;
	return d < -half ? d + box : d;
}

// near list: softened kernel; entries with w < 0 take per-target images
template <int TPL>
__device__ __forceinline__ void flush_slow(const GroupParams &p, const float4 *list, int nl,
                                           Target (&t)[TPL])
{
	float ax[TPL], ay[TPL], az[TPL];
#pragma unroll
	for (int k = 0; k < TPL; k++) ax[k] = ay[k] = az[k] = 0.f;
	for (int e = 0; e < nl; e++) {
		const float4 s = list[e];
		const bool wrap = s.w < 0.f;
		const float gm = fabsf(s.w);
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			float dx = s.x - t[k].tx, dy = s.y - t[k].ty, dz = s.z - t[k].tz;
			if (wrap) {
				dx = wrap_half(dx, p.box, p.half_box);
				dy = wrap_half(dy, p.box, p.half_box);
				dz = wrap_half(dz, p.box, p.half_box);
			}
			pair_full(p, dx, dy, dz, gm, ax[k], ay[k], az[k]);
		}
	}
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		t[k].ax += (double) ax[k];
		t[k].ay += (double) ay[k];
		t[k].az += (double) az[k];
		t[k].cost += (float) nl;
	}
}

// gravity walk of one group: 32 * TPL PH-contiguous active particles, lane l
// holds the particles first + l + 32 k
template <int MODE, int TPL, bool QUAD>
__device__ void walk_group(const GroupParams &p, WarpSmem &S, const tvg_wnode *__restrict__ wt,
                           const uint32_t *__restrict__ ix, const uint32_t *__restrict__ iy,
                           const uint32_t *__restrict__ iz, const float *__restrict__ mass_f,
                           const float *__restrict__ last_acc, int64_t first, int cnt,
                           const int32_t *__restrict__ active, Target (&t)[TPL], QuadList *QL,
                           const float4 *__restrict__ wq, int *status)
{
	const int lane = threadIdx.x & 31;
	const unsigned lt = (1u << lane) - 1u;
	GroupBox g;
	group_setup<TPL>(p, ix, iy, iz, last_acc, active, first, cnt, t, g);
	// with per-target images: a source this close to the half-box plane needs
	// them. With the Ewald walk, only groups too large for its expansion
	// about the centre take them (the same test there).
	const bool per_target = p.periodic
	    && (MODE == GM_NEAREST || fmaxf(g.hx, fmaxf(g.hy, g.hz)) >= p.taylor_h);
	const float wlimx = p.half_box - 2.f * g.hx, wlimy = p.half_box - 2.f * g.hy,
	            wlimz = p.half_box - 2.f * g.hz;
	// per-target images go to the monopole list: their nodes keep the
	// monopole criterion (the Ewald walk makes the same choice)
	const bool quad_open = QUAD && !per_target;

	int sp = 0, nl = 0, nw = 0, nq = 0;
	const int ntop = p.dc->ntop;
	int guard = 0;
	bool halt = false;
	// the roots in chunks of GW_ROOTS (a balanced decomposition can have
	// thousands of top nodes, more than the stack holds at once)
	for (int r0 = 0; r0 < ntop && !halt; r0 += GW_ROOTS) {
		const int nr = min(GW_ROOTS, ntop - r0);
		for (int r = lane; r < nr; r += 32) S.stack[r] = r0 + r;
		sp = nr;
		__syncwarp();
		while (sp > 0) {
			if (++guard > p.max_iter) { atomicOr(status, TVG_ST_TIMEOUT); halt = true; break; }
			bool stop;
			const int node = pop_nodes(S.stack, sp, status, stop);
			if (stop) { halt = true; break; }
			bool accept = false, open_int = false, open_bundle = false, wrap = false, near = false;
			float4 entry = make_float4(0.f, 0.f, 0.f, 0.f);
			int nchild = 0, child = 0;
			if (node >= 0) {
				const tvg_wnode nd = wt[node];
				const float dx = ioff(nd.cx, g.cx, p.scale), dy = ioff(nd.cy, g.cy, p.scale),
				            dz = ioff(nd.cz, g.cz, p.scale);
				float r2;
				const bool open = gravity_opens(p, g, nd, node, dx, dy, dz, ioff(nd.gx, g.cx, p.scale),
				                                ioff(nd.gy, g.cy, p.scale), ioff(nd.gz, g.cz, p.scale), r2,
				                                quad_open);
				if (!open) {
					accept = true;
					entry = make_float4(dx, dy, dz, p.gravity * nd.mass);
					wrap = per_target && (fabsf(dx) > wlimx || fabsf(dy) > wlimy || fabsf(dz) > wlimz);
					near = r2 < p.near2;
				} else if (nd.nchild > 0) {
					open_int = true;
					nchild = nd.nchild;
					child = nd.child;
				} else {
					open_bundle = true;
					nchild = -nd.nchild;
					child = nd.child;
				}
			}
			// accepted nodes -> interaction lists
			const bool to_far = accept && !wrap && !near;
			const bool to_slow = accept && (wrap || near);
			if (wrap) entry.w = -entry.w;
			const unsigned bm = __ballot_sync(0xFFFFFFFFu, to_far);
			const unsigned bw = __ballot_sync(0xFFFFFFFFu, to_slow);
			// (with quadrupoles the accepted nodes go to the quadrupole list;
			// the far list then holds the particles of opened bundles)
			if (QUAD) {
				if (nq + __popc(bm) > GW_QLIST) {
					flush_quad<TPL>(*QL, nq, t);
					nq = 0;
					__syncwarp();
				}
			} else if (nl + __popc(bm) > GW_LIST) {
				flush_far<TPL>(S, nl, t);
				nl = 0;
				__syncwarp();
			}
			if (nw + __popc(bw) > GW_WLIST) {
				flush_slow<TPL>(p, S.wlist, nw, t);
				nw = 0;
				__syncwarp();
			}
			if (to_far) {
				if (QUAD) quad_put(*QL, nq + __popc(bm & lt), entry, wq[2 * node], wq[2 * node + 1]);
				else far_put(S, nl + __popc(bm & lt), entry);
			}
			if (to_slow) S.wlist[nw + __popc(bw & lt)] = entry;
			if (QUAD) nq += __popc(bm);
			else nl += __popc(bm);
			nw += __popc(bw);
			push_children(S.stack, sp, open_int, nchild, child);
			// opened bundles -> bundle queue
			const unsigned bb = __ballot_sync(0xFFFFFFFFu, open_bundle);
			if (open_bundle) S.bq[__popc(bb & lt)] = make_int2(child, nchild);
			__syncwarp();
			const int nb = __popc(bb);
			for (int b = 0; b < nb; b++) {
				const int2 q = S.bq[b];
				for (int o = 0; o < q.y; o += 32) {
					const int j = o + lane;
					const bool have = j < q.y;
					float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
					bool wr = false, nr = false;
					if (have) {
						const int64_t jp = (int64_t) q.x + j;
						e.x = ioff(ix[jp], g.cx, p.scale);
						e.y = ioff(iy[jp], g.cy, p.scale);
						e.z = ioff(iz[jp], g.cz, p.scale);
						e.w = p.gravity * mass_f[jp];
						const float ax = fmaxf(fabsf(e.x) - g.hx, 0.f), ay = fmaxf(fabsf(e.y) - g.hy, 0.f),
						            az = fmaxf(fabsf(e.z) - g.hz, 0.f);
						nr = ax * ax + ay * ay + az * az < p.near2;
						wr = per_target && (fabsf(e.x) > wlimx || fabsf(e.y) > wlimy || fabsf(e.z) > wlimz);
					}
					const bool tm = have && !wr && !nr, tw = have && (wr || nr);
					if (wr) e.w = -e.w;
					const unsigned m1 = __ballot_sync(0xFFFFFFFFu, tm), m2 = __ballot_sync(0xFFFFFFFFu, tw);
					if (nl + __popc(m1) > GW_LIST) {
						flush_far<TPL>(S, nl, t);
						nl = 0;
						__syncwarp();
					}
					if (nw + __popc(m2) > GW_WLIST) {
						flush_slow<TPL>(p, S.wlist, nw, t);
						nw = 0;
						__syncwarp();
					}
					if (tm) far_put(S, nl + __popc(m1 & lt), e);
					if (tw) S.wlist[nw + __popc(m2 & lt)] = e;
					nl += __popc(m1);
					nw += __popc(m2);
					__syncwarp();
				}
			}
			__syncwarp();
		}
	}
	__syncwarp();
	flush_far<TPL>(S, nl, t);
	flush_slow<TPL>(p, S.wlist, nw, t);
	if (QUAD) flush_quad<TPL>(*QL, nq, t);
#pragma unroll
	for (int k = 0; k < TPL; k++) t[k].cost -= 1.f;     // the self pair, which the reference skips
	__syncwarp();
}

template <int MODE, int TPL, typename F, bool QUAD>
__global__ void __launch_bounds__(GW_THREADS, GW_WALK_MINB)
k_walk_group(GroupParams p, const int32_t *__restrict__ active, const int32_t *__restrict__ gfirst,
             const tvg_wnode *__restrict__ wt, const float4 *__restrict__ wq,
             const uint32_t *__restrict__ ix, const uint32_t *__restrict__ iy,
             const uint32_t *__restrict__ iz, const float *__restrict__ mass_f,
             const float *__restrict__ last_acc, F *acc0, F *acc1, F *acc2, F *gacc0, F *gacc1,
             F *gacc2, F *cost_out, int32_t *work, double *counter, int *status)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	WarpSmem &S = ((WarpSmem *) smem_raw)[threadIdx.x >> 5];
	QuadList *QL = QUAD ? ((QuadList *) (smem_raw + sizeof(WarpSmem) * GW_WARPS)) + (threadIdx.x >> 5)
	                    : nullptr;
	const int lane = threadIdx.x & 31;
	double cnt_acc = 0, qcnt_acc = 0;
	const int64_t ngroups = p.dc->ngroups;
	for (;;) {
		int64_t g = 0;
		if (lane == 0) g = atomicAdd(work, 1);
		g = __shfl_sync(0xFFFFFFFFu, g, 0);
		if (g >= ngroups) break;
		int64_t first;
		int cnt;
		if (gfirst) {
			first = gfirst[g];
			cnt = (int) (gfirst[g + 1] - first);
		} else {
			first = g * p.gsize;
			cnt = (int) min((int64_t) p.gsize, p.n - first);
		}
		Target t[TPL];
		walk_group<MODE, TPL, QUAD>(p, S, wt, ix, iy, iz, mass_f, last_acc, first, cnt, active, t, QL, wq,
		                            status);
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			if (!t[k].valid) continue;
			const int slot = lane + 32 * k;
			const int64_t i = active ? (int64_t) active[first + slot] : first + slot;
			acc0[i] += (F) t[k].ax;
			acc1[i] += (F) t[k].ay;
			acc2[i] += (F) t[k].az;
			gacc0[i] = (F) t[k].ax;
			gacc1[i] = (F) t[k].ay;
			gacc2[i] = (F) t[k].az;
			cost_out[i] = (F) t[k].cost;
			cnt_acc += t[k].cost;
			qcnt_acc += t[k].qcost;
		}
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		cnt_acc += __shfl_xor_sync(0xFFFFFFFFu, cnt_acc, o);
		qcnt_acc += __shfl_xor_sync(0xFFFFFFFFu, qcnt_acc, o);
	}
	if (lane == 0 && cnt_acc != 0) atomicAdd(counter, cnt_acc);
	if (QUAD && lane == 0 && qcnt_acc != 0) atomicAdd(counter + 2, qcnt_acc);
}

// ------------------------------------------------------ the Ewald walk

// 4-point Lagrange basis on the nodes -1, 0, 1, 2 at t in [0, 1]: weights,
// first and second derivatives
__device__ __forceinline__ void lagrange4(float t, float w[4], float d[4], float dd[4])
{
	const float t2 = t * t, t3 = t2 * t;
	w[0] = (-t3 + 3.f * t2 - 2.f * t) * (1.f / 6.f);
	w[1] = (t3 - 2.f * t2 - t + 2.f) * 0.5f;
	w[2] = (-t3 + t2 + 2.f * t) * 0.5f;
	w[3] = (t3 - t) * (1.f / 6.f);
	d[0] = (-3.f * t2 + 6.f * t - 2.f) * (1.f / 6.f);
	d[1] = (3.f * t2 - 4.f * t - 1.f) * 0.5f;
	d[2] = (-3.f * t2 + 2.f * t + 2.f) * 0.5f;
	d[3] = (3.f * t2 - 1.f) * (1.f / 6.f);
	dd[0] = 1.f - t;
	dd[1] = 3.f * t - 2.f;
	dd[2] = 1.f - 3.f * t;
	dd[3] = t;
}

// The lattice-minus-image force T(x) (box units, unit G m, target at x from
// the source) is tabulated on x = 0.5 i / 64, i = -1..66 per axis (one ghost
// layer below 0 and the analytic continuation beyond 1/2), interleaved
// (Tx, Ty, Tz, 0). The correction for a source at d from the target is
// K(d) = -G m T(d / L) / L^2 (the reference's sign rule, periodic.c:100-112),
// looked up at |d| with the symmetries T_a(.., -x_b, ..) = -T_a if a = b,
// +T_a otherwise.

// K(d), its Jacobian J and Hessian H, summed into c, from the Taylor table
// (tvg_ewald.cu, k_ewald_taylor): the record of the node nearest to |d| holds
// T and its first three derivatives in node units; with D = d3T . du, the
// value is T + du . (dT + 1/2 (d2T + D/3) du), the gradient dT + (d2T + D/2)
// du and the second derivatives d2T + D (exact for a cubic). With OVR the
// value is ovr (T at |d| from the learned correction) instead.
// K_a = -s_a T_a, J_ab = -s_a s_b g dT_a/du_b, H_abc = -s_a s_b s_c g^2
// d2T_a/du_b du_c, all times G m / L^2 (s the signs of d, g node spacings per
// length).
// index of the Taylor-table record nearest to |d| (node units)
__device__ __forceinline__ int taylor_record(const GroupParams &p, float4 e)
{
	const int i = min(__float2int_rn(fabsf(e.x) * p.tay_grid), TVG_TAYLOR_NODES - 1);
	const int j = min(__float2int_rn(fabsf(e.y) * p.tay_grid), TVG_TAYLOR_NODES - 1);
	const int l = min(__float2int_rn(fabsf(e.z) * p.tay_grid), TVG_TAYLOR_NODES - 1);
	return (i * TVG_TAYLOR_NODES + j) * TVG_TAYLOR_NODES + l;
}

// STAGED: the record is `staged` (shared memory) instead of the table entry.
// SQ (TVG_CFG_QUADRUPOLE): srcq is the source node's stored -G Q (two float4,
// null for a particle), and the value also takes the node's quadrupole term,
// the second-order term of the expansion about its centre of mass:
// sum_j m_j y_b y_c / 2 d2K_a/dd_b dd_c = Q_bc / 6 d2K_a/dd_b dd_c (d2K_a is
// traceless: the lattice sum's divergence is constant away from the source).
template <bool OVR, bool STAGED = false, bool SQ = false>
__device__ __forceinline__ void ewald_kjh_taylor(const GroupParams &p, const float4 *__restrict__ tay,
                                                 float4 e, CorrSum &c, const float *ovr,
                                                 const float4 *staged = nullptr,
                                                 const float4 *__restrict__ srcq = nullptr)
{
	const float sg[3] = { e.x < 0.f ? -1.f : 1.f, e.y < 0.f ? -1.f : 1.f, e.z < 0.f ? -1.f : 1.f };
	const float u = fabsf(e.x) * p.tay_grid, v = fabsf(e.y) * p.tay_grid, w = fabsf(e.z) * p.tay_grid;
	const int i = min(__float2int_rn(u), TVG_TAYLOR_NODES - 1);
	const int j = min(__float2int_rn(v), TVG_TAYLOR_NODES - 1);
	const int l = min(__float2int_rn(w), TVG_TAYLOR_NODES - 1);
	const float du = u - (float) i, dv = v - (float) j, dw = w - (float) l;
	const float4 *rec = STAGED ? staged : tay + 16 * ((i * TVG_TAYLOR_NODES + j) * TVG_TAYLOR_NODES + l);
	const float m0 = -e.w * p.inv_box * p.inv_box, m1 = m0 * p.tay_grid, m2 = m1 * p.tay_grid;
	float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = q0;
	if (SQ && srcq) {
		q0 = __ldg(srcq);
		q1 = __ldg(srcq + 1);
		q0.w *= 2.f * sg[0] * sg[1];      // both off-diagonal terms, with their signs
		q1.x *= 2.f * sg[0] * sg[2];
		q1.y *= 2.f * sg[1] * sg[2];
	}
	const float mq = p.tay_grid * p.tay_grid * p.inv_box * p.inv_box * (1.f / 6.f);
#pragma unroll
	for (int q = 0; q < 3; q++) {
		float4 r0, r1, r2, r3, r4;
		if (STAGED) {
			r0 = rec[5 * q]; r1 = rec[5 * q + 1]; r2 = rec[5 * q + 2]; r3 = rec[5 * q + 3]; r4 = rec[5 * q + 4];
		} else {
			r0 = __ldg(rec + 5 * q); r1 = __ldg(rec + 5 * q + 1); r2 = __ldg(rec + 5 * q + 2);
			r3 = __ldg(rec + 5 * q + 3); r4 = __ldg(rec + 5 * q + 4);
		}
		// D_bc = sum_d d3T_bcd du_d
		const float dxx = fmaf(r2.z, du, fmaf(r3.y, dv, r3.z * dw));
		const float dyy = fmaf(r3.w, du, fmaf(r2.w, dv, r4.x * dw));
		const float dzz = fmaf(r4.y, du, fmaf(r4.z, dv, r3.x * dw));
		const float dxy = fmaf(r3.y, du, fmaf(r3.w, dv, r4.w * dw));
		const float dxz = fmaf(r3.z, du, fmaf(r4.w, dv, r4.y * dw));
		const float dyz = fmaf(r4.w, du, fmaf(r4.x, dv, r4.z * dw));
		const float hxx = r1.x + dxx, hyy = r1.y + dyy, hzz = r1.z + dzz;
		const float hxy = r1.w + dxy, hxz = r2.x + dxz, hyz = r2.y + dyz;
		// gradient: dT + (d2T + D/2) du
		const float gx = r0.y + fmaf(fmaf(0.5f, dxx, r1.x), du, fmaf(fmaf(0.5f, dxy, r1.w), dv,
		                              fmaf(0.5f, dxz, r2.x) * dw));
		const float gy = r0.z + fmaf(fmaf(0.5f, dxy, r1.w), du, fmaf(fmaf(0.5f, dyy, r1.y), dv,
		                              fmaf(0.5f, dyz, r2.y) * dw));
		const float gz = r0.w + fmaf(fmaf(0.5f, dxz, r2.x), du, fmaf(fmaf(0.5f, dyz, r2.y), dv,
		                              fmaf(0.5f, dzz, r1.z) * dw));
		// value: T + du . (dT + 1/2 (d2T + D/3) du)
		const float t3 = 1.f / 3.f;
		const float bx = fmaf(fmaf(t3, dxx, r1.x), du, fmaf(fmaf(t3, dxy, r1.w), dv, fmaf(t3, dxz, r2.x) * dw));
		const float by = fmaf(fmaf(t3, dxy, r1.w), du, fmaf(fmaf(t3, dyy, r1.y), dv, fmaf(t3, dyz, r2.y) * dw));
		const float bz = fmaf(fmaf(t3, dxz, r2.x), du, fmaf(fmaf(t3, dyz, r2.y), dv, fmaf(t3, dzz, r1.z) * dw));
		const float val = OVR ? ovr[q]
		                      : r0.x + fmaf(fmaf(0.5f, bx, r0.y), du, fmaf(fmaf(0.5f, by, r0.z), dv,
		                                                                    fmaf(0.5f, bz, r0.w) * dw));
		const float sq = sg[q];
		c.k[q] = fmaf(m0 * sq, val, c.k[q]);
		if (SQ) {
			// per unit G m, d2K_a/dd_b dd_c = -s_a s_b s_c h_bc tay_grid^2 / L^2;
			// with G Q = -(stored), the term is mq s_a sum_bc stored_bc s_b s_c h_bc
			const float hq = fmaf(q0.x, hxx, fmaf(q0.y, hyy, fmaf(q0.z, hzz,
			                 fmaf(q0.w, hxy, fmaf(q1.x, hxz, q1.y * hyz)))));
			c.k[q] = fmaf(mq * sq, hq, c.k[q]);
		}
		c.j[3 * q + 0] = fmaf(m1 * sq * sg[0], gx, c.j[3 * q + 0]);
		c.j[3 * q + 1] = fmaf(m1 * sq * sg[1], gy, c.j[3 * q + 1]);
		c.j[3 * q + 2] = fmaf(m1 * sq * sg[2], gz, c.j[3 * q + 2]);
		c.h[6 * q + 0] = fmaf(m2 * sq, hxx, c.h[6 * q + 0]);
		c.h[6 * q + 1] = fmaf(m2 * sq, hyy, c.h[6 * q + 1]);
		c.h[6 * q + 2] = fmaf(m2 * sq, hzz, c.h[6 * q + 2]);
		c.h[6 * q + 3] = fmaf(m2 * sq * sg[0] * sg[1], hxy, c.h[6 * q + 3]);
		c.h[6 * q + 4] = fmaf(m2 * sq * sg[0] * sg[2], hxz, c.h[6 * q + 4]);
		c.h[6 * q + 5] = fmaf(m2 * sq * sg[1] * sg[2], hyz, c.h[6 * q + 5]);
	}
}

// K(d) alone (tricubic value of the extended table), for per-target
// evaluation, added to a
__device__ __forceinline__ void ewald_k(const GroupParams &p, const float4 *__restrict__ tab, float ex,
                                        float ey, float ez, float gm, float &ax, float &ay, float &az)
{
	const float sx = ex < 0.f ? -1.f : 1.f, sy = ey < 0.f ? -1.f : 1.f, sz = ez < 0.f ? -1.f : 1.f;
	const float u = fabsf(ex) * p.grid, v = fabsf(ey) * p.grid, w = fabsf(ez) * p.grid;
	const int i = min((int) u, 64), j = min((int) v, 64), l = min((int) w, 64);
	float wx[4], wy[4], wz[4], d_[4], dd_[4];
	lagrange4(u - (float) i, wx, d_, dd_);
	lagrange4(v - (float) j, wy, d_, dd_);
	lagrange4(w - (float) l, wz, d_, dd_);
	float vx = 0.f, vy = 0.f, vz = 0.f;
	const int base = (i * 68 + j) * 68 + l;
#pragma unroll 1
	for (int a = 0; a < 4; a++) {
		float yx = 0.f, yy = 0.f, yz = 0.f;
#pragma unroll
		for (int b = 0; b < 4; b++) {
			const float4 *row = tab + base + (a * 68 + b) * 68;
			const float4 t0 = __ldg(row), t1 = __ldg(row + 1), t2 = __ldg(row + 2), t3 = __ldg(row + 3);
			yx = fmaf(wy[b], wz[0] * t0.x + wz[1] * t1.x + wz[2] * t2.x + wz[3] * t3.x, yx);
			yy = fmaf(wy[b], wz[0] * t0.y + wz[1] * t1.y + wz[2] * t2.y + wz[3] * t3.y, yy);
			yz = fmaf(wy[b], wz[0] * t0.z + wz[1] * t1.z + wz[2] * t2.z + wz[3] * t3.z, yz);
		}
		vx = fmaf(wx[a], yx, vx);
		vy = fmaf(wx[a], yy, vy);
		vz = fmaf(wx[a], yz, vz);
	}
	const float m0 = -gm * p.inv_box * p.inv_box;
	ax = fmaf(m0 * sx, vx, ax);
	ay = fmaf(m0 * sy, vy, ay);
	az = fmaf(m0 * sz, vz, az);
}

// bound of |d2 T| (box units) within distance r (box units) of the source:
// 92 at the face centres, growing as (2 r)^1.5 from 7 at r = 0.1
__device__ __forceinline__ float ewald_h2(float r)
{
	const float x = fminf(2.f * r, 1.f);
	return 92.f * x * sqrtf(x);
}

// bound of |d3 T| (box units) within distance r of the source: 75 near the
// source (the lattice sum's cubic term), 753 at the face centres; 77 + 680
// (2 r)^4 bounds the table's third derivatives at every node
__device__ __forceinline__ float ewald_h3(float r)
{
	const float x = fminf(2.f * r, 1.f), x2 = x * x;
	return fmaf(680.f, x2 * x2, 77.f);
}

// The field of the uniform unit-density cube [-1/2, 1/2]^3 (G = 1) beyond its
// linear term, R_a(tau) = g_a(tau) + 4 pi tau_a / 3, as the degree-7 odd
// polynomial of tvg_uniform_cube.inc (fitted to the prism closed form, Nagy
// 1966, within 2e-8 of max |R| for |tau_i| <= 0.06), a the component and b, c
// the other two coordinates
#include "tvg_uniform_cube.inc"

__device__ __forceinline__ double uniform_cube_poly(double a, double b, double c)
{
	const double A = a * a, B = b * b, C = c * c;
	const double s1 = B + C, s2 = B * B + C * C, p = B * C;
	const double d3 = kUniformCube[0] * s1 + kUniformCube[1] * A;
	const double d5 = kUniformCube[2] * s2 + kUniformCube[3] * p + A * (kUniformCube[4] * s1 + kUniformCube[5] * A);
	const double d7 = kUniformCube[6] * (B * B * B + C * C * C) + kUniformCube[7] * p * s1
	                + A * (kUniformCube[8] * s2 + kUniformCube[9] * p
	                       + A * (kUniformCube[10] * s1 + kUniformCube[11] * A));
	return a * (d3 + d5 + d7);
}

// The expansion about the group centre misses the third and higher orders of
// the correction's sum. Over the uniform part of the sources -- the cube of
// side L about the centre, where every source sits at its image nearest to
// the centre -- that sum is -G rho g_cube(t) (the lattice force has zero
// mean over a period), whose part beyond the linear term is added:
// R(t) = -(G M / L^2) [g(t / L) + 4 pi t / (3 L)] (g of the unit cube). The
// expansion is used for groups narrower than L / 20 only.
__device__ __forceinline__ void uniform_remainder(const GroupParams &p, double tx, double ty,
                                                  double tz, double out[3])
{
	const double x = tx * p.inv_box, y = ty * p.inv_box, z = tz * p.inv_box;
	const double u = p.uniform_g * p.dc->mass_total;
	out[0] = -u * uniform_cube_poly(x, y, z);
	out[1] = -u * uniform_cube_poly(y, x, z);
	out[2] = -u * uniform_cube_poly(z, x, y);
}

// the learned correction for per-target images (groups wider than L/20,
// rare): out of line, so that its registers do not add to the walk's
__device__ __noinline__ void mlp_forward_warp_call(const float *mlp, const uint32_t *w2b, const float x[3],
                                                   float out[3])
{
	mlp_forward_warp(mlp, w2b, x, out);
}

// Evaluates list entries [from, from + cnt), 1 <= cnt <= 32 (every lane of
// the warp calls): about the group centre one entry per lane (K, J, H), or,
// for a group that takes per-target images, every entry for every target of
// the lane (K at the target's nearest image; FP32 per batch, carried in
// FP64). With the learned correction the value of K comes from the warp's
// tensor-core evaluation of the network (one point per lane).
// wq (TVG_CFG_QUADRUPOLE, groups without per-target images): the walk
// nodes' stored quadrupoles, lnode the list entries' nodes
template <int TPL, bool MLP>
__device__ __forceinline__ void ewald_batch(const GroupParams &p, const float4 *tab, const float4 *tay,
                                            const float *mlp, const uint32_t *w2b, const float4 *list,
                                            int from, int cnt, bool per_target, CorrSum &c,
                                            Target (&t)[TPL], float &nev,
                                            const int32_t *lnode = nullptr,
                                            const float4 *__restrict__ wq = nullptr)
{
	const int lane = threadIdx.x & 31;
	if (!per_target) {
		const float4 *srcq = nullptr;
		if (wq && lane < cnt) {
			const int nd = lnode[from + lane];
			srcq = nd >= 0 ? wq + 2 * (int64_t) nd : nullptr;
		}
		if (MLP) {
			// lanes past cnt repeat the last entry and drop the result
			const float4 e = list[from + min(lane, cnt - 1)];
			const float xs[3] = { fabsf(e.x) * p.inv_box, fabsf(e.y) * p.inv_box, fabsf(e.z) * p.inv_box };
			float tv[3];
			mlp_forward_warp(mlp, w2b, xs, tv);
			if (lane < cnt) {
				if (wq) ewald_kjh_taylor<true, false, true>(p, tay, e, c, tv, nullptr, srcq);
				else ewald_kjh_taylor<true>(p, tay, e, c, tv);
				nev += 1.f;
			}
		} else if (lane < cnt) {
			if (wq) ewald_kjh_taylor<false, false, true>(p, tay, list[from + lane], c, nullptr, nullptr, srcq);
			else ewald_kjh_taylor<false>(p, tay, list[from + lane], c, nullptr);
			nev += 1.f;
		}
	} else {
		float ax[TPL], ay[TPL], az[TPL];
#pragma unroll
		for (int k = 0; k < TPL; k++) ax[k] = ay[k] = az[k] = 0.f;
		for (int e = 0; e < cnt; e++) {
			const float4 s = list[from + e];
#pragma unroll
			for (int k = 0; k < TPL; k++) {
				const float dx = wrap_half(s.x - t[k].tx, p.box, p.half_box);
				const float dy = wrap_half(s.y - t[k].ty, p.box, p.half_box);
				const float dz = wrap_half(s.z - t[k].tz, p.box, p.half_box);
				if (MLP) {
					const float xs[3] = { fabsf(dx) * p.inv_box, fabsf(dy) * p.inv_box, fabsf(dz) * p.inv_box };
					float tv[3];
					mlp_forward_warp_call(mlp, w2b, xs, tv);
					const float m0 = -s.w * p.inv_box * p.inv_box;
					ax[k] = fmaf(dx < 0.f ? -m0 : m0, tv[0], ax[k]);
					ay[k] = fmaf(dy < 0.f ? -m0 : m0, tv[1], ay[k]);
					az[k] = fmaf(dz < 0.f ? -m0 : m0, tv[2], az[k]);
				} else {
					ewald_k(p, tab, dx, dy, dz, s.w, ax[k], ay[k], az[k]);
				}
				if (t[k].valid) nev += 1.f;
			}
		}
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			t[k].ax += (double) ax[k];
			t[k].ay += (double) ay[k];
			t[k].az += (double) az[k];
		}
	}
}

// pipeline state of a warp's record stage (uniform across its lanes)
struct StageState {
	uint32_t phase;    // bit b: parity of buffer b's next completion
	int cur;           // the buffer the next batch goes to
	bool pending;      // the other buffer holds an issued batch
	bool ok;           // false after a wait gave up: no more staging
};

// bounded wait for buffer b's copies (TVG_ST_TIMEOUT when they never land)
__device__ __forceinline__ bool stage_wait(EwaldStage *st, int b, StageState &ss, int *status)
{
	const uint32_t par = (ss.phase >> b) & 1u;
	for (int it = 0; !mbar_try_wait(&st->bar[b], par);) {
		if (++it > (1 << 20)) {
			atomicOr(status, TVG_ST_TIMEOUT);
			ss.ok = false;
			return false;
		}
	}
	ss.phase ^= 1u << b;
	return true;
}

__device__ __forceinline__ void stage_eval(const GroupParams &p, EwaldStage *st, int b, CorrSum &c, float &nev)
{
	const int lane = threadIdx.x & 31;
	ewald_kjh_taylor<false, true>(p, nullptr, st->pend[b][lane], c, nullptr, &st->rec[b][lane][0]);
	nev += 1.f;
}

// a full batch of 32 sources (list[from + lane]) goes to the free buffer;
// then the batch issued before it is evaluated. Every lane copies its own
// record; lane 0 posts the batch's 8 KB on the buffer's barrier first.
__device__ __forceinline__ void stage_batch(const GroupParams &p, const float4 *__restrict__ tay,
                                            EwaldStage *st, const float4 *list, int from, StageState &ss,
                                            CorrSum &c, float &nev, int *status)
{
	const int lane = threadIdx.x & 31;
	const float4 e = list[from + lane];
	const int b = ss.cur;
	if (lane == 0) mbar_arrive_expect_tx(&st->bar[b], 32 * 16 * sizeof(float4));
	__syncwarp();
	st->pend[b][lane] = e;
	// this lane read the slot as generic memory when the buffer was last
	// evaluated: order that before the bulk copy writes it
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
	bulk_g2s(&st->rec[b][lane][0], tay + 16 * taylor_record(p, e), 16 * sizeof(float4), &st->bar[b]);
	if (ss.pending && stage_wait(st, b ^ 1, ss, status)) stage_eval(p, st, b ^ 1, c, nev);
	ss.pending = true;
	ss.cur = b ^ 1;
	__syncwarp();
}

// evaluates the batch still in flight (end of a group)
__device__ __forceinline__ void stage_drain(const GroupParams &p, EwaldStage *st, StageState &ss, CorrSum &c,
                                            float &nev, int *status)
{
	if (ss.pending && stage_wait(st, ss.cur ^ 1, ss, status)) stage_eval(p, st, ss.cur ^ 1, c, nev);
	ss.pending = false;
	__syncwarp();
}

template <int TPL, bool MLP>
__device__ void ewald_group(const GroupParams &p, EwaldSmem &S, const tvg_wnode *__restrict__ wt,
                            const uint32_t *__restrict__ ix, const uint32_t *__restrict__ iy,
                            const uint32_t *__restrict__ iz, const float *__restrict__ mass_f,
                            const float *__restrict__ last_acc, const float4 *__restrict__ tab,
                            const float4 *__restrict__ tay, const float *mlp, const uint32_t *w2b,
                            int64_t first, int cnt, const int32_t *__restrict__ active,
                            Target (&t)[TPL], float &nev, EwaldStage *st, StageState &ss, int *status,
                            const float4 *__restrict__ wq_all)
{
	const int lane = threadIdx.x & 31;
	const unsigned lt = (1u << lane) - 1u;
	GroupBox g;
	group_setup<TPL>(p, ix, iy, iz, last_acc, active, first, cnt, t, g);
	const float hmax = fmaxf(g.hx, fmaxf(g.hy, g.hz));
	// the gravity walk makes the same choice (walk_group)
	const bool per_target = hmax >= p.taylor_h;
	// node quadrupoles (TVG_CFG_QUADRUPOLE) in the expansion about the group
	// centre; per-target images evaluate K alone and keep monopoles
	const float4 *wq = per_target ? nullptr : wq_all;
	if (wq) st = nullptr;
	// straddling: the node (and, with per-target images, the group box) reaches
	// the half-box plane; then the gravity walk's decision is repeated
	const float margin = 8.f * p.scale;
	const float ex = per_target ? g.hx : 0.f, ey = per_target ? g.hy : 0.f,
	            ez = per_target ? g.hz : 0.f;
	CorrSum c;
#pragma unroll
	for (int a = 0; a < 3; a++) c.k[a] = 0.f;
#pragma unroll
	for (int a = 0; a < 9; a++) c.j[a] = 0.f;
#pragma unroll
	for (int a = 0; a < 18; a++) c.h[a] = 0.f;

	int sp = 0, nl = 0, r0 = 0;
	const int ntop = p.dc->ntop;
	int guard = 0;
	bool final = false;
	// One loop step pops up to 32 nodes, lists the accepted ones and queues
	// the opened bundles; then the drain below evaluates every full batch of
	// 32 sources (at the end the rest too) and lists the next 32 particles of
	// the queued bundles, so that the evaluation is inlined once in the loop.
	for (;;) {
		int nb = 0;
		if (sp == 0 && !final) {
			// the roots in chunks of GW_ROOTS (a balanced decomposition can have
			// thousands of top nodes, more than the stack holds at once)
			if (r0 < ntop) {
				const int nr = min(GW_ROOTS, ntop - r0);
				for (int r = lane; r < nr; r += 32) S.stack[r] = r0 + r;
				sp = nr;
				r0 += GW_ROOTS;
				__syncwarp();
			} else {
				final = true;
			}
		}
		if (!final && ++guard > p.max_iter) {
			atomicOr(status, TVG_ST_TIMEOUT);
			final = true;
		}
		if (!final) {
			bool stop;
			const int node = pop_nodes(S.stack, sp, status, stop);
			if (stop) {
				final = true;
			} else {
				bool accept = false, open_int = false, open_bundle = false;
				float4 entry = make_float4(0.f, 0.f, 0.f, 0.f);
				int nchild = 0, child = 0;
				if (node >= 0) {
					const tvg_wnode nd = wt[node];
					const float dx = ioff(nd.cx, g.cx, p.scale), dy = ioff(nd.cy, g.cy, p.scale),
					            dz = ioff(nd.cz, g.cz, p.scale);
					const float gx = ioff(nd.gx, g.cx, p.scale), gy = ioff(nd.gy, g.cy, p.scale),
					            gz = ioff(nd.gz, g.cz, p.scale);
					const float hs = 0.5f * nd.size + margin;
					const bool straddle = fabsf(gx) + hs + ex > p.half_box || fabsf(gy) + hs + ey > p.half_box
					                   || fabsf(gz) + hs + ez > p.half_box;
					bool open;
					if (straddle) {
						float r2;
						open = gravity_opens(p, g, nd, node, dx, dy, dz, gx, gy, gz, r2, p.quad && !per_target);
					} else {
						// monopole error of K: G M h2 s^2 / (8 L^4) (s^2 / 4: the mean square
						// offset of a uniform cube's mass from its centre); with the node's
						// quadrupole the next term, G M h3 s^3 / (48 L^5) (s / 2 per axis)
						const float rfar = (sqrtf(gx * gx + gy * gy + gz * gz) + nd.size + hmax) * p.inv_box;
						const float l2 = p.inv_box * p.inv_box;
						const float hs2 = ewald_h2(rfar) * nd.size2 * l2;     // h2 s^2 / L^2
						if (p.use_bh) open = hs2 > p.ew_bh;
						else if (wq) {
							const float sl = nd.size * p.inv_box;
							open = nd.mass * ewald_h3(rfar) * sl * sl * sl * (1.f / 48.f) * l2 > p.ew_rel * g.fac;
						} else open = nd.mass * hs2 * 0.125f * l2 > p.ew_rel * g.fac;
					}
					if (!open) {
						accept = true;
						entry = make_float4(dx, dy, dz, p.gravity * nd.mass);
					} else if (nd.nchild > 0) {
						open_int = true;
						nchild = nd.nchild;
						child = nd.child;
					} else {
						open_bundle = true;
						nchild = -nd.nchild;
						child = nd.child;
					}
				}
				const unsigned bm = __ballot_sync(0xFFFFFFFFu, accept);
				if (accept) {
					S.list[nl + __popc(bm & lt)] = entry;
					S.lnode[nl + __popc(bm & lt)] = node;
				}
				nl += __popc(bm);       // below 64: the drain left fewer than 32
				push_children(S.stack, sp, open_int, nchild, child);
				const unsigned bb = __ballot_sync(0xFFFFFFFFu, open_bundle);
				if (open_bundle) S.bq[__popc(bb & lt)] = make_int2(child, nchild);
				nb = __popc(bb);
				__syncwarp();
			}
		}
		int b = 0, o = 0;
		for (;;) {
			const bool full = nl >= 32;
			if (full || (final && nl > 0)) {
				const int cnt = full ? 32 : nl;
				if (full && st && ss.ok && !per_target) stage_batch(p, tay, st, S.list, nl - 32, ss, c, nev, status);
				else ewald_batch<TPL, MLP>(p, tab, tay, mlp, w2b, S.list, nl - cnt, cnt, per_target, c, t, nev,
				                           S.lnode, wq);
				nl -= cnt;
				continue;
			}
			if (b >= nb) break;
			// the next 32 particles of queued bundle b
			const int2 q = S.bq[b];
			const int jj = o + lane;
			const bool have = jj < q.y;
			float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
			if (have) {
				const int64_t jp = (int64_t) q.x + jj;
				e = make_float4(ioff(ix[jp], g.cx, p.scale), ioff(iy[jp], g.cy, p.scale),
				                ioff(iz[jp], g.cz, p.scale), p.gravity * mass_f[jp]);
			}
			const unsigned mb = __ballot_sync(0xFFFFFFFFu, have);
			if (have) {
				S.list[nl + __popc(mb & lt)] = e;
				S.lnode[nl + __popc(mb & lt)] = -1;
			}
			nl += __popc(mb);
			__syncwarp();
			o += 32;
			if (o >= q.y) {
				b++;
				o = 0;
			}
		}
		__syncwarp();
		if (final) break;
	}
	if (st && ss.ok) stage_drain(p, st, ss, c, nev, status);
	if (per_target) return;
	// sum over lanes (FP64), then K(d_c - t) ~ K - J t + H:tt / 2 per target
	double K[3], J[9], H[18];
#pragma unroll
	for (int a = 0; a < 3; a++) K[a] = c.k[a];
#pragma unroll
	for (int a = 0; a < 9; a++) J[a] = c.j[a];
#pragma unroll
	for (int a = 0; a < 18; a++) H[a] = c.h[a];
#pragma unroll
	for (int o = 16; o; o >>= 1) {
#pragma unroll
		for (int a = 0; a < 3; a++) K[a] += __shfl_xor_sync(0xFFFFFFFFu, K[a], o);
#pragma unroll
		for (int a = 0; a < 9; a++) J[a] += __shfl_xor_sync(0xFFFFFFFFu, J[a], o);
#pragma unroll
		for (int a = 0; a < 18; a++) H[a] += __shfl_xor_sync(0xFFFFFFFFu, H[a], o);
	}
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		const double x = t[k].tx, y = t[k].ty, z = t[k].tz;
		double out[3];
#pragma unroll
		for (int a = 0; a < 3; a++) {
			const double *h = H + 6 * a;
			out[a] = K[a] - (J[3 * a] * x + J[3 * a + 1] * y + J[3 * a + 2] * z)
			       + 0.5 * (h[0] * x * x + h[1] * y * y + h[2] * z * z)
			       + h[3] * x * y + h[4] * x * z + h[5] * y * z;
		}
		double rem[3];
		uniform_remainder(p, x, y, z, rem);
		out[0] += rem[0];
		out[1] += rem[1];
		out[2] += rem[2];
		t[k].ax = out[0];
		t[k].ay = out[1];
		t[k].az = out[2];
	}
}

template <int TPL, bool MLP, typename F>
__global__ void __launch_bounds__(GE_THREADS, MLP ? 1 : GW_EWALD_MINB)
k_ewald_group(GroupParams p, const int32_t *__restrict__ active, const int32_t *__restrict__ gfirst,
              const tvg_wnode *__restrict__ wt,
              const uint32_t *__restrict__ ix, const uint32_t *__restrict__ iy,
              const uint32_t *__restrict__ iz, const float *__restrict__ mass_f,
              const float *__restrict__ last_acc, const float4 *__restrict__ tab,
              const float4 *__restrict__ tay, const __nv_bfloat16 *__restrict__ mlp_w,
              const float *__restrict__ mlp_f32, F *acc0, F *acc1,
              F *acc2, F *gacc0, F *gacc1, F *gacc2, int32_t *work, double *counter, int *status,
              const float4 *__restrict__ wq)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	EwaldSmem &S = ((EwaldSmem *) smem_raw)[threadIdx.x >> 5];
	// the learned correction's parameters, once per block: the network BF16 ->
	// FP32, the fitted cubic and scale FP32, and W2 as BF16 pairs for the MMAs
	float *mlp = (float *) (smem_raw + sizeof(EwaldSmem) * GE_WARPS);
	uint32_t *w2b = (uint32_t *) (mlp + MLP_NPARAM);
	if (MLP) {
		mlp_load_shared(mlp_w, mlp_f32, mlp, w2b);
		__syncthreads();
	}
	const int lane = threadIdx.x & 31;
	// with GW_EWALD_STAGE the table path stages its records (EwaldStage after
	// the warps' areas)
	EwaldStage *st = (MLP || !GW_EWALD_STAGE)
	                     ? nullptr
	                     : ((EwaldStage *) (smem_raw + sizeof(EwaldSmem) * GE_WARPS)) + (threadIdx.x >> 5);
	StageState ss = { 0u, 0, false, true };
	if (st) {
		if (lane == 0) {
			mbar_init(&st->bar[0], 1);
			mbar_init(&st->bar[1], 1);
			asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		}
		__syncwarp();
	}
	double ev_acc = 0;
	const int64_t ngroups = p.dc->ngroups;
	for (;;) {
		int64_t g = 0;
		if (lane == 0) g = atomicAdd(work, 1);
		g = __shfl_sync(0xFFFFFFFFu, g, 0);
		if (g >= ngroups) break;
		int64_t first;
		int cnt;
		if (gfirst) {
			first = gfirst[g];
			cnt = (int) (gfirst[g + 1] - first);
		} else {
			first = g * p.gsize;
			cnt = (int) min((int64_t) p.gsize, p.n - first);
		}
		Target t[TPL];
		float nev = 0.f;
		ewald_group<TPL, MLP>(p, S, wt, ix, iy, iz, mass_f, last_acc, tab, tay, mlp, w2b, first, cnt, active, t, nev,
		                 st, ss, status, wq);
		ev_acc += nev;
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			if (!t[k].valid) continue;
			const int slot = lane + 32 * k;
			const int64_t i = active ? (int64_t) active[first + slot] : first + slot;
			acc0[i] += (F) t[k].ax;
			acc1[i] += (F) t[k].ay;
			acc2[i] += (F) t[k].az;
			gacc0[i] += (F) t[k].ax;
			gacc1[i] += (F) t[k].ay;
			gacc2[i] += (F) t[k].az;
		}
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) ev_acc += __shfl_xor_sync(0xFFFFFFFFu, ev_acc, o);
	if (lane == 0 && ev_acc != 0) atomicAdd(counter, ev_acc);
}

template <typename F>
__global__ void k_to_float(int64_t n, const F *__restrict__ a, float *__restrict__ b)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) b[i] = (float) a[i];
}

// Origin of the integer grid: the box origin when periodic (2^32 units per
// box, wrap-around = nearest image); isolated, half a domain size below the
// domain's origin (2^31 units per domain size, so the grid spans
// [origin - size/2, origin + 3 size/2) and particles that drift out of the
// domain between decompositions stay on it).
static void grid_origin(const tvg_context *ctx, double o[3])
{
	for (int d = 0; d < 3; d++)
		o[d] = ctx->cfg.periodic ? ctx->origin[d] : ctx->origin[d] - 0.5 * ctx->dsize;
}

template <typename F>
static int prepare_typed(tvg_context *ctx)
{
	const int64_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	const double fac = ctx->cfg.periodic ? 4294967296.0 / ctx->dsize : 2147483648.0 / ctx->dsize;
	double go[3];
	grid_origin(ctx, go);
	k_int_pos<F><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(
	    n, (const F *) ctx->f[FS_POS0], (const F *) ctx->f[FS_POS1], (const F *) ctx->f[FS_POS2],
	    go[0], go[1], go[2], fac, ctx->ipos[0], ctx->ipos[1], ctx->ipos[2], ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	// node count from the device: grid-stride launches, and a scan over the
	// capacity (zeros past the count)
	int32_t *nch = ctx->u_count, *choff = ctx->u_endu;     // free after the build
	const int64_t tcap = ctx->tcap, lscan = ctx->tcap < ctx->ucap ? ctx->tcap : ctx->ucap;
	const GNode<F> *tree = (const GNode<F> *) ctx->tree;
	k_wt_nchild<F><<<TVG_CNT(ctx, 148 * 16), 256, 0, s>>>(ctx->dc, tcap, lscan, tree, nch);
	TVG_CUDA(ctx, cudaGetLastError());
	const bool quad = (ctx->cfg.flags & TVG_CFG_QUADRUPOLE) != 0;
	int2 *wrange = nullptr;
	if (quad) {
		if (!ctx->wrange) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->wrange, sizeof(int2) * ctx->tcap));
		if (!ctx->wquad) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->wquad, 2 * sizeof(float4) * ctx->tcap));
		wrange = (int2 *) ctx->wrange;
		TVG_CUDA(ctx, cudaMemsetAsync(wrange, 0, sizeof(int2) * ctx->tcap, s));
		TVG_CHECK(tvg_device_scan_i32_dev(ctx, nch, choff, lscan, &ctx->dc->nwchild));
	} else {
		TVG_CHECK(tvg_device_scan_i32(ctx, nch, choff, lscan, nullptr));
	}
	k_wt_emit<F><<<TVG_CNT(ctx, 148 * 16), 256, 0, s>>>(ctx->dc, tcap, tree, nch, choff, go[0], go[1],
	                                                   go[2], fac, ctx->dsize, ctx->wtree, wrange);
	TVG_CUDA(ctx, cudaGetLastError());
	k_wt_small_top<<<TVG_CNT(ctx, TVG_MAX_TOP / 128), 128, 0, s>>>(ctx->dc, ctx->d_top, ctx->cfg.vector_size, go[0], go[1],
	                                 go[2], fac, ctx->dsize, ctx->wtree, wrange);
	TVG_CUDA(ctx, cudaGetLastError());
	if (quad) {
		const float *mf = (const float *) ctx->f[FS_MASS];
		if (ctx->cfg.float_bytes != 4) {   // the walks' FP32 masses (the FP64 build keeps a copy)
			mf = (const float *) ctx->falt[FS_MASS];
			k_to_float<F><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, (const F *) ctx->f[FS_MASS],
			                                                                (float *) mf);
		}
		TVG_CUDA(ctx, cudaMemsetAsync(ctx->big_list, 0, 4, s));
		k_wt_list_big<<<TVG_CNT(ctx, 148 * 16), 256, 0, s>>>(ctx->dc, wrange, ctx->big_list);
		k_wt_quad_dev<<<TVG_CNT(ctx, 148 * 16), 256, 0, s>>>(ctx->dc, ctx->wtree, wrange, ctx->ipos[0],
		                                                     ctx->ipos[1], ctx->ipos[2], mf,
		                                                     1.0 / fac, ctx->cfg.gravity, ctx->wquad);
		k_wt_quad_block<<<TVG_CNT(ctx, 148 * 4), GW_QUAD_BLOCK_THREADS, 0, s>>>(
		    ctx->wtree, wrange, ctx->ipos[0], ctx->ipos[1], ctx->ipos[2], mf, 1.0 / fac, ctx->cfg.gravity,
		    ctx->wquad, ctx->big_list);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	ctx->have_walktree = true;
	return TVG_OK;
}

// targets per lane: 1 (32-particle groups) or 2 (64): the context's choice
// (tvg_autotune), else TVG_GROUP_TPL from the environment, else the default
static int group_tpl(const tvg_context *ctx)
{
	if (ctx->group_tpl == 1 || ctx->group_tpl == 2 || ctx->group_tpl == 4) return ctx->group_tpl;
	static int tpl = 0;
	if (!tpl) {
		const char *e = getenv("TVG_GROUP_TPL");
		const int v = e ? atoi(e) : 0;
		tpl = (v == 1 || v == 2 || v == 4) ? v : GW_DEFAULT_TPL;
	}
	return tpl;
}

// Groups of an active list: the active particles of each window of gsize
// consecutive (PH-ordered) particles form one group, so that a group is as
// compact as a full one however few of its particles are active.
// (the active count from the device; flags past it are zero, n entries)
__global__ void k_window_flags(int64_t n, const tvg_devcount *__restrict__ dc,
                               const int32_t *__restrict__ active, int gsize, int32_t *flag)
{
	const int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (k >= n) return;
	flag[k] = k < dc->n_active && (k == 0 || active[k] / gsize != active[k - 1] / gsize);
}

__global__ void k_window_scatter(int64_t n, const tvg_devcount *__restrict__ dc,
                                 const int32_t *__restrict__ flag, const int32_t *__restrict__ off,
                                 int32_t *gfirst)
{
	const int64_t n_act = dc->n_active;
	const int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (k < n_act && flag[k]) gfirst[off[k]] = (int32_t) k;
	if (k == 0 && n_act > 0) gfirst[off[n_act - 1] + flag[n_act - 1]] = (int32_t) n_act;
}

// groups of consecutive particles: their number into the device counts
__global__ void k_set_groups(tvg_devcount *dc, int64_t ngroups) { dc->ngroups = ngroups; }

static int build_groups(tvg_context *ctx, int gsize)
{
	const int64_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	k_window_flags<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, ctx->dc, ctx->active, gsize, ctx->act_flag);
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CHECK(tvg_device_scan_i32_dev(ctx, ctx->act_flag, ctx->act_off, n, &ctx->dc->ngroups));
	k_window_scatter<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, ctx->dc, ctx->act_flag, ctx->act_off,
	                                                                  ctx->group_first);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

// the dynamic shared-memory attribute and the occupancy belong to a device:
// the launch helpers cache them per device index
static int device_slot(tvg_context *ctx)
{
	if (ctx->device < 0 || ctx->device >= TVG_MAX_DEVICES)
		return tvg_fail(ctx, TVG_E_BADINPUT, "device index %d out of range", ctx->device);
	return TVG_OK;
}

template <typename K>
static int blocks_for(tvg_context *ctx, K kernel, size_t smem, int *cache, int threads = GW_THREADS)
{
	if (!*cache) {
		TVG_CUDA(ctx, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
		int per_sm = 0, nsm = 0;
		TVG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
		TVG_CUDA(ctx, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
		*cache = (per_sm > 0 ? per_sm : 1) * nsm;
	}
	return TVG_OK;
}

template <int MODE, int TPL, typename F, bool QUAD>
static int launch_walk_q(tvg_context *ctx, GroupParams p, const float *mass_f, const float *last_f,
                         double *counter)
{
	static int nblk_dev[TVG_MAX_DEVICES] = { 0 };
	TVG_CHECK(device_slot(ctx));
	int &nblk = nblk_dev[ctx->device];
	const size_t smem = (sizeof(WarpSmem) + (QUAD ? sizeof(QuadList) : 0)) * GW_WARPS;
	TVG_CHECK(blocks_for(ctx, k_walk_group<MODE, TPL, F, QUAD>, smem, &nblk));
	k_walk_group<MODE, TPL, F, QUAD><<<TVG_CNT(ctx, nblk), GW_THREADS, smem, ctx->stream>>>(
	    p, ctx->use_active ? ctx->active : nullptr, ctx->use_active ? ctx->group_first : nullptr,
	    ctx->wtree, ctx->wquad, ctx->ipos[0], ctx->ipos[1],
	    ctx->ipos[2], mass_f, last_f, (F *) ctx->f[FS_ACC0], (F *) ctx->f[FS_ACC1],
	    (F *) ctx->f[FS_ACC2], (F *) ctx->f[FS_GACC0], (F *) ctx->f[FS_GACC1], (F *) ctx->f[FS_GACC2],
	    (F *) ctx->f[FS_COST], ctx->work_counter, counter, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

template <int MODE, int TPL, typename F>
static int launch_walk(tvg_context *ctx, GroupParams p, const float *mass_f, const float *last_f,
                       double *counter)
{
	if (p.quad) return launch_walk_q<MODE, TPL, F, true>(ctx, p, mass_f, last_f, counter);
	return launch_walk_q<MODE, TPL, F, false>(ctx, p, mass_f, last_f, counter);
}

template <int TPL, bool MLP, typename F>
static int launch_ewald(tvg_context *ctx, GroupParams p, const float *mass_f, const float *last_f,
                        double *counter)
{
	static int nblk_dev[TVG_MAX_DEVICES] = { 0 };
	TVG_CHECK(device_slot(ctx));
	int &nblk = nblk_dev[ctx->device];
	const size_t smem = sizeof(EwaldSmem) * GE_WARPS
	                  + (MLP ? 4 * MLP_NPARAM + 2 * MLP_H * MLP_H : (GW_EWALD_STAGE ? sizeof(EwaldStage) * GE_WARPS : 0));
	TVG_CHECK(blocks_for(ctx, k_ewald_group<TPL, MLP, F>, smem, &nblk, GE_THREADS));
	k_ewald_group<TPL, MLP, F><<<TVG_CNT(ctx, nblk), GE_THREADS, smem, ctx->stream>>>(
	    p, ctx->use_active ? ctx->active : nullptr, ctx->use_active ? ctx->group_first : nullptr,
	    ctx->wtree, ctx->ipos[0], ctx->ipos[1],
	    ctx->ipos[2], mass_f, last_f, (const float4 *) ctx->ewald_ext,
	    (const float4 *) ctx->ewald_taylor, (const __nv_bfloat16 *) ctx->mlp_bf16, ctx->mlp_prm,
	    (F *) ctx->f[FS_ACC0],
	    (F *) ctx->f[FS_ACC1], (F *) ctx->f[FS_ACC2], (F *) ctx->f[FS_GACC0], (F *) ctx->f[FS_GACC1],
	    (F *) ctx->f[FS_GACC2], ctx->work_counter + 1, counter, ctx->status,
	    p.quad ? (const float4 *) ctx->wquad : nullptr);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

__global__ void k_mass_total(int64_t n, const float *__restrict__ m, double *out)
{
	double s = 0;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
	     i += (int64_t) gridDim.x * blockDim.x)
		s += (double) m[i];
#pragma unroll
	for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
	if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// the gravity walk, then (with Ewald) the Ewald walk, for one group size;
// events ev[0], ev[1] bracket the gravity walk, ev[1], ev[2] the Ewald walk
template <int TPL, typename F>
static int launch_pair(tvg_context *ctx, const GroupParams &p, bool ewald, bool mlp,
                       const float *mass_f, const float *last_f, double *cnt)
{
	if (ewald) TVG_CHECK((launch_walk<GM_CENTRE, TPL, F>(ctx, p, mass_f, last_f, cnt)));
	else TVG_CHECK((launch_walk<GM_NEAREST, TPL, F>(ctx, p, mass_f, last_f, cnt)));
	TVG_CUDA(ctx, tvg_record(ctx, ctx->ev[1]));
	if (ewald && mlp) TVG_CHECK((launch_ewald<TPL, true, F>(ctx, p, mass_f, last_f, cnt + 1)));
	else if (ewald) TVG_CHECK((launch_ewald<TPL, false, F>(ctx, p, mass_f, last_f, cnt + 1)));
	return TVG_OK;
}

template <typename F>
static int walk_group_typed(tvg_context *ctx, int use_bh, uint32_t parts, int ewald_kind)
{
	const int64_t n = ctx->n;
	if (n == 0) return TVG_OK;
	const bool ewald = (parts & TVG_WALK_EWALD) != 0;
	if (!(parts & TVG_WALK_GRAVITY))
		return tvg_fail(ctx, TVG_E_BADINPUT,
		                "group form: the gravity and Ewald parts share the particle images; "
		                "pass TVG_WALK_GRAVITY | TVG_WALK_EWALD");
	if (ctx->cfg.flags & TVG_CFG_POTENTIAL)
		return tvg_fail(ctx, TVG_E_BADINPUT, "group form: no potential (TVG_CFG_POTENTIAL); use "
		                "TVG_FORM_PLAIN");
	const bool mlp = ewald && ewald_kind == TVG_EWALD_MLP;
	if (ewald && ewald_kind != TVG_EWALD_TABLE && ewald_kind != TVG_EWALD_MLP)
		return tvg_fail(ctx, TVG_E_BADINPUT, "unknown Ewald kind %d", ewald_kind);
	if (mlp && !(ctx->have_mlp && ctx->mlp_ok))
		return tvg_fail(ctx, TVG_E_STATE, "learned Ewald correction not trained or not accepted by "
		                "the table (tvg_ewald_mlp_validate)");
	cudaStream_t s = ctx->stream;
	if (!ctx->have_walktree) TVG_CHECK(prepare_typed<F>(ctx));
	if (ewald && !ctx->ewald_ext) TVG_CHECK(tvg_impl_ewald_ext(ctx));
	if (ewald && !ctx->ewald_taylor) TVG_CHECK(tvg_impl_ewald_taylor(ctx));
	// FP32 copies of mass / last |a| (views when Float is float)
	const float *mass_f = (const float *) ctx->f[FS_MASS];
	const float *last_f = (const float *) ctx->f[FS_LAST_ACC];
	if (sizeof(F) == 8) {
		float *mf = (float *) ctx->falt[FS_MASS], *lf = (float *) ctx->falt[FS_LAST_ACC];
		k_to_float<F><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, (const F *) ctx->f[FS_MASS], mf);
		k_to_float<F><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, (const F *) ctx->f[FS_LAST_ACC], lf);
		mass_f = mf;
		last_f = lf;
	}
	const tvg_config &cf = ctx->cfg;
	const int tpl = group_tpl(ctx);
	GroupParams p;
	p.n = n;
	p.dc = ctx->dc;
	p.max_iter = ctx->walk_limit;
	p.quad = (ctx->cfg.flags & TVG_CFG_QUADRUPOLE) ? 1 : 0;
	p.gsize = 32 * tpl;
	if (ctx->use_active) {
		TVG_CHECK(build_groups(ctx, p.gsize));
	} else {
		k_set_groups<<<TVG_CNT(ctx, 1), 1, 0, s>>>(ctx->dc, (n + p.gsize - 1) / p.gsize);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	p.periodic = cf.periodic;
	p.use_bh = use_bh;
	p.open_bundles = (cf.flags & TVG_CFG_OPEN_BUNDLES) ? 1 : 0;
	p.scale = (float) (cf.periodic ? ctx->dsize / 4294967296.0 : ctx->dsize / 2147483648.0);
	p.box = (float) (cf.periodic ? cf.boxsize : 0.0);
	p.half_box = (float) (cf.periodic ? 0.5 * cf.boxsize : 3.0e38);
	p.theta2 = (float) cf.open_bh;
	p.rel_fac = (float) (cf.open_rel / cf.gravity);
	p.gravity = (float) cf.gravity;
	const double h = -41.0 / 32.0 * cf.softening;
	p.eps2 = (float) (h * h);
	p.inv_eps2 = (float) (1.0 / (h * h));
	p.c16 = (float) (1.0 / (16.0 * h * h * h));
	p.near2 = (float) (h * h * 1.001);
	p.grid = (float) (cf.periodic ? 2.0 * 64.0 / cf.boxsize : 0.0);
	p.inv_box = (float) (cf.periodic ? 1.0 / cf.boxsize : 0.0);
	p.tay_grid = (float) (cf.periodic ? 2.0 * (TVG_TAYLOR_NODES - 1) / cf.boxsize : 0.0);
	p.ew_rel = (float) (ctx->ewald_open_rel / cf.open_rel);   // times g.fac: alpha_E |a_old| / G
	p.ew_bh = (float) (ctx->ewald_open_bh * cf.open_bh);
	// half extent beyond which a group takes per-target images with the Ewald
	// part. The expansion's third-order remainder is dominated by the uniform
	// background, which uniform_remainder adds exactly; what is left (the
	// density fluctuations' share) kept the expansion within 1.2x of the
	// per-target force error at h ~ L / 32 (64^3 box, z = 50).
	p.taylor_h = (float) (cf.periodic ? cf.boxsize / 20.0 : 3.0e38);
	p.uniform_g = cf.periodic ? cf.gravity / (cf.boxsize * cf.boxsize) : 0.0;
	if (ewald) {
		double *dm = &ctx->dc->mass_total;
		TVG_CUDA(ctx, cudaMemsetAsync(dm, 0, 8, s));
		k_mass_total<<<TVG_CNT(ctx, 148 * 4), 256, 0, s>>>(n, mass_f, dm);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->counters, 0, 24, s));
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->work_counter, 0, 8, s));
	TVG_CUDA(ctx, tvg_record(ctx, ctx->ev[0]));
	double *cnt = ctx->counters;
	if (tpl == 1) TVG_CHECK((launch_pair<1, F>(ctx, p, ewald, mlp, mass_f, last_f, cnt)));
	else if (tpl == 2) TVG_CHECK((launch_pair<2, F>(ctx, p, ewald, mlp, mass_f, last_f, cnt)));
	else TVG_CHECK((launch_pair<4, F>(ctx, p, ewald, mlp, mass_f, last_f, cnt)));
	TVG_CUDA(ctx, tvg_record(ctx, ctx->ev[2]));
	if (ctx->capturing) return TVG_OK;
	return tvg_walk_group_results(ctx);
}

// walk and Ewald-walk times and interaction counts of the last group walk
// (synchronises)
int tvg_walk_group_results(tvg_context *ctx)
{
	TVG_CUDA(ctx, cudaEventSynchronize(ctx->ev[2]));
	float ms = 0, ms_e = 0;
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
	TVG_CUDA(ctx, cudaEventElapsedTime(&ms_e, ctx->ev[1], ctx->ev[2]));
	ctx->phase_ms[4] = ms;
	ctx->phase_ms[5] = ms_e;
	double c[3];
	TVG_CUDA(ctx, cudaMemcpy(c, ctx->counters, 24, cudaMemcpyDeviceToHost));
	ctx->last_counts[0] = c[0];
	ctx->last_counts[1] = c[1];
	ctx->last_counts[2] = c[2];
	return TVG_OK;
}

// Autotuner of the group form: times the walks of the current tree and active
// set with each group size (targets per lane) and keeps the fastest; the walk
// of the chosen size runs last, so its accelerations are the ones left.
// The autotuner's sample: the active particles (all particles without an
// active list) that lie in every TUNE_STRIDE-th window of 128 particles, so
// that groups of 32, 64 and 128 are all full windows of the sample.
#define TUNE_WINDOW 128
#define TUNE_STRIDE 8

__global__ void k_tune_flags(int64_t n_src, const tvg_devcount *__restrict__ dc,
                             const int32_t *__restrict__ src, int32_t *__restrict__ flag)
{
	const int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (k >= n_src) return;
	const int64_t m = src ? dc->n_active : n_src;
	const int64_t i = src ? (int64_t) src[k] : k;
	flag[k] = k < m && (i / TUNE_WINDOW) % TUNE_STRIDE == 0;
}

__global__ void k_tune_scatter(int64_t n_src, const int32_t *__restrict__ src, const int32_t *__restrict__ flag,
                               const int32_t *__restrict__ off, int32_t *__restrict__ out)
{
	const int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (k < n_src && flag[k]) out[off[k]] = src ? src[k] : (int32_t) k;
}

extern "C" int tvg_autotune(tvg_context *ctx, int32_t use_bh, uint32_t parts, int32_t ewald_kind,
                            int32_t *choice, double *ms)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_tree) return tvg_fail(ctx, TVG_E_STATE, "autotune: no tree");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	// the active count as the walks read it, on the device
	int64_t dev_n_active = 0;
	TVG_CUDA(ctx, cudaMemcpyAsync(&dev_n_active, &ctx->dc->n_active, 8, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	// the sample as a temporary active list
	const int64_t n_src = ctx->use_active ? dev_n_active : ctx->n;
	if (!ctx->tune_active) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->tune_active, 4 * (size_t) ctx->cap));
	if (!ctx->act_flag) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->act_flag, 4 * (size_t) ctx->cap));
	if (!ctx->act_off) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->act_off, 4 * (size_t) ctx->cap));
	const int32_t *src = ctx->use_active ? ctx->active : nullptr;
	k_tune_flags<<<TVG_CNT(ctx, tvg_blocks(n_src, 256)), 256, 0, s>>>(n_src, ctx->dc, src, ctx->act_flag);
	TVG_CUDA(ctx, cudaGetLastError());
	int64_t n_tune = 0;
	TVG_CHECK(tvg_device_scan_i32(ctx, ctx->act_flag, ctx->act_off, n_src, &n_tune));
	k_tune_scatter<<<TVG_CNT(ctx, tvg_blocks(n_src, 256)), 256, 0, s>>>(n_src, src, ctx->act_flag,
	                                                                    ctx->act_off, ctx->tune_active);
	TVG_CUDA(ctx, cudaGetLastError());
	const bool was_active = ctx->use_active;
	int32_t *const saved_list = ctx->active;
	const int64_t saved_n = ctx->n_active;
	ctx->active = ctx->tune_active;
	ctx->use_active = true;
	ctx->n_active = n_tune;
	TVG_CUDA(ctx, cudaMemcpyAsync(&ctx->dc->n_active, &n_tune, 8, cudaMemcpyHostToDevice, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	// the walks add to Acc: keep it (in the sort's free second buffers) so
	// that only the final walk's contribution remains
	const size_t acc_bytes = tvg_fsize(ctx) * (size_t) ctx->n;
	for (int k = 0; k < 3; k++)
		TVG_CUDA(ctx, cudaMemcpyAsync(ctx->falt[FS_ACC0 + k], ctx->f[FS_ACC0 + k], acc_bytes,
		                              cudaMemcpyDeviceToDevice, s));
	const int sizes[3] = { 1, 2, 4 };
	double t[3] = { 0, 0, 0 };
	int best = 0, rc = TVG_OK;
	for (int c = 0; c < 3 && rc == TVG_OK && n_tune > 0; c++) {
		ctx->group_tpl = sizes[c];
		rc = tvg_impl_walk_group(ctx, use_bh, parts, ewald_kind);
		t[c] = ctx->phase_ms[4] + ctx->phase_ms[5];
		if (t[c] < t[best]) best = c;
	}
	// the caller's active set back, then the chosen walk over all of it
	ctx->active = saved_list;
	ctx->use_active = was_active;
	ctx->n_active = saved_n;
	TVG_CUDA(ctx, cudaMemcpyAsync(&ctx->dc->n_active, &dev_n_active, 8, cudaMemcpyHostToDevice, s));
	for (int k = 0; k < 3; k++)
		TVG_CUDA(ctx, cudaMemcpyAsync(ctx->f[FS_ACC0 + k], ctx->falt[FS_ACC0 + k], acc_bytes,
		                              cudaMemcpyDeviceToDevice, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	if (rc != TVG_OK) return rc;
	ctx->group_tpl = n_tune > 0 ? sizes[best] : GW_DEFAULT_TPL;
	TVG_CHECK(tvg_impl_walk_group(ctx, use_bh, parts, ewald_kind));
	if (choice) *choice = ctx->group_tpl;
	if (ms) for (int c = 0; c < 3; c++) ms[c] = t[c];
	return tvg_sync_status(ctx, "autotune");
}

int tvg_impl_walk_group(tvg_context *ctx, int use_bh, uint32_t parts, int ewald_kind)
{
	if (ctx->cfg.float_bytes == 4) return walk_group_typed<float>(ctx, use_bh, parts, ewald_kind);
	return walk_group_typed<double>(ctx, use_bh, parts, ewald_kind);
}
