// tvg_walk_plain.cu -- the plain GPU form: the reference tree walk, one
// thread per active particle, in the host's Float width.
//
// Gravity part: Gravity_Tree_Acceleration (tree_accel.c:32-394) -- every top
// node (interact_with_topnode), then the subtree walk with the BH or the
// relative criterion over the DNext skip pointers; softened monopole
// interact() with the Dehnen K1 kernel at h = -41/32 eps (tree_build.c:136,
// kept as in the reference: the sign flip of quirk Q1).
// Ewald part: Gravity_Tree_Periodic (tree_periodic.c:23-450) with the
// trilinear table lookup of Ewald_Correction (Gravity/periodic.c:35-113).
// With TVG_CFG_POTENTIAL (GRAVITY_POTENTIAL) the potential of interact()
// (tree_accel.c:362-389) and of interact_with_ewald_cube (tree_periodic.c:
// 425-447, Ewald_Potential at Gravity/periodic.c:115-170) are summed in double
// as the reference's Recv.Grav_Potential.
// This file is compiled with -fmad=false: every expression rounds in the
// reference's order (float/double promotion as in C), so given the same tree
// the accelerations are the reference's bit for bit.
// Roofline: FP64/FP32 issue bound with divergent per-thread walks; it is the
// baseline the group form is measured against.
#include "tvg_internal.cuh"

template <typename F> struct WNode {
	int32_t DNext;
	uint32_t Bitfield;
	int32_t DUp;
	int32_t Npart;
	F Pos[3];
	F Mass;
	F CoM[3];
	F Dp[3];
};

struct PlainParams {
	double gravity, domain_size, boxsize, open_bh, open_rel;
	double eps, eps2, eps3, box2grid;
	int periodic, use_bh, vsize, ntop, fix_small;
};

template <typename F> struct PlainCtx {
	const F *x, *y, *z, *m;
	const tvg_topnode *top;
	const WNode<F> *tree;
	const F *fx, *fy, *fz, *fp;
	F boxhalf;
	int64_t tree_cap;    // node capacity: the walks never read past it
	PlainParams p;
};

template <typename F>
__device__ __forceinline__ void nearest(const PlainCtx<F> &c, F dr[3])
{
	if (!c.p.periodic) return;
#pragma unroll
	for (int k = 0; k < 3; k++) {
		if (dr[k] > c.boxhalf) dr[k] = (F) (dr[k] - c.p.boxsize);
		else if (dr[k] < -c.boxhalf) dr[k] = (F) (dr[k] + c.p.boxsize);
	}
}

template <typename F> __device__ __forceinline__ F fsqrt(F v);
template <> __device__ __forceinline__ float fsqrt<float>(float v) { return __fsqrt_rn(v); }
template <> __device__ __forceinline__ double fsqrt<double>(double v) { return __dsqrt_rn(v); }

// interact(), tree_accel.c:362-394; with POT the potential fac_pot, whose
// inner polynomial is the reference's (u2 * (175 - (u2 * 147 - u2 * 45))
// - 105) / (32 Epsilon), summed into pot
template <bool POT, typename F>
__device__ __forceinline__ void interact(const PlainCtx<F> &c, F mass, const F dr[3], F r2,
                                         double acc[3], F &cost, double &pot)
{
	F fac = (F) (c.p.gravity * mass);
	F fac_pot = fac;
	if (r2 < c.p.eps2) {
		F u2 = (F) (r2 / c.p.eps2);
		F poly = (F) 175 - u2 * ((F) 294 - u2 * (F) 135);
		fac = (F) (fac * (poly / (16 * c.p.eps3)));
		if (POT) {
			const F ppoly = u2 * ((F) 175 - (u2 * (F) 147 - u2 * (F) 45)) - (F) 105;
			fac_pot = (F) (fac_pot * (ppoly / (32 * c.p.eps)));
		}
	} else {
		F r_inv = (F) 1 / fsqrt<F>(r2);
		fac *= r_inv * r_inv * r_inv;
		if (POT) fac_pot *= r_inv;
	}
	acc[0] += fac * dr[0];
	acc[1] += fac * dr[1];
	acc[2] += fac * dr[2];
	if (POT) pot += fac_pot;
	cost += 1;
}

template <typename F>
__device__ __forceinline__ F node_size(const PlainCtx<F> &c, int lvl)
{
	return (F) (c.p.domain_size / (double) (F) (1ULL << lvl));
}

template <bool POT, typename F>
__device__ void walk_gravity(const PlainCtx<F> &c, const F sp[3], F sacc, double acc[3], F &cost,
                             double &pot)
{
	const F fac = (F) (sacc / c.p.gravity * c.p.open_rel);
	for (int j = 0; j < c.p.ntop; j++) {
		const tvg_topnode &t = c.top[j];
		const F nsize = (F) (c.p.domain_size / (double) (F) (1UL << t.level));
		F dr[3] = { (F) t.pos[0] - sp[0], (F) t.pos[1] - sp[1], (F) t.pos[2] - sp[2] };
		const bool inside = fabs((double) dr[0]) < 0.6 * nsize && fabs((double) dr[1]) < 0.6 * nsize
		                 && fabs((double) dr[2]) < 0.6 * nsize;
		if (!inside) {
			dr[0] = (F) t.com[0] - sp[0];
			dr[1] = (F) t.com[1] - sp[1];
			dr[2] = (F) t.com[2] - sp[2];
			nearest(c, dr);
			F r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
			F nmass = (F) t.mass;
			bool open;
			if (c.p.use_bh) open = (double) (nsize * nsize) > r2 * c.p.open_bh;
			else open = nmass * nsize * nsize > r2 * r2 * fac;
			if (!open) { interact<POT>(c, nmass, dr, r2, acc, cost, pot); continue; }
		}
		if (t.npart <= c.p.vsize) {
			const int64_t f0 = c.p.fix_small ? t.first_part : t.target;
			for (int64_t jp = f0; jp < f0 + t.npart; jp++) {
				F d[3] = { c.x[jp] - sp[0], c.y[jp] - sp[1], c.z[jp] - sp[2] };
				nearest(c, d);
				F r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
				if (r2 != 0) interact<POT>(c, c.m[jp], d, r2, acc, cost, pot);
			}
			continue;
		}
		const int start = t.target;
		int node = start;
		// (a valid tree ends every subtree with a terminator, DNext = 0, well
		// inside the capacity; the bound only keeps a damaged one in memory)
		while (node < c.tree_cap && (c.tree[node].DNext != 0 || node == start)) {
			const WNode<F> &nd = c.tree[node];
			const int32_t dn = nd.DNext;
			if (dn < 0) {
				const int64_t f = -(int64_t) dn - 1;
				const int np = nd.Npart;
				for (int64_t jp = f; jp < f + np; jp++) {
					F d[3] = { c.x[jp] - sp[0], c.y[jp] - sp[1], c.z[jp] - sp[2] };
					nearest(c, d);
					F r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
					if (r2 != 0) interact<POT>(c, c.m[jp], d, r2, acc, cost, pot);
				}
				node++;
				continue;
			}
			F d[3] = { nd.CoM[0] - sp[0], nd.CoM[1] - sp[1], nd.CoM[2] - sp[2] };
			nearest(c, d);
			F r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
			F nmass = nd.Mass;
			F nsz = node_size(c, (int) (nd.Bitfield & 0x3F));
			if (c.p.use_bh) {
				if ((double) (nsz * nsz) > r2 * c.p.open_bh) { node++; continue; }
			} else {
				if (nmass * nsz * nsz > r2 * r2 * fac) { node++; continue; }
				F ds[3] = { nd.Pos[0] - sp[0], nd.Pos[1] - sp[1], nd.Pos[2] - sp[2] };
				nearest(c, ds);
				if (fabs((double) ds[0]) < 0.6 * nsz && fabs((double) ds[1]) < 0.6 * nsz
				    && fabs((double) ds[2]) < 0.6 * nsz) { node++; continue; }
			}
			interact<POT>(c, nmass, d, r2, acc, cost, pot);
			node += dn;
		}
	}
}

// Ewald_Correction, Gravity/periodic.c:35-113
template <typename F>
__device__ __forceinline__ void ewald_corr(const PlainCtx<F> &c, const F dr[3], F f[3])
{
	int sg[3] = { -1, -1, -1 };
	F dx = dr[0], dy = dr[1], dz = dr[2];
	if (dx < 0) { dx = -dx; sg[0] = 1; }
	if (dy < 0) { dy = -dy; sg[1] = 1; }
	if (dz < 0) { dz = -dz; sg[2] = 1; }
	F u = (F) (dx * c.p.box2grid), v = (F) (dy * c.p.box2grid), w = (F) (dz * c.p.box2grid);
	int i = (int) u, j = (int) v, k = (int) w;
	if (i >= 64) i = 63;
	if (j >= 64) j = 63;
	if (k >= 64) k = 63;
	u -= i; v -= j; w -= k;
	const F one = 1;
	const F wt[8] = { (one - u) * (one - v) * (one - w), (one - u) * (one - v) * w,
	                  (one - u) * v * (one - w), (one - u) * v * w,
	                  u * (one - v) * (one - w), u * (one - v) * w,
	                  u * v * (one - w), u * v * w };
	const int64_t b = ((int64_t) i * 65 + j) * 65 + k;
	const int64_t o1 = 1, o2 = 65, o3 = 66, o4 = 65 * 65, o5 = 65 * 65 + 1, o6 = 65 * 65 + 65,
	              o7 = 65 * 65 + 66;
	const F *tab[3] = { c.fx, c.fy, c.fz };
#pragma unroll
	for (int d = 0; d < 3; d++) {
		const F *T = tab[d];
		f[d] = wt[0] * T[b] + wt[1] * T[b + o1] + wt[2] * T[b + o2] + wt[3] * T[b + o3]
		     + wt[4] * T[b + o4] + wt[5] * T[b + o5] + wt[6] * T[b + o6] + wt[7] * T[b + o7];
	}
	f[0] *= sg[0];
	f[1] *= sg[1];
	f[2] *= sg[2];
}

// Ewald_Potential, Gravity/periodic.c:115-170: trilinear in double on the
// potential table at |dr|, the result stored as Float
template <typename F>
__device__ __forceinline__ F ewald_pot(const PlainCtx<F> &c, const F dr[3])
{
	const double dx = fabs((double) dr[0]), dy = fabs((double) dr[1]), dz = fabs((double) dr[2]);
	double u = dx * c.p.box2grid, v = dy * c.p.box2grid, w = dz * c.p.box2grid;
	int i = (int) u, j = (int) v, k = (int) w;
	if (i >= 64) i = 63;
	if (j >= 64) j = 63;
	if (k >= 64) k = 63;
	u -= i;
	v -= j;
	w -= k;
	const double wt[8] = { (1 - u) * (1 - v) * (1 - w), (1 - u) * (1 - v) * w,
	                       (1 - u) * v * (1 - w), (1 - u) * v * w,
	                       u * (1 - v) * (1 - w), u * (1 - v) * w,
	                       u * v * (1 - w), u * v * w };
	const int64_t b = ((int64_t) i * 65 + j) * 65 + k;
	const F *T = c.fp;
	return (F) (wt[0] * T[b] + wt[1] * T[b + 1] + wt[2] * T[b + 65] + wt[3] * T[b + 66]
	            + wt[4] * T[b + 65 * 65] + wt[5] * T[b + 65 * 65 + 1] + wt[6] * T[b + 65 * 65 + 65]
	            + wt[7] * T[b + 65 * 65 + 66]);
}

// interact_with_ewald_cube, tree_periodic.c:425-447
template <bool POT, typename F>
__device__ __forceinline__ void ewald_cube(const PlainCtx<F> &c, const F dr[3], F mass, double acc[3],
                                           F &cost, double &pot)
{
	F r[3];
	ewald_corr(c, dr, r);
	acc[0] += c.p.gravity * mass * r[0];
	acc[1] += c.p.gravity * mass * r[1];
	acc[2] += c.p.gravity * mass * r[2];
	cost += 1;
	if (POT) pot += c.p.gravity * mass * ewald_pot(c, dr);
}

template <bool POT, typename F>
__device__ void walk_ewald(const PlainCtx<F> &c, const F sp[3], F sacc, double acc[3], F &cost,
                           double &pot)
{
	const double box = c.p.boxsize;
	const F fac = (F) (sacc / c.p.gravity * c.p.open_rel);
	const double bh2 = c.p.open_bh * c.p.open_bh;
	for (int j = 0; j < c.p.ntop; j++) {
		const tvg_topnode &t = c.top[j];
		const F nsize = (F) (c.p.domain_size / (double) (1UL << t.level));
		bool want = false;
		F dr[3] = { (F) t.com[0] - sp[0], (F) t.com[1] - sp[1], (F) t.com[2] - sp[2] };
		nearest(c, dr);
		F r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
		if (c.p.use_bh) {
			if ((double) (nsize * nsize) > r2 * c.p.open_bh) want = true;
		} else {
			F nmass = (F) t.mass;
			if (nmass * nsize * nsize > r2 * r2 * fac) want = true;
		}
		double dx = fabs((double) (F) (sp[0] - (F) t.pos[0]));
		if (dx < 0.6 * nsize) {
			double dy = fabs((double) (F) (sp[1] - (F) t.pos[1]));
			if (dy < 0.6 * nsize) {
				double dz = fabs((double) (F) (sp[2] - (F) t.pos[2]));
				if (dz < 0.6 * nsize) want = true;
			}
		}
		bool open = false;
		if (want) {
			const double lim = 0.5 * (box - nsize);
			if (fabs((double) dr[0]) > lim || fabs((double) dr[1]) > lim || fabs((double) dr[2]) > lim
			    || nsize > 0.2 * box)
				open = true;
		}
		if (!open) { ewald_cube<POT>(c, dr, (F) t.mass, acc, cost, pot); continue; }
		if (t.npart <= c.p.vsize) {
			const int64_t f0 = c.p.fix_small ? t.first_part : t.target;
			for (int64_t jp = f0; jp < f0 + t.npart; jp++) {
				F d[3] = { c.x[jp] - sp[0], c.y[jp] - sp[1], c.z[jp] - sp[2] };
				nearest(c, d);
				if (d[0] != 0 && d[1] != 0 && d[2] != 0) ewald_cube<POT>(c, d, c.m[jp], acc, cost, pot);
			}
			continue;
		}
		const int start = t.target;
		const int end = start + c.tree[start].DNext;
		int node = start;
		while (node < end && node < c.tree_cap) {
			const WNode<F> &nd = c.tree[node];
			const int32_t dn = nd.DNext;
			if (dn < 0) {
				const int64_t f = -(int64_t) dn - 1;
				const int np = nd.Npart;
				for (int64_t jp = f; jp < f + np; jp++) {
					F d[3] = { c.x[jp] - sp[0], c.y[jp] - sp[1], c.z[jp] - sp[2] };
					nearest(c, d);
					if (d[0] != 0 && d[1] != 0 && d[2] != 0) ewald_cube<POT>(c, d, c.m[jp], acc, cost, pot);
				}
				node++;
				continue;
			}
			F d[3] = { nd.CoM[0] - sp[0], nd.CoM[1] - sp[1], nd.CoM[2] - sp[2] };
			nearest(c, d);
			F rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
			F nmass = nd.Mass;
			F nsz = node_size(c, (int) (nd.Bitfield & 0x3F));
			F ds[3] = { nd.Pos[0] - sp[0], nd.Pos[1] - sp[1], nd.Pos[2] - sp[2] };
			bool wo = false;
			if (c.p.use_bh) {
				if ((double) (nsz * nsz) > rr * bh2) wo = true;
			} else {
				if (nmass * nsz * nsz > rr * rr * fac) wo = true;
			}
			if (!wo && fabs((double) ds[0]) < 0.6 * nsz && fabs((double) ds[1]) < 0.6 * nsz
			    && fabs((double) ds[2]) < 0.6 * nsz)
				wo = true;
			nearest(c, ds);
			if (wo) {
				const double dl = 0.5 * (box - nsz);
				if (fabs((double) ds[0]) > dl || fabs((double) ds[1]) > dl || fabs((double) ds[2]) > dl
				    || nsz > 0.2 * box) { node++; continue; }
			}
			ewald_cube<POT>(c, d, nmass, acc, cost, pot);
			node += dn;
		}
	}
}

template <bool POT, typename F>
__global__ void __launch_bounds__(128)
k_walk_plain(int64_t n_act, const int32_t *__restrict__ active, PlainCtx<F> c, int ewald,
             const F *__restrict__ last_acc, F *acc0, F *acc1, F *acc2, F *gacc0, F *gacc1,
             F *gacc2, F *cost_out, F *pot_out, double *counter)
{
	// every thread reads every top node: staged in shared memory when they
	// fit (one target: <= 64 level-2 cells), else read through L1
	__shared__ tvg_topnode s_top[64];
	PlainCtx<F> cc = c;
	if (c.p.ntop <= 64) {
		for (int j = threadIdx.x; j < c.p.ntop; j += blockDim.x) s_top[j] = c.top[j];
		__syncthreads();
		cc.top = s_top;
	}
	const int64_t t = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	F cost = 0;
	if (t < n_act) {
		const int64_t i = active ? active[t] : t;     // Active_Particle_List[t]
		const F sp[3] = { c.x[i], c.y[i], c.z[i] };
		double a[3] = { 0, 0, 0 }, pot = 0;
		if (ewald) walk_ewald<POT>(cc, sp, last_acc[i], a, cost, pot);
		else walk_gravity<POT>(cc, sp, last_acc[i], a, cost, pot);
		// add_recv_to (tree_accel.c:110-129, tree_periodic.c:91-110)
		acc0[i] += a[0];
		acc1[i] += a[1];
		acc2[i] += a[2];
		if (ewald) {
			gacc0[i] += a[0];
			gacc1[i] += a[1];
			gacc2[i] += a[2];
			cost_out[i] += cost;
			if (POT) pot_out[i] += pot;
		} else {
			gacc0[i] = (F) a[0];
			gacc1[i] = (F) a[1];
			gacc2[i] = (F) a[2];
			cost_out[i] = cost;
			if (POT) pot_out[i] = (F) pot;
		}
	}
	// interaction count for the roofline accounting
	double cw = (double) cost;
#pragma unroll
	for (int o = 16; o; o >>= 1) cw += __shfl_xor_sync(0xFFFFFFFFu, cw, o);
	if ((threadIdx.x & 31) == 0 && cw != 0) atomicAdd(counter, cw);
}

template <typename F>
static int walk_typed(tvg_context *ctx, int use_bh, uint32_t parts)
{
	const int64_t n = ctx->n;
	if (n == 0) return TVG_OK;
	PlainCtx<F> c;
	c.x = (const F *) ctx->f[FS_POS0];
	c.y = (const F *) ctx->f[FS_POS1];
	c.z = (const F *) ctx->f[FS_POS2];
	c.m = (const F *) ctx->f[FS_MASS];
	c.top = ctx->d_top;
	c.tree = (const WNode<F> *) ctx->tree;
	c.tree_cap = ctx->tcap;
	c.fx = (const F *) ctx->ewald_f[0];
	c.fy = (const F *) ctx->ewald_f[1];
	c.fz = (const F *) ctx->ewald_f[2];
	c.fp = (const F *) ctx->ewald_f[3];
	const tvg_config &cf = ctx->cfg;
	c.p.gravity = cf.gravity;
	c.p.domain_size = ctx->dsize;
	c.p.boxsize = cf.periodic ? cf.boxsize : 0;
	c.p.open_bh = cf.open_bh;
	c.p.open_rel = cf.open_rel;
	const double eps = -41.0 / 32.0 * cf.softening;    // tree_build.c:136-138
	c.p.eps = eps;
	c.p.eps2 = eps * eps;
	c.p.eps3 = eps * eps * eps;
	c.p.box2grid = cf.periodic ? 2 * 64 / cf.boxsize : 0;
	c.p.periodic = cf.periodic;
	c.p.use_bh = use_bh;
	c.p.vsize = cf.vector_size;
	c.p.ntop = ctx->ntop;
	c.p.fix_small = (cf.flags & TVG_CFG_FIX_SMALL_TOPNODES) ? 1 : 0;
	c.boxhalf = (F) (c.p.boxsize / 2.0);
	cudaStream_t s = ctx->stream;
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->counters, 0, 16, s));
	for (int part = 0; part < 2; part++) {
		const bool ew = part == 1;
		if (!(parts & (ew ? TVG_WALK_EWALD : TVG_WALK_GRAVITY))) continue;
		TVG_CUDA(ctx, cudaEventRecord(ctx->ev[0], s));
		const int64_t n_act = ctx->use_active ? ctx->n_active : n;
		const bool pot = (cf.flags & TVG_CFG_POTENTIAL) != 0;
		auto kern = pot ? k_walk_plain<true, F> : k_walk_plain<false, F>;
		kern<<<TVG_CNT(ctx, tvg_blocks(n_act, 128)), 128, 0, s>>>(
		    n_act, ctx->use_active ? ctx->active : nullptr, c, ew ? 1 : 0,
		    (const F *) ctx->f[FS_LAST_ACC], (F *) ctx->f[FS_ACC0],
		    (F *) ctx->f[FS_ACC1], (F *) ctx->f[FS_ACC2], (F *) ctx->f[FS_GACC0],
		    (F *) ctx->f[FS_GACC1], (F *) ctx->f[FS_GACC2], (F *) ctx->f[FS_COST],
		    (F *) ctx->f[FS_GRAV_POT], ctx->counters + (ew ? 1 : 0));
		TVG_CUDA(ctx, cudaGetLastError());
		TVG_CUDA(ctx, cudaEventRecord(ctx->ev[1], s));
		TVG_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
		float ms = 0;
		TVG_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
		ctx->phase_ms[ew ? 5 : 4] = ms;
	}
	double cnt[2];
	TVG_CUDA(ctx, cudaMemcpy(cnt, ctx->counters, 16, cudaMemcpyDeviceToHost));
	ctx->last_counts[0] = cnt[0];
	ctx->last_counts[1] = cnt[1];
	return TVG_OK;
}

int tvg_impl_walk_plain(tvg_context *ctx, int use_bh, uint32_t parts)
{
	if (ctx->cfg.float_bytes == 4) return walk_typed<float>(ctx, use_bh, parts);
	return walk_typed<double>(ctx, use_bh, parts);
}

// accel.c:28-43: Last_Acc_Mag = |Acc|, Acc = 0 (the active particles; their
// number from the device when n_dev is given, n bounds it)
template <typename F>
__global__ void k_save_last(int64_t n, const int64_t *__restrict__ n_dev, const int32_t *__restrict__ active,
                            F *a0, F *a1, F *a2, F *last)
{
	const int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (k >= n || (n_dev && k >= *n_dev)) return;
	const int64_t i = active ? active[k] : k;
	last[i] = fsqrt<F>(a0[i] * a0[i] + a1[i] * a1[i] + a2[i] * a2[i]);
	a0[i] = a1[i] = a2[i] = 0;
}

int tvg_impl_save_last_accel(tvg_context *ctx)
{
	// with an active list its length is read on the device (the list may be
	// built in the same captured step)
	const int64_t n = ctx->n;
	const int32_t *act = ctx->use_active ? ctx->active : nullptr;
	const int64_t *nd = ctx->use_active ? &ctx->dc->n_active : nullptr;
	if (!n) return TVG_OK;
	if (ctx->cfg.float_bytes == 4)
		k_save_last<float><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, ctx->stream>>>(
		    n, nd, act, (float *) ctx->f[FS_ACC0], (float *) ctx->f[FS_ACC1], (float *) ctx->f[FS_ACC2],
		    (float *) ctx->f[FS_LAST_ACC]);
	else
		k_save_last<double><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, ctx->stream>>>(
		    n, nd, act, (double *) ctx->f[FS_ACC0], (double *) ctx->f[FS_ACC1], (double *) ctx->f[FS_ACC2],
		    (double *) ctx->f[FS_LAST_ACC]);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

template <typename F>
__global__ void k_zero_active(int64_t n, const int32_t *__restrict__ active, F *a0, F *a1, F *a2,
                              F *g0, F *g1, F *g2, F *cost)
{
	const int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (k >= n) return;
	const int64_t i = active[k];
	a0[i] = a1[i] = a2[i] = 0;
	g0[i] = g1[i] = g2[i] = 0;
	cost[i] = 0;
}

// Acc, Grav_Acc and Cost of the active particles (all when no list is set)
int tvg_impl_zero_accel(tvg_context *ctx)
{
	if (ctx->use_active) {
		const int64_t n = ctx->n_active;
		if (!n) return TVG_OK;
		void **f = ctx->f;
		if (ctx->cfg.float_bytes == 4)
			k_zero_active<float><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, ctx->stream>>>(
			    n, ctx->active, (float *) f[FS_ACC0], (float *) f[FS_ACC1], (float *) f[FS_ACC2],
			    (float *) f[FS_GACC0], (float *) f[FS_GACC1], (float *) f[FS_GACC2], (float *) f[FS_COST]);
		else
			k_zero_active<double><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, ctx->stream>>>(
			    n, ctx->active, (double *) f[FS_ACC0], (double *) f[FS_ACC1], (double *) f[FS_ACC2],
			    (double *) f[FS_GACC0], (double *) f[FS_GACC1], (double *) f[FS_GACC2],
			    (double *) f[FS_COST]);
		TVG_CUDA(ctx, cudaGetLastError());
		return TVG_OK;
	}
	const size_t b = tvg_fsize(ctx) * ctx->n;
	const int slots[] = { FS_ACC0, FS_ACC1, FS_ACC2, FS_GACC0, FS_GACC1, FS_GACC2, FS_COST, FS_GRAV_POT };
	for (int s : slots) TVG_CUDA(ctx, cudaMemsetAsync(ctx->f[s], 0, b, ctx->stream));
	return TVG_OK;
}
