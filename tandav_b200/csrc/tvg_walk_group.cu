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
// Two lists: sources whose distance to the group box exceeds the softening
// length and that lie away from the half-box plane go to the far list, whose
// pair kernel is the bare 1/r^2 law (one MUFU.RSQ and ~12 FP32 instructions);
// the rest (the group's own particles, sources inside the softening length,
// and sources within two group half-widths of the half-box plane, whose image
// is chosen per target) go to the near list with the full softened kernel.
//
// Precision: positions are 32-bit integer box coordinates (2^32 per box when
// periodic, so that integer wrap-around is the nearest image; 2^31 per
// domain when isolated). Each list entry is converted once to an FP32 offset
// from the group centre; the pair loop then runs in FP32 with FP32
// accumulation.
//
// Ewald part: the reference's Ewald walk rules (tree_periodic.c:112-422): a
// node is opened only when it wants opening and straddles the half-box plane
// for some target or is larger than 0.2 L; everything else contributes its
// monopole's Ewald correction, evaluated per target from the FP32 65^3 table
// (trilinear, Gravity/periodic.c:35-113).
//
// Roofline: FP32 pipe bound in the pair loop; 20 flop per interaction by
// convention.
#include <stdlib.h>

#include "tvg_internal.cuh"

#define GW_WARPS 4
#define GW_THREADS (GW_WARPS * 32)
#define GW_STACK 1024
#define GW_LIST 256
#define GW_WLIST 64
#define GW_BQ 64
#define GW_DEFAULT_TPL 1

// -------------------------------------------------- integer coordinates

template <typename F>
__global__ void k_int_pos(int64_t n, const F *__restrict__ x, const F *__restrict__ y,
                          const F *__restrict__ z, double ox, double oy, double oz, double fac,
                          uint32_t *__restrict__ ix, uint32_t *__restrict__ iy, uint32_t *__restrict__ iz)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	ix[i] = (uint32_t) (uint64_t) (((double) x[i] - ox) * fac);
	iy[i] = (uint32_t) (uint64_t) (((double) y[i] - oy) * fac);
	iz[i] = (uint32_t) (uint64_t) (((double) z[i] - oz) * fac);
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
__global__ void k_wt_nchild(int64_t nn, const GNode<F> *__restrict__ tree, int32_t *__restrict__ nch)
{
	const int64_t g = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (g >= nn) return;
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
	nch[g] = cnt;
}

__device__ __forceinline__ uint32_t to_int(double v, double o, double fac)
{
	return (uint32_t) (uint64_t) ((v - o) * fac);
}

template <typename F>
__global__ void k_wt_emit(int64_t nn, int ntop, const GNode<F> *__restrict__ tree,
                          const int32_t *__restrict__ nch, const int32_t *__restrict__ choff,
                          double ox, double oy, double oz, double fac, double dsize,
                          tvg_wnode *__restrict__ wt)
{
	const int64_t g = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (g >= nn) return;
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
}

// top nodes without subtree: one bundle record each (their First_Part; the
// reference's interact_with_topnode_particles reads from Target instead,
// quirk Q3, which the group form does not repeat)
__global__ void k_wt_small_top(int ntop, const tvg_topnode *__restrict__ top, int vsize, double ox,
                               double oy, double oz, double fac, double dsize, tvg_wnode *__restrict__ wt)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= ntop || top[t].npart > vsize) return;
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
}

// ------------------------------------------------------------- the walk

struct GroupParams {
	int64_t n;
	int64_t ngroups;
	int gsize;
	int ntop;
	int periodic;
	int use_bh;
	float scale;        // length per integer unit
	float box, half_box;
	float theta2;       // TREE_OPEN_PARAM_BH
	float rel_fac;      // TREE_OPEN_PARAM_REL / G
	float gravity;
	float eps2, inv_eps2, c16;     // softening (h^2, 1/h^2, 1/(16 h^3))
	float near2;        // h^2 with a rounding margin: closer sources use the softened kernel
	float box2grid;
};

struct WarpSmem {
	int32_t stack[GW_STACK];
	float4 list[GW_LIST];      // far sources (plain 1/r^2), or Ewald sources
	float4 wlist[GW_WLIST];    // near or wrapped sources (softened kernel, per-target image)
	int2 bq[GW_BQ];
};

struct Target {
	float tx, ty, tz;       // offset from the group centre
	float ax, ay, az;
	float cost;
	bool valid;
};

// a source certainly outside the softening length of every target: 1/r^2 law
__device__ __forceinline__ void pair_far(float4 s, Target &t)
{
	const float dx = s.x - t.tx, dy = s.y - t.ty, dz = s.z - t.tz;
	const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
	const float ri = rsqrtf(r2);
	const float f = (s.w * ri) * (ri * ri);
	t.ax = fmaf(f, dx, t.ax);
	t.ay = fmaf(f, dy, t.ay);
	t.az = fmaf(f, dz, t.az);
}

// softened monopole, reference kernel (Dehnen K1 with h = -41/32 eps,
// tree_accel.c:362-394) in FP32; the r2 = 0 self term selects the inner
// branch and adds exactly zero
__device__ __forceinline__ void pair_full(const GroupParams &p, float4 s, Target &t)
{
	const float dx = s.x - t.tx, dy = s.y - t.ty, dz = s.z - t.tz;
	const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
	const float ri = rsqrtf(r2);
	const float fout = ri * ri * ri;
	const float u2 = r2 * p.inv_eps2;
	const float fin = fmaf(u2, fmaf(u2, 135.0f, -294.0f), 175.0f) * p.c16;
	const float f = s.w * (r2 < p.eps2 ? fin : fout);
	t.ax = fmaf(f, dx, t.ax);
	t.ay = fmaf(f, dy, t.ay);
	t.az = fmaf(f, dz, t.az);
}

template <int TPL>
__device__ __forceinline__ void flush_far(const float4 *list, int nl, Target (&t)[TPL])
{
	int e = 0;
#pragma unroll 1
	for (; e + 4 <= nl; e += 4) {
		const float4 s0 = list[e], s1 = list[e + 1], s2 = list[e + 2], s3 = list[e + 3];
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			pair_far(s0, t[k]);
			pair_far(s1, t[k]);
			pair_far(s2, t[k]);
			pair_far(s3, t[k]);
		}
	}
	for (; e < nl; e++) {
		const float4 s = list[e];
#pragma unroll
		for (int k = 0; k < TPL; k++) pair_far(s, t[k]);
	}
#pragma unroll
	for (int k = 0; k < TPL; k++) t[k].cost += (float) nl;
}

__device__ __forceinline__ float wrap_half(float d, float box, float half)
{
	d = d > half ? d - box : d;
	return d < -half ? d + box : d;
}

template <int TPL>
__device__ __forceinline__ void flush_slow(const GroupParams &p, const float4 *list, int nl,
                                           Target (&t)[TPL])
{
	for (int e = 0; e < nl; e++) {
		const float4 s = list[e];
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			float4 q = s;
			if (p.periodic) {
				q.x = wrap_half(s.x - t[k].tx, p.box, p.half_box) + t[k].tx;
				q.y = wrap_half(s.y - t[k].ty, p.box, p.half_box) + t[k].ty;
				q.z = wrap_half(s.z - t[k].tz, p.box, p.half_box) + t[k].tz;
			}
			pair_full(p, q, t[k]);
		}
	}
#pragma unroll
	for (int k = 0; k < TPL; k++) t[k].cost += (float) nl;
}

// Ewald_Correction (Gravity/periodic.c:35-113) in FP32 for one separation
__device__ __forceinline__ void ewald_table(const GroupParams &p, const float *__restrict__ fx,
                                            const float *__restrict__ fy, const float *__restrict__ fz,
                                            float dx, float dy, float dz, float out[3])
{
	const float sx = dx < 0 ? 1.f : -1.f, sy = dy < 0 ? 1.f : -1.f, sz = dz < 0 ? 1.f : -1.f;
	float u = fabsf(dx) * p.box2grid, v = fabsf(dy) * p.box2grid, w = fabsf(dz) * p.box2grid;
	int i = min((int) u, 63), j = min((int) v, 63), k = min((int) w, 63);
	u -= i; v -= j; w -= k;
	const int b = (i * 65 + j) * 65 + k;
	const float w000 = (1 - u) * (1 - v) * (1 - w), w001 = (1 - u) * (1 - v) * w,
	            w010 = (1 - u) * v * (1 - w), w011 = (1 - u) * v * w, w100 = u * (1 - v) * (1 - w),
	            w101 = u * (1 - v) * w, w110 = u * v * (1 - w), w111 = u * v * w;
	const float *T[3] = { fx, fy, fz };
#pragma unroll
	for (int d = 0; d < 3; d++) {
		const float *tb = T[d];
		out[d] = w000 * __ldg(tb + b) + w001 * __ldg(tb + b + 1) + w010 * __ldg(tb + b + 65)
		       + w011 * __ldg(tb + b + 66) + w100 * __ldg(tb + b + 4225) + w101 * __ldg(tb + b + 4226)
		       + w110 * __ldg(tb + b + 4290) + w111 * __ldg(tb + b + 4291);
	}
	out[0] *= sx;
	out[1] *= sy;
	out[2] *= sz;
}

template <int TPL>
__device__ __forceinline__ void flush_ewald(const GroupParams &p, const float4 *list, int nl,
                                            const float *fx, const float *fy, const float *fz,
                                            Target (&t)[TPL])
{
	for (int e = 0; e < nl; e++) {
		const float4 s = list[e];
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			const float dx = wrap_half(s.x - t[k].tx, p.box, p.half_box);
			const float dy = wrap_half(s.y - t[k].ty, p.box, p.half_box);
			const float dz = wrap_half(s.z - t[k].tz, p.box, p.half_box);
			if (dx == 0.f && dy == 0.f && dz == 0.f) continue;      // self
			float c[3];
			ewald_table(p, fx, fy, fz, dx, dy, dz, c);
			t[k].ax = fmaf(s.w, c[0], t[k].ax);
			t[k].ay = fmaf(s.w, c[1], t[k].ay);
			t[k].az = fmaf(s.w, c[2], t[k].az);
			t[k].cost += 1.f;
		}
	}
}

// one group: 32 * TPL PH-contiguous active particles, lane l holds the
// particles first + l + 32 k
template <bool EWALD, int TPL>
__device__ void walk_group(const GroupParams &p, WarpSmem &S, const tvg_wnode *__restrict__ wt,
                           const uint32_t *__restrict__ ix, const uint32_t *__restrict__ iy,
                           const uint32_t *__restrict__ iz, const float *__restrict__ mass_f,
                           const float *__restrict__ last_acc, const float *fx, const float *fy,
                           const float *fz, int64_t first, int cnt, const int32_t *__restrict__ active,
                           Target (&t)[TPL], int *status)
{
	const int lane = threadIdx.x & 31;
	const unsigned lt = (1u << lane) - 1u;
	uint32_t px[TPL], py[TPL], pz[TPL];
	int64_t me0 = active ? (int64_t) active[first] : first;
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
	const uint32_t cx = rx + (uint32_t) (((int64_t) minx + maxx) >> 1);
	const uint32_t cy = ry + (uint32_t) (((int64_t) miny + maxy) >> 1);
	const uint32_t cz = rz + (uint32_t) (((int64_t) minz + maxz) >> 1);
	const float hx = ((float) ((int64_t) maxx - minx) * 0.5f + 1.f) * p.scale;
	const float hy = ((float) ((int64_t) maxy - miny) * 0.5f + 1.f) * p.scale;
	const float hz = ((float) ((int64_t) maxz - minz) * 0.5f + 1.f) * p.scale;
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		// rounded products (no FMA contraction into the later subtraction): a
		// particle's own list entry must sit at exactly zero separation, since
		// the reference's inner kernel (h < 0) turns any residue into a force
		t[k].tx = __fmul_rn((float) (int) (px[k] - cx), p.scale);
		t[k].ty = __fmul_rn((float) (int) (py[k] - cy), p.scale);
		t[k].tz = __fmul_rn((float) (int) (pz[k] - cz), p.scale);
		t[k].ax = t[k].ay = t[k].az = 0.f;
		t[k].cost = 0.f;
	}
	// group-wide relative criterion: the smallest |a_old| opens the most
#pragma unroll
	for (int o = 16; o; o >>= 1) amin = fminf(amin, __shfl_xor_sync(0xFFFFFFFFu, amin, o));
	const float fac = amin * p.rel_fac;
	// a source this close to the half-box plane needs per-target images
	const float wlimx = p.half_box - 2.f * hx, wlimy = p.half_box - 2.f * hy,
	            wlimz = p.half_box - 2.f * hz;

	int sp = 0, nl = 0, nw = 0;
	for (int r = lane; r < p.ntop; r += 32) S.stack[r] = r;
	sp = p.ntop;
	__syncwarp();
	int guard = 0;
	while (sp > 0) {
		if (++guard > (1 << 24)) { atomicOr(status, TVG_ST_TIMEOUT); break; }
		int k = min(32, sp);
		const int room = (GW_STACK - sp) / 7;
		if (room < k) k = room;
		if (k <= 0) { atomicOr(status, TVG_ST_LIST_OVERFLOW); break; }
		int node = -1;
		if (lane < k) node = S.stack[sp - 1 - lane];
		sp -= k;
		__syncwarp();
		bool accept = false, open_int = false, open_bundle = false, slow = false;
		float4 entry = make_float4(0.f, 0.f, 0.f, 0.f);
		int nchild = 0, child = 0;
		if (node >= 0) {
			const tvg_wnode nd = wt[node];
			const float dx = __fmul_rn((float) (int) (nd.cx - cx), p.scale);
			const float dy = __fmul_rn((float) (int) (nd.cy - cy), p.scale);
			const float dz = __fmul_rn((float) (int) (nd.cz - cz), p.scale);
			const float qx = fmaxf(fabsf(dx) - hx, 0.f), qy = fmaxf(fabsf(dy) - hy, 0.f),
			            qz = fmaxf(fabsf(dz) - hz, 0.f);
			const float r2 = qx * qx + qy * qy + qz * qz;
			bool want;
			if (p.use_bh) want = nd.size2 > r2 * p.theta2;
			else want = nd.mass * nd.size2 > r2 * r2 * fac;
			const float gx = __fmul_rn((float) (int) (nd.gx - cx), p.scale);
			const float gy = __fmul_rn((float) (int) (nd.gy - cy), p.scale);
			const float gz = __fmul_rn((float) (int) (nd.gz - cz), p.scale);
			const float lim = 0.6f * nd.size;
			if (fabsf(gx) < lim + hx && fabsf(gy) < lim + hy && fabsf(gz) < lim + hz) want = true;
			// a bundle below the top level is never a monopole: the reference
			// interacts its particles whenever the walk reaches it
			// (tree_accel.c:221-243, tree_periodic.c:228-251)
			const bool force_open = nd.nchild < 0 && node >= p.ntop;
			bool open = want || force_open;
			if (EWALD && want) {
				// open only when the node straddles the half-box plane for some
				// target, or is larger than 0.2 L (tree_periodic.c:158-172, 278-310)
				const float dl = 0.5f * (p.box - nd.size);
				open = force_open || fabsf(gx) + hx > dl || fabsf(gy) + hy > dl
				    || fabsf(gz) + hz > dl || nd.size > 0.2f * p.box;
			}
			if (!open) {
				accept = true;
				entry = make_float4(dx, dy, dz, p.gravity * nd.mass);
				slow = (p.periodic && (fabsf(dx) > wlimx || fabsf(dy) > wlimy || fabsf(dz) > wlimz))
				    || r2 < p.near2;
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
		const bool to_main = accept && (EWALD || !slow);
		const bool to_slow = accept && !EWALD && slow;
		const unsigned bm = __ballot_sync(0xFFFFFFFFu, to_main);
		const unsigned bw = __ballot_sync(0xFFFFFFFFu, to_slow);
		if (nl + __popc(bm) > GW_LIST) {
			if (EWALD) flush_ewald<TPL>(p, S.list, nl, fx, fy, fz, t);
			else flush_far<TPL>(S.list, nl, t);
			nl = 0;
			__syncwarp();
		}
		if (!EWALD && nw + __popc(bw) > GW_WLIST) {
			flush_slow<TPL>(p, S.wlist, nw, t);
			nw = 0;
			__syncwarp();
		}
		if (to_main) S.list[nl + __popc(bm & lt)] = entry;
		if (to_slow) S.wlist[nw + __popc(bw & lt)] = entry;
		nl += __popc(bm);
		nw += __popc(bw);
		// children -> stack (exclusive prefix sum of child counts)
		int c = open_int ? nchild : 0, incl = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			int u = __shfl_up_sync(0xFFFFFFFFu, incl, o);
			if (lane >= o) incl += u;
		}
		const int tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
		for (int q = 0; q < c; q++) S.stack[sp + incl - c + q] = child + c - 1 - q;
		sp += tot;
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
				bool sl = false;
				if (have) {
					const int64_t jp = (int64_t) q.x + j;
					e.x = __fmul_rn((float) (int) (ix[jp] - cx), p.scale);
					e.y = __fmul_rn((float) (int) (iy[jp] - cy), p.scale);
					e.z = __fmul_rn((float) (int) (iz[jp] - cz), p.scale);
					e.w = p.gravity * mass_f[jp];
					if (!EWALD) {
						const float ax = fmaxf(fabsf(e.x) - hx, 0.f), ay = fmaxf(fabsf(e.y) - hy, 0.f),
						            az = fmaxf(fabsf(e.z) - hz, 0.f);
						sl = ax * ax + ay * ay + az * az < p.near2
						  || (p.periodic && (fabsf(e.x) > wlimx || fabsf(e.y) > wlimy || fabsf(e.z) > wlimz));
					}
				}
				const bool tm = have && !sl, tw = have && sl;
				const unsigned m1 = __ballot_sync(0xFFFFFFFFu, tm), m2 = __ballot_sync(0xFFFFFFFFu, tw);
				if (nl + __popc(m1) > GW_LIST) {
					if (EWALD) flush_ewald<TPL>(p, S.list, nl, fx, fy, fz, t);
					else flush_far<TPL>(S.list, nl, t);
					nl = 0;
					__syncwarp();
				}
				if (!EWALD && nw + __popc(m2) > GW_WLIST) {
					flush_slow<TPL>(p, S.wlist, nw, t);
					nw = 0;
					__syncwarp();
				}
				if (tm) S.list[nl + __popc(m1 & lt)] = e;
				if (tw) S.wlist[nw + __popc(m2 & lt)] = e;
				nl += __popc(m1);
				nw += __popc(m2);
				__syncwarp();
			}
		}
		__syncwarp();
	}
	__syncwarp();
	if (EWALD) {
		flush_ewald<TPL>(p, S.list, nl, fx, fy, fz, t);
	} else {
		flush_far<TPL>(S.list, nl, t);
		flush_slow<TPL>(p, S.wlist, nw, t);
		// the self pair is counted by the list but not by the reference
#pragma unroll
		for (int k = 0; k < TPL; k++) t[k].cost -= 1.f;
	}
	__syncwarp();
}

template <bool EWALD, int TPL, typename F>
__global__ void __launch_bounds__(GW_THREADS)
k_walk_group(GroupParams p, const int32_t *__restrict__ active, const tvg_wnode *__restrict__ wt,
             const uint32_t *__restrict__ ix, const uint32_t *__restrict__ iy,
             const uint32_t *__restrict__ iz, const float *__restrict__ mass_f,
             const float *__restrict__ last_acc, const float *fx, const float *fy, const float *fz,
             F *acc0, F *acc1, F *acc2, F *gacc0, F *gacc1, F *gacc2, F *cost_out, int32_t *work,
             double *counter, int *status)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	WarpSmem &S = ((WarpSmem *) smem_raw)[threadIdx.x >> 5];
	const int lane = threadIdx.x & 31;
	double cnt_acc = 0;
	for (;;) {
		int64_t g = 0;
		if (lane == 0) g = atomicAdd(work, 1);
		g = __shfl_sync(0xFFFFFFFFu, g, 0);
		if (g >= p.ngroups) break;
		const int64_t first = g * p.gsize;
		const int cnt = (int) min((int64_t) p.gsize, p.n - first);
		Target t[TPL];
		walk_group<EWALD, TPL>(p, S, wt, ix, iy, iz, mass_f, last_acc, fx, fy, fz, first, cnt, active,
		                       t, status);
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			if (!t[k].valid) continue;
			const int slot = lane + 32 * k;
			const int64_t i = active ? (int64_t) active[first + slot] : first + slot;
			acc0[i] += (F) t[k].ax;
			acc1[i] += (F) t[k].ay;
			acc2[i] += (F) t[k].az;
			if (EWALD) {
				gacc0[i] += (F) t[k].ax;
				gacc1[i] += (F) t[k].ay;
				gacc2[i] += (F) t[k].az;
				cost_out[i] += (F) t[k].cost;
			} else {
				gacc0[i] = (F) t[k].ax;
				gacc1[i] = (F) t[k].ay;
				gacc2[i] = (F) t[k].az;
				cost_out[i] = (F) t[k].cost;
			}
			cnt_acc += t[k].cost;
		}
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) cnt_acc += __shfl_xor_sync(0xFFFFFFFFu, cnt_acc, o);
	if (lane == 0 && cnt_acc != 0) atomicAdd(counter, cnt_acc);
}

template <typename F>
__global__ void k_to_float(int64_t n, const F *__restrict__ a, float *__restrict__ b)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) b[i] = (float) a[i];
}

template <typename F>
static int prepare_typed(tvg_context *ctx)
{
	const int64_t n = ctx->n, nn = ctx->nnodes;
	cudaStream_t s = ctx->stream;
	const double fac = ctx->cfg.periodic ? 4294967296.0 / ctx->dsize : 2147483648.0 / ctx->dsize;
	k_int_pos<F><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(
	    n, (const F *) ctx->f[FS_POS0], (const F *) ctx->f[FS_POS1], (const F *) ctx->f[FS_POS2],
	    ctx->origin[0], ctx->origin[1], ctx->origin[2], fac, ctx->ipos[0], ctx->ipos[1], ctx->ipos[2]);
	TVG_CUDA(ctx, cudaGetLastError());
	int32_t *nch = ctx->u_count, *choff = ctx->u_endu;     // free after the build
	if (nn > 0) {
		const GNode<F> *tree = (const GNode<F> *) ctx->tree;
		k_wt_nchild<F><<<TVG_CNT(ctx, tvg_blocks(nn, 256)), 256, 0, s>>>(nn, tree, nch);
		TVG_CUDA(ctx, cudaGetLastError());
		TVG_CHECK(tvg_device_scan_i32(ctx, nch, choff, nn, nullptr));
		k_wt_emit<F><<<TVG_CNT(ctx, tvg_blocks(nn, 256)), 256, 0, s>>>(nn, ctx->ntop, tree, nch, choff,
		                                                 ctx->origin[0], ctx->origin[1],
		                                                 ctx->origin[2], fac, ctx->dsize, ctx->wtree);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	k_wt_small_top<<<TVG_CNT(ctx, 1), 64, 0, s>>>(ctx->ntop, ctx->d_top, ctx->cfg.vector_size, ctx->origin[0],
	                                 ctx->origin[1], ctx->origin[2], fac, ctx->dsize, ctx->wtree);
	TVG_CUDA(ctx, cudaGetLastError());
	ctx->have_walktree = true;
	return TVG_OK;
}

// targets per lane: 1 (32-particle groups) or 2 (64); TVG_GROUP_TPL overrides
static int group_tpl()
{
	static int tpl = 0;
	if (!tpl) {
		const char *e = getenv("TVG_GROUP_TPL");
		tpl = (e && atoi(e) == 1) ? 1 : (e && atoi(e) == 2) ? 2 : GW_DEFAULT_TPL;
	}
	return tpl;
}

template <bool EWALD, int TPL, typename F>
static int launch_walk(tvg_context *ctx, GroupParams p, const float *mass_f, const float *last_f,
                       const float *fx, const float *fy, const float *fz, double *counter)
{
	static int nblk = 0;
	const size_t smem = sizeof(WarpSmem) * GW_WARPS;
	if (!nblk) {
		TVG_CUDA(ctx, cudaFuncSetAttribute(k_walk_group<EWALD, TPL, F>,
		                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
		int per_sm = 0, nsm = 0;
		TVG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_group<EWALD, TPL, F>,
		                                                             GW_THREADS, smem));
		TVG_CUDA(ctx, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
		nblk = (per_sm > 0 ? per_sm : 1) * nsm;
	}
	p.gsize = 32 * TPL;
	p.ngroups = (p.n + p.gsize - 1) / p.gsize;
	k_walk_group<EWALD, TPL, F><<<TVG_CNT(ctx, nblk), GW_THREADS, smem, ctx->stream>>>(
	    p, ctx->use_active ? ctx->active : nullptr, ctx->wtree, ctx->ipos[0], ctx->ipos[1],
	    ctx->ipos[2], mass_f, last_f, fx, fy, fz, (F *) ctx->f[FS_ACC0], (F *) ctx->f[FS_ACC1],
	    (F *) ctx->f[FS_ACC2], (F *) ctx->f[FS_GACC0], (F *) ctx->f[FS_GACC1], (F *) ctx->f[FS_GACC2],
	    (F *) ctx->f[FS_COST], ctx->work_counter, counter, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

template <typename F>
static int walk_group_typed(tvg_context *ctx, int use_bh, uint32_t parts, int ewald_kind)
{
	const int64_t n = ctx->n;
	if (n == 0) return TVG_OK;
	if (ewald_kind != TVG_EWALD_TABLE && (parts & TVG_WALK_EWALD))
		return tvg_fail(ctx, TVG_E_STATE, "learned Ewald correction not loaded");
	cudaStream_t s = ctx->stream;
	if (!ctx->have_walktree) TVG_CHECK(prepare_typed<F>(ctx));
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
	const float *fx = nullptr, *fy = nullptr, *fz = nullptr;
	if (parts & TVG_WALK_EWALD) {
		if (sizeof(F) == 8) {
			// FP32 tables for the group form
			const int npt = 65 * 65 * 65;
			if (!ctx->ewald32) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->ewald32, 3 * 4 * (size_t) npt));
			float *tf = ctx->ewald32;
			for (int d = 0; d < 3; d++)
				k_to_float<F><<<TVG_CNT(ctx, tvg_blocks(npt, 256)), 256, 0, s>>>(npt, (const F *) ctx->ewald_f[d],
				                                                    tf + d * npt);
			fx = tf; fy = tf + npt; fz = tf + 2 * npt;
		} else {
			fx = (const float *) ctx->ewald_f[0];
			fy = (const float *) ctx->ewald_f[1];
			fz = (const float *) ctx->ewald_f[2];
		}
	}
	const tvg_config &cf = ctx->cfg;
	GroupParams p;
	p.n = ctx->use_active ? ctx->n_active : n;
	p.ntop = ctx->ntop;
	p.periodic = cf.periodic;
	p.use_bh = use_bh;
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
	p.box2grid = (float) (cf.periodic ? 2.0 * 64.0 / cf.boxsize : 0.0);
	const int tpl = group_tpl();
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->counters, 0, 16, s));
	for (int part = 0; part < 2; part++) {
		const bool ew = part == 1;
		if (!(parts & (ew ? TVG_WALK_EWALD : TVG_WALK_GRAVITY))) continue;
		TVG_CUDA(ctx, cudaMemsetAsync(ctx->work_counter, 0, 4, s));
		TVG_CUDA(ctx, cudaEventRecord(ctx->ev[0], s));
		double *cnt = ctx->counters + (ew ? 1 : 0);
		if (ew && tpl == 1) TVG_CHECK((launch_walk<true, 1, F>(ctx, p, mass_f, last_f, fx, fy, fz, cnt)));
		else if (ew) TVG_CHECK((launch_walk<true, 2, F>(ctx, p, mass_f, last_f, fx, fy, fz, cnt)));
		else if (tpl == 1) TVG_CHECK((launch_walk<false, 1, F>(ctx, p, mass_f, last_f, fx, fy, fz, cnt)));
		else TVG_CHECK((launch_walk<false, 2, F>(ctx, p, mass_f, last_f, fx, fy, fz, cnt)));
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

int tvg_impl_walk_group(tvg_context *ctx, int use_bh, uint32_t parts, int ewald_kind)
{
	if (ctx->cfg.float_bytes == 4) return walk_group_typed<float>(ctx, use_bh, parts, ewald_kind);
	return walk_group_typed<double>(ctx, use_bh, parts, ewald_kind);
}
