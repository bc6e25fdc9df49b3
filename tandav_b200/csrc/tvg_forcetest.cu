// tvg_forcetest.cu -- Gravity_Forcetest (Gravity/forcetest.c:25-172) on the GPU.
//
// FP64 direct summation over all resident particles for a list of target
// particles, with the reference's softened kernel (h = -41/32 eps, the same
// branch and polynomial as forcetest.c:81-99 and tree_accel.c:362-394) on the
// nearest image. In a periodic box the sum is Ewald-summed, not tabulated:
//
//   a_i = sum_j [ K_soft(d_ij) - G m_j d_ij / r^3 (erf(a r) - 2 a r / sqrt(pi) e^{-a^2 r^2}) ]
//       + (4 G / L^2) sum_{h in half space} h / |h|^2 e^{-pi^2 |h|^2 / (a L)^2}
//                     [cos(k.x_i) S_s(k) - sin(k.x_i) S_c(k)],   k = 2 pi h / L
//
// with d_ij the nearest-image separation (source minus target), S_c + i S_s
// = sum_j m_j e^{i k.x_j} the structure factor, and a L = 12: the real-space
// terms of all further images are below erfc(6) ~ 2e-17 of their Newtonian
// value, and the k-space sum is cut at |h|^2 <= 576 where its terms fall
// below e^{-39} ~ 1e-17. Softened Newton on the nearest image plus this sum is
// exactly what the reference's tree adds up (nearest image + Ewald_Correction,
// whose table is the same sum at a L = 2 with images to |n|, |h| <= 4,
// Gravity/periodic.c:368-411), minus the table's interpolation error.
//
// parts selects the sum: TVG_WALK_GRAVITY alone is the nearest-image softened
// sum (what the gravity walk approximates), with TVG_WALK_EWALD the Ewald sum
// (what gravity + Ewald walks approximate together).
//
// Error statistics compare the resident Grav_Acc (the walk's output) with the
// direct sum: e = |a_tree - a_direct| / |a_direct| per target; rms, 99th
// percentile (nearest rank), mean and max.
//
// Cost at 16.7M sources and 10^4 targets: 1.7e11 FP64 pair terms (~100 FP64
// instructions each, erfc and exp) plus 5e11 structure-factor terms.
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "tvg_internal.cuh"

#define FT_THREADS 256
#define FT_DCHUNKS 64          // source chunks of the real-space sum
#define FT_SCHUNKS 32          // source chunks of the structure factor
#define FT_ALPHA_L 12.0
#define FT_HMAX 24
#define FT_H2 576
#define FT_KPT 4               // k-vectors per thread in the structure factor
#define FT_STILE 32            // sources per shared-memory tile

struct FtParams {
	int64_t n, nt, chunk;
	int periodic, ewald;
	double box, half_box;
	double G, h2, c16;         // softening: h^2 and 1/(16 h^3), h = -41/32 eps
	double alpha, c2a;         // Ewald alpha and 2 alpha / sqrt(pi)
};

template <typename F>
__global__ void k_ft_gather(int64_t nt, const int64_t *__restrict__ idx, const F *x, const F *y,
                            const F *z, const F *gx, const F *gy, const F *gz, double *tp,
                            double *ta)
{
	const int64_t t = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (t >= nt) return;
	const int64_t i = idx[t];
	tp[t] = (double) x[i];
	tp[nt + t] = (double) y[i];
	tp[2 * nt + t] = (double) z[i];
	ta[t] = (double) gx[i];
	ta[nt + t] = (double) gy[i];
	ta[2 * nt + t] = (double) gz[i];
}

// real-space part: one thread per target, sources of one chunk staged in
// shared memory; partial sums per chunk, added in chunk order later
template <typename F>
__global__ void __launch_bounds__(FT_THREADS)
k_ft_direct(FtParams p, const F *__restrict__ x, const F *__restrict__ y, const F *__restrict__ z,
            const F *__restrict__ m, const double *__restrict__ tp, double *part)
{
	__shared__ double sx[FT_THREADS], sy[FT_THREADS], sz[FT_THREADS], sm[FT_THREADS];
	const int64_t t = blockIdx.x * (int64_t) FT_THREADS + threadIdx.x;
	const bool have = t < p.nt;
	const double xi = have ? tp[t] : 0.0, yi = have ? tp[p.nt + t] : 0.0,
	             zi = have ? tp[2 * p.nt + t] : 0.0;
	const int64_t j0 = blockIdx.y * p.chunk, j1 = min(p.n, j0 + p.chunk);
	double ax = 0, ay = 0, az = 0;
	for (int64_t b = j0; b < j1; b += FT_THREADS) {
		const int64_t j = b + threadIdx.x;
		__syncthreads();
		if (j < j1) {
			sx[threadIdx.x] = (double) x[j];
			sy[threadIdx.x] = (double) y[j];
			sz[threadIdx.x] = (double) z[j];
			sm[threadIdx.x] = (double) m[j];
		}
		__syncthreads();
		const int nb = (int) min((int64_t) FT_THREADS, j1 - b);
		for (int s = 0; s < nb; s++) {
			double dx = sx[s] - xi, dy = sy[s] - yi, dz = sz[s] - zi;
			if (p.periodic) {       // Periodic_Nearest (periodic.c:62-80)
				dx = dx > p.half_box ? dx - p.box : (dx < -p.half_box ? dx + p.box : dx);
				dy = dy > p.half_box ? dy - p.box : (dy < -p.half_box ? dy + p.box : dy);
				dz = dz > p.half_box ? dz - p.box : (dz < -p.half_box ? dz + p.box : dz);
			}
			const double r2 = dx * dx + dy * dy + dz * dz;
			if (!(r2 > 0)) continue;        // forcetest.c:79
			const double ri = 1.0 / sqrt(r2);
			const double ri3 = ri * ri * ri;
			double fac;
			if (p.ewald) {
				const double r = r2 * ri, a = p.alpha * r;
				const double g = p.c2a * r * exp(-a * a);
				if (r2 < p.h2) {
					const double u2 = r2 / p.h2;
					fac = (175.0 - u2 * (294.0 - u2 * 135.0)) * p.c16 - ri3 * (erf(a) - g);
				} else {
					fac = ri3 * (erfc(a) + g);
				}
			} else {
				if (r2 < p.h2) {
					const double u2 = r2 / p.h2;
					fac = (175.0 - u2 * (294.0 - u2 * 135.0)) * p.c16;
				} else {
					fac = ri3;
				}
			}
			fac *= p.G * sm[s];
			ax += fac * dx;
			ay += fac * dy;
			az += fac * dz;
		}
	}
	if (have) {
		double *o = part + (int64_t) blockIdx.y * 3 * p.nt;
		o[t] = ax;
		o[p.nt + t] = ay;
		o[2 * p.nt + t] = az;
	}
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
	return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// structure factor S(k) = sum_j m_j e^{i k.x_j} over one source chunk for
// FT_THREADS * FT_KPT k-vectors; per-axis phase factors e^{2 pi i h x / L},
// h = 0..FT_HMAX, of a tile of sources are tabulated in shared memory
template <typename F>
__global__ void __launch_bounds__(FT_THREADS)
k_ft_structure(int64_t n, int64_t chunk, int nk, const char4 *__restrict__ hk, const F *x,
               const F *y, const F *z, const F *m, double two_over_box, double2 *partS)
{
	__shared__ double2 E[FT_STILE][3][FT_HMAX + 1];
	__shared__ double sm[FT_STILE];
	int kx[FT_KPT], ky[FT_KPT], kz[FT_KPT];
	double sc[FT_KPT], ss[FT_KPT];
#pragma unroll
	for (int r = 0; r < FT_KPT; r++) {
		const int k = blockIdx.x * FT_THREADS * FT_KPT + r * FT_THREADS + threadIdx.x;
		const char4 h = k < nk ? hk[k] : make_char4(0, 0, 0, 0);
		kx[r] = h.x; ky[r] = h.y; kz[r] = h.z;
		sc[r] = ss[r] = 0;
	}
	const int64_t j0 = blockIdx.y * chunk, j1 = min(n, j0 + chunk);
	const F *X[3] = { x, y, z };
	for (int64_t b = j0; b < j1; b += FT_STILE) {
		__syncthreads();
		for (int e = threadIdx.x; e < FT_STILE * 3 * (FT_HMAX + 1); e += FT_THREADS) {
			const int s = e / (3 * (FT_HMAX + 1)), rem = e % (3 * (FT_HMAX + 1));
			const int ax = rem / (FT_HMAX + 1), h = rem % (FT_HMAX + 1);
			const int64_t j = b + s;
			const double v = j < j1 ? (double) X[ax][j] : 0.0;
			double sn, cs;
			sincospi(v * two_over_box * h, &sn, &cs);
			E[s][ax][h] = make_double2(cs, sn);
		}
		if (threadIdx.x < FT_STILE) {
			const int64_t j = b + threadIdx.x;
			sm[threadIdx.x] = j < j1 ? (double) m[j] : 0.0;
		}
		__syncthreads();
		const int ns = (int) min((int64_t) FT_STILE, j1 - b);
		for (int s = 0; s < ns; s++) {
			const double ms = sm[s];
#pragma unroll
			for (int r = 0; r < FT_KPT; r++) {
				const double2 ex = E[s][0][kx[r]];
				double2 ey = E[s][1][abs(ky[r])], ez = E[s][2][abs(kz[r])];
				if (ky[r] < 0) ey.y = -ey.y;
				if (kz[r] < 0) ez.y = -ez.y;
				const double2 c = cmul(cmul(ex, ey), ez);
				sc[r] += ms * c.x;
				ss[r] += ms * c.y;
			}
		}
	}
#pragma unroll
	for (int r = 0; r < FT_KPT; r++) {
		const int k = blockIdx.x * FT_THREADS * FT_KPT + r * FT_THREADS + threadIdx.x;
		if (k < nk) partS[(int64_t) blockIdx.y * nk + k] = make_double2(sc[r], ss[r]);
	}
}

__global__ void k_ft_sum_structure(int nk, int nchunks, const double2 *partS, double2 *S)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nk) return;
	double2 a = make_double2(0, 0);
	for (int c = 0; c < nchunks; c++) {
		const double2 v = partS[(int64_t) c * nk + k];
		a.x += v.x;
		a.y += v.y;
	}
	S[k] = a;
}

// partial real-space sums in chunk order, plus the k-space sum
__global__ void k_ft_final(int64_t nt, int nchunks, const double *part, const double *tp, int nk,
                           const char4 *__restrict__ hk, const double *__restrict__ wk,
                           const double2 *__restrict__ S, double two_over_box, double *acc)
{
	const int64_t t = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (t >= nt) return;
	double ax = 0, ay = 0, az = 0;
	for (int c = 0; c < nchunks; c++) {
		const double *o = part + (int64_t) c * 3 * nt;
		ax += o[t];
		ay += o[nt + t];
		az += o[2 * nt + t];
	}
	const double xi = tp[t], yi = tp[nt + t], zi = tp[2 * nt + t];
	double kx = 0, ky = 0, kz = 0;
	for (int k = 0; k < nk; k++) {
		const char4 h = hk[k];
		double sn, cs;
		sincospi((h.x * xi + h.y * yi + h.z * zi) * two_over_box, &sn, &cs);
		const double2 s = S[k];
		const double v = wk[k] * (cs * s.y - sn * s.x);
		kx += v * h.x;
		ky += v * h.y;
		kz += v * h.z;
	}
	acc[t] = ax + kx;
	acc[nt + t] = ay + ky;
	acc[2 * nt + t] = az + kz;
}

namespace {

struct DevBufs {
	std::vector<void *> p;
	~DevBufs() { for (void *q : p) cudaFree(q); }
	int get(tvg_context *ctx, void **out, size_t bytes)
	{
		cudaError_t e = cudaMalloc(out, bytes ? bytes : 16);
		if (e != cudaSuccess) {
			cudaGetLastError();
			return tvg_fail(ctx, TVG_E_NOMEM, "forcetest: cudaMalloc(%zu) failed: %s", bytes,
			                cudaGetErrorString(e));
		}
		p.push_back(*out);
		return TVG_OK;
	}
};

}   // namespace

template <typename F>
static int forcetest_typed(tvg_context *ctx, bool ewald, int64_t nt, const int64_t *targets,
                           double *acc_direct, double *acc_tree, double *err)
{
	const int64_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	const tvg_config &cf = ctx->cfg;
	DevBufs B;
	int64_t *d_idx;
	double *tp, *ta, *part, *acc;
	TVG_CHECK(B.get(ctx, (void **) &d_idx, 8 * (size_t) nt));
	TVG_CHECK(B.get(ctx, (void **) &tp, 24 * (size_t) nt));
	TVG_CHECK(B.get(ctx, (void **) &ta, 24 * (size_t) nt));
	TVG_CHECK(B.get(ctx, (void **) &acc, 24 * (size_t) nt));
	TVG_CHECK(B.get(ctx, (void **) &part, 24 * (size_t) nt * FT_DCHUNKS));
	TVG_CUDA(ctx, cudaMemcpyAsync(d_idx, targets, 8 * (size_t) nt, cudaMemcpyHostToDevice, s));
	const F *X = (const F *) ctx->f[FS_POS0], *Y = (const F *) ctx->f[FS_POS1],
	        *Z = (const F *) ctx->f[FS_POS2], *M = (const F *) ctx->f[FS_MASS];
	k_ft_gather<F><<<TVG_CNT(ctx, tvg_blocks(nt, 256)), 256, 0, s>>>(
	    nt, d_idx, X, Y, Z, (const F *) ctx->f[FS_GACC0], (const F *) ctx->f[FS_GACC1],
	    (const F *) ctx->f[FS_GACC2], tp, ta);
	TVG_CUDA(ctx, cudaGetLastError());

	FtParams p;
	p.n = n;
	p.nt = nt;
	p.chunk = (n + FT_DCHUNKS - 1) / FT_DCHUNKS;
	p.periodic = cf.periodic;      // nearest image
	p.ewald = ewald;
	p.box = cf.periodic ? cf.boxsize : 0.0;
	p.half_box = 0.5 * p.box;
	p.G = cf.gravity;
	const double h = -41.0 / 32.0 * cf.softening;      // tree_build.c:136
	p.h2 = h * h;
	p.c16 = 1.0 / (16.0 * h * h * h);
	p.alpha = ewald ? FT_ALPHA_L / cf.boxsize : 0.0;
	p.c2a = 2.0 * p.alpha / sqrt(M_PI);
	const dim3 gd(tvg_blocks(nt, FT_THREADS), FT_DCHUNKS);
	k_ft_direct<F><<<TVG_CNT(ctx, gd), FT_THREADS, 0, s>>>(p, X, Y, Z, M, tp, part);
	TVG_CUDA(ctx, cudaGetLastError());

	// k-space: half space h_x > 0, or h_x = 0 and (h_y > 0, or h_y = 0 and h_z > 0)
	int nk = 0;
	char4 *d_hk = nullptr;
	double *d_wk = nullptr;
	double2 *d_S = nullptr;
	const double two_over_box = ewald ? 2.0 / cf.boxsize : 0.0;
	if (ewald) {
		std::vector<char4> hk;
		std::vector<double> wk;
		const double L = cf.boxsize, aL = FT_ALPHA_L;
		for (int hx = 0; hx <= FT_HMAX; hx++)
			for (int hy = -FT_HMAX; hy <= FT_HMAX; hy++)
				for (int hz = -FT_HMAX; hz <= FT_HMAX; hz++) {
					const int h2 = hx * hx + hy * hy + hz * hz;
					if (h2 == 0 || h2 > FT_H2) continue;
					if (hx == 0 && (hy < 0 || (hy == 0 && hz < 0))) continue;
					hk.push_back(make_char4((signed char) hx, (signed char) hy, (signed char) hz, 0));
					wk.push_back(4.0 * cf.gravity / (L * L) * exp(-M_PI * M_PI * h2 / (aL * aL)) / h2);
				}
		nk = (int) hk.size();
		double2 *partS;
		TVG_CHECK(B.get(ctx, (void **) &d_hk, sizeof(char4) * nk));
		TVG_CHECK(B.get(ctx, (void **) &d_wk, sizeof(double) * nk));
		TVG_CHECK(B.get(ctx, (void **) &d_S, sizeof(double2) * nk));
		TVG_CHECK(B.get(ctx, (void **) &partS, sizeof(double2) * nk * (size_t) FT_SCHUNKS));
		TVG_CUDA(ctx, cudaMemcpyAsync(d_hk, hk.data(), sizeof(char4) * nk, cudaMemcpyHostToDevice, s));
		TVG_CUDA(ctx, cudaMemcpyAsync(d_wk, wk.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, s));
		const int64_t chunk = (n + FT_SCHUNKS - 1) / FT_SCHUNKS;
		const dim3 gs((nk + FT_THREADS * FT_KPT - 1) / (FT_THREADS * FT_KPT), FT_SCHUNKS);
		k_ft_structure<F><<<TVG_CNT(ctx, gs), FT_THREADS, 0, s>>>(n, chunk, nk, d_hk, X, Y, Z, M,
		                                                          two_over_box, partS);
		TVG_CUDA(ctx, cudaGetLastError());
		k_ft_sum_structure<<<TVG_CNT(ctx, tvg_blocks(nk, 256)), 256, 0, s>>>(nk, FT_SCHUNKS, partS, d_S);
		TVG_CUDA(ctx, cudaGetLastError());
		// hold the host vectors until the copies are done
		TVG_CUDA(ctx, cudaStreamSynchronize(s));
	}
	k_ft_final<<<TVG_CNT(ctx, tvg_blocks(nt, 128)), 128, 0, s>>>(nt, FT_DCHUNKS, part, tp, nk, d_hk,
	                                                            d_wk, d_S, two_over_box, acc);
	TVG_CUDA(ctx, cudaGetLastError());
	std::vector<double> ad(3 * nt), at(3 * nt);
	TVG_CUDA(ctx, cudaMemcpyAsync(ad.data(), acc, 24 * (size_t) nt, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaMemcpyAsync(at.data(), ta, 24 * (size_t) nt, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	if (acc_direct) memcpy(acc_direct, ad.data(), 24 * (size_t) nt);
	if (acc_tree) memcpy(acc_tree, at.data(), 24 * (size_t) nt);
	if (err) {
		std::vector<double> e(nt);
		double sum2 = 0, sum = 0, mx = 0;
		for (int64_t t = 0; t < nt; t++) {
			double d2 = 0, a2 = 0;
			for (int k = 0; k < 3; k++) {
				const double d = at[k * nt + t] - ad[k * nt + t];
				d2 += d * d;
				a2 += ad[k * nt + t] * ad[k * nt + t];
			}
			e[t] = a2 > 0 ? sqrt(d2 / a2) : 0.0;
			sum2 += e[t] * e[t];
			sum += e[t];
			mx = std::max(mx, e[t]);
		}
		std::sort(e.begin(), e.end());
		const int64_t r99 = (int64_t) ceil(0.99 * (double) nt) - 1;
		err[0] = sqrt(sum2 / nt);
		err[1] = e[std::max<int64_t>(r99, 0)];
		err[2] = sum / nt;
		err[3] = mx;
	}
	return TVG_OK;
}

extern "C" int tvg_forcetest(tvg_context *ctx, uint32_t parts, int64_t n_targets,
                             const int64_t *targets, double *acc_direct, double *acc_tree,
                             double *err)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!(parts & TVG_WALK_GRAVITY))
		return tvg_fail(ctx, TVG_E_BADINPUT, "forcetest: parts must include TVG_WALK_GRAVITY");
	if ((parts & TVG_WALK_EWALD) && !ctx->cfg.periodic)
		return tvg_fail(ctx, TVG_E_STATE, "forcetest: Ewald part needs a periodic box");
	const bool ewald = (parts & TVG_WALK_EWALD) != 0;
	if (n_targets <= 0 || n_targets > TVG_FORCETEST_MAX_TARGETS || !targets)
		return tvg_fail(ctx, TVG_E_BADINPUT, "forcetest: n_targets must be in 1..%d",
		                TVG_FORCETEST_MAX_TARGETS);
	for (int64_t t = 0; t < n_targets; t++)
		if (targets[t] < 0 || targets[t] >= ctx->n)
			return tvg_fail(ctx, TVG_E_BADINPUT, "forcetest: target %lld out of range",
			                (long long) targets[t]);
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (ctx->cfg.float_bytes == 4)
		return forcetest_typed<float>(ctx, ewald, n_targets, targets, acc_direct, acc_tree, err);
	return forcetest_typed<double>(ctx, ewald, n_targets, targets, acc_direct, acc_tree, err);
}
