// tvg_ewald.cu -- Ewald correction tables on the GPU (Gravity_Periodic_Init,
// Gravity/periodic.c:180-300).
//
// compute_ewald_force / compute_ewald_potential (Gravity/periodic.c:352-461):
// the force of the periodic lattice minus the nearest image, after Hernquist,
// Bouchet & Suto (1991, eqs. 2.14-2.16), alpha = 2, real-space images and
// k-space vectors with |n|, |h| <= 4 per axis, evaluated in FP64 at the
// (64+1)^3 points of the folded octant [0, L/2]^3 (box units), one thread per
// point and axis-sum. Stored as Float, then divided by Boxsize^2 (force) and
// Boxsize (potential) as the reference does after loading (periodic.c:215-228).
// The raw FP64 values stay on the device as the training target and max-error
// reference for validating the learned correction.
#include "tvg_internal.cuh"
#include "tvg_ewald_sum.cuh"

#define N_EWALD 64
#define N_EW1 (N_EWALD + 1)

template <typename F>
__global__ void k_ewald_table(double box, F *fx, F *fy, F *fz, F *fp, double *raw)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= N_EW1 * N_EW1 * N_EW1) return;
	const int i = idx / (N_EW1 * N_EW1), j = (idx / N_EW1) % N_EW1, k = idx % N_EW1;
	const double x[3] = { (0.5 * i) / N_EWALD, (0.5 * j) / N_EWALD, (0.5 * k) / N_EWALD };
	double f[3], pot;
	ewald_point(x, f, &pot);
	raw[4 * idx + 0] = f[0];
	raw[4 * idx + 1] = f[1];
	raw[4 * idx + 2] = f[2];
	raw[4 * idx + 3] = pot;
	// Float storage, then the division after the load (periodic.c:215-228)
	fx[idx] = (F) ((double) (F) f[0] / (box * box));
	fy[idx] = (F) ((double) (F) f[1] / (box * box));
	fz[idx] = (F) ((double) (F) f[2] / (box * box));
	fp[idx] = (F) ((double) (F) pot / box);
}

int tvg_impl_ewald_init(tvg_context *ctx)
{
	const size_t npt = (size_t) N_EW1 * N_EW1 * N_EW1;
	for (int t = 0; t < 4; t++)
		if (!ctx->ewald_f[t]) TVG_CUDA(ctx, cudaMalloc(&ctx->ewald_f[t], tvg_fsize(ctx) * npt));
	if (!ctx->ewald_raw) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->ewald_raw, 4 * 8 * npt));
	const unsigned nb = tvg_blocks((int64_t) npt, 128);
	if (ctx->cfg.float_bytes == 4)
		k_ewald_table<float><<<TVG_CNT(ctx, nb), 128, 0, ctx->stream>>>(
		    ctx->cfg.boxsize, (float *) ctx->ewald_f[0], (float *) ctx->ewald_f[1],
		    (float *) ctx->ewald_f[2], (float *) ctx->ewald_f[3], ctx->ewald_raw);
	else
		k_ewald_table<double><<<TVG_CNT(ctx, nb), 128, 0, ctx->stream>>>(
		    ctx->cfg.boxsize, (double *) ctx->ewald_f[0], (double *) ctx->ewald_f[1],
		    (double *) ctx->ewald_f[2], (double *) ctx->ewald_f[3], ctx->ewald_raw);
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	return TVG_OK;
}

// The group form's correction table: T(x) (box units, unit G m: the force of
// the periodic lattice minus the image at the origin, the quantity of the
// table above) at x = 0.5 i / 64 for i = -1..66 per axis, in FP64 then stored
// FP32 as (Tx, Ty, Tz, 0). The layer at i = -1 and the layers beyond L/2 let
// a 4-point stencil stay centred everywhere on the octant; beyond L/2 the
// values are the analytic continuation of that correction, which a Taylor
// expansion about a point near the half-box plane needs.
#define N_EXT 68

__global__ void k_ewald_ext(float4 *ext)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= N_EXT * N_EXT * N_EXT) return;
	const int i = idx / (N_EXT * N_EXT) - 1, j = (idx / N_EXT) % N_EXT - 1, k = idx % N_EXT - 1;
	const double x[3] = { (0.5 * i) / N_EWALD, (0.5 * j) / N_EWALD, (0.5 * k) / N_EWALD };
	double f[3], pot;
	ewald_point(x, f, &pot);
	ext[idx] = make_float4((float) f[0], (float) f[1], (float) f[2], 0.f);
}

int tvg_impl_ewald_ext(tvg_context *ctx)
{
	const size_t npt = (size_t) N_EXT * N_EXT * N_EXT;
	if (!ctx->ewald_ext) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->ewald_ext, 16 * npt));
	k_ewald_ext<<<TVG_CNT(ctx, tvg_blocks((int64_t) npt, 128)), 128, 0, ctx->stream>>>(
	    (float4 *) ctx->ewald_ext);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

// Taylor table of the group form: at each node x = i / (2 (N - 1)) (box
// units, i = 0..N-1 per axis, N = TVG_TAYLOR_NODES) of the octant, T and its
// first three derivatives, the k-th derivative taken with respect to the node
// coordinate u = 2 (N - 1) x (so scaled by the node spacing^k). Record of 64
// floats, 20 per component a (then 4 pad):
//   [20a] T_a; [20a + 1 + b] dT_a/du_b; [20a + 4 + s] d2T_a, s over
//   xx yy zz xy xz yz; [20a + 10 + t] d3T_a, t over xxx yyy zzz xxy xxz yyx
//   yyz zzx zzy xyz.
// A lookup expands T about the nearest node (|du| <= 1/2 per axis): T to
// third order, dT to second, d2T to first. With 33 nodes (spacing 1/64, a
// 9.2 MB table that stays in L2) the value is within 4e-7 of |T| and the
// gradient within 3e-5 of its largest component, against direct lattice sums
// at off-node points across the octant (the origin, face, edge and corner
// nodes included); with 65 nodes, 6e-8 and 7e-6. The derivatives are
// finite differences of FP64 lattice sums on a grid of half the node spacing
// (two ghost points beyond each end): fourth-order central differences for the
// first and pure second derivatives, second-order ones for the mixed and third
// derivatives (small correction terms); FP64 round-off enters as
// ~1e-16 / delta^3, below 1e-8.
#define N_TAY TVG_TAYLOR_NODES
#define N_FINE (2 * (N_TAY - 1) + 1 + 4)

__global__ void k_ewald_fine(double *fine)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= N_FINE * N_FINE * N_FINE) return;
	const int i = idx / (N_FINE * N_FINE), j = (idx / N_FINE) % N_FINE, k = idx % N_FINE;
	const double d = 1.0 / (4.0 * (N_TAY - 1));
	const double x[3] = { (i - 2) * d, (j - 2) * d, (k - 2) * d };
	double f[3], pot;
	ewald_point(x, f, &pot);
	fine[3 * (int64_t) idx + 0] = f[0];
	fine[3 * (int64_t) idx + 1] = f[1];
	fine[3 * (int64_t) idx + 2] = f[2];
}

__global__ void k_ewald_taylor(const double *__restrict__ fine, float *tay)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= N_TAY * N_TAY * N_TAY) return;
	const int ni = idx / (N_TAY * N_TAY), nj = (idx / N_TAY) % N_TAY, nk = idx % N_TAY;
	const int ci = 2 * ni + 2, cj = 2 * nj + 2, ck = 2 * nk + 2;
	// fine spacing in node units: 1/2
	const double h = 0.5, h2 = h * h, h3 = h2 * h;
	float *r = tay + 64 * (int64_t) idx;
	for (int a = 0; a < 3; a++) {
		float *ra = r + 20 * a;
		// component a at fine offsets from the node
		auto f = [&](int di, int dj, int dk) {
			return fine[3 * (((int64_t) (ci + di) * N_FINE + (cj + dj)) * N_FINE + (ck + dk)) + a];
		};
		auto g = [&](int b, int s) { return b == 0 ? f(s, 0, 0) : b == 1 ? f(0, s, 0) : f(0, 0, s); };
		auto g2 = [&](int b, int sb, int e, int se) {
			int d[3] = { 0, 0, 0 };
			d[b] += sb;
			d[e] += se;
			return f(d[0], d[1], d[2]);
		};
		const double c = f(0, 0, 0);
		ra[0] = (float) c;
		for (int b = 0; b < 3; b++)
			ra[1 + b] = (float) ((-g(b, 2) + 8 * g(b, 1) - 8 * g(b, -1) + g(b, -2)) / (12 * h));
		for (int b = 0; b < 3; b++)
			ra[4 + b] = (float) ((-g(b, 2) + 16 * g(b, 1) - 30 * c + 16 * g(b, -1) - g(b, -2)) / (12 * h2));
		const int pr[3][2] = { { 0, 1 }, { 0, 2 }, { 1, 2 } };
		for (int q = 0; q < 3; q++) {
			const int b = pr[q][0], e = pr[q][1];
			ra[7 + q] = (float) ((g2(b, 1, e, 1) - g2(b, 1, e, -1) - g2(b, -1, e, 1) + g2(b, -1, e, -1))
			                     / (4 * h2));
		}
		for (int b = 0; b < 3; b++)
			ra[10 + b] = (float) ((g(b, 2) - 2 * g(b, 1) + 2 * g(b, -1) - g(b, -2)) / (2 * h3));
		// d3 T / db db de: the difference along e of the second differences along b
		const int bbe[6][2] = { { 0, 1 }, { 0, 2 }, { 1, 0 }, { 1, 2 }, { 2, 0 }, { 2, 1 } };
		for (int q = 0; q < 6; q++) {
			const int b = bbe[q][0], e = bbe[q][1];
			const double up = g2(b, 1, e, 1) - 2 * g2(b, 0, e, 1) + g2(b, -1, e, 1);
			const double dn = g2(b, 1, e, -1) - 2 * g2(b, 0, e, -1) + g2(b, -1, e, -1);
			ra[13 + q] = (float) ((up - dn) / (2 * h3));
		}
		double s3 = 0;
		for (int sx = -1; sx <= 1; sx += 2)
			for (int sy = -1; sy <= 1; sy += 2)
				for (int sz = -1; sz <= 1; sz += 2) s3 += sx * sy * sz * f(sx, sy, sz);
		ra[19] = (float) (s3 / (8 * h3));
	}
	for (int q = 60; q < 64; q++) r[q] = 0.f;
}

int tvg_impl_ewald_taylor(tvg_context *ctx)
{
	const size_t ntay = (size_t) N_TAY * N_TAY * N_TAY, nfine = (size_t) N_FINE * N_FINE * N_FINE;
	if (!ctx->ewald_taylor) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->ewald_taylor, 256 * ntay));
	double *fine = nullptr;
	TVG_CUDA(ctx, cudaMalloc((void **) &fine, 24 * nfine));
	k_ewald_fine<<<TVG_CNT(ctx, tvg_blocks((int64_t) nfine, 128)), 128, 0, ctx->stream>>>(fine);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) {
		k_ewald_taylor<<<TVG_CNT(ctx, tvg_blocks((int64_t) ntay, 128)), 128, 0, ctx->stream>>>(
		    fine, ctx->ewald_taylor);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
	cudaFree(fine);
	if (e != cudaSuccess) return tvg_fail(ctx, TVG_E_CUDA, "ewald taylor table: %s", cudaGetErrorString(e));
	return TVG_OK;
}

// raw Float tables (box units) -> device tables, as after
// read_ewald_correction_table + the division at periodic.c:215-228
template <typename F>
__global__ void k_ewald_from_raw(double box, const F *rx, const F *ry, const F *rz, const F *rp,
                                 F *fx, F *fy, F *fz, F *fp, double *raw)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= N_EW1 * N_EW1 * N_EW1) return;
	raw[4 * idx + 0] = (double) rx[idx];
	raw[4 * idx + 1] = (double) ry[idx];
	raw[4 * idx + 2] = (double) rz[idx];
	raw[4 * idx + 3] = (double) rp[idx];
	fx[idx] = (F) ((double) rx[idx] / (box * box));
	fy[idx] = (F) ((double) ry[idx] / (box * box));
	fz[idx] = (F) ((double) rz[idx] / (box * box));
	fp[idx] = (F) ((double) rp[idx] / box);
}

extern "C" int tvg_upload_ewald_table(tvg_context *ctx, const void *fx, const void *fy,
                                      const void *fz, const void *fp)
{
	if (!ctx || !fx || !fy || !fz || !fp) return TVG_E_BADINPUT;
	if (!ctx->cfg.periodic) return tvg_fail(ctx, TVG_E_STATE, "upload_ewald_table: not periodic");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	const size_t npt = (size_t) N_EW1 * N_EW1 * N_EW1, b = tvg_fsize(ctx) * npt;
	for (int t = 0; t < 4; t++)
		if (!ctx->ewald_f[t]) TVG_CUDA(ctx, cudaMalloc(&ctx->ewald_f[t], b));
	if (!ctx->ewald_raw) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->ewald_raw, 4 * 8 * npt));
	void *tmp = nullptr;
	TVG_CUDA(ctx, cudaMalloc(&tmp, 4 * b));
	const void *src[4] = { fx, fy, fz, fp };
	for (int t = 0; t < 4; t++)
		TVG_CUDA(ctx, cudaMemcpyAsync((char *) tmp + t * b, src[t], b, cudaMemcpyHostToDevice, ctx->stream));
	const unsigned nb = tvg_blocks((int64_t) npt, 256);
	if (ctx->cfg.float_bytes == 4) {
		const float *r = (const float *) tmp;
		k_ewald_from_raw<float><<<TVG_CNT(ctx, nb), 256, 0, ctx->stream>>>(
		    ctx->cfg.boxsize, r, r + npt, r + 2 * npt, r + 3 * npt, (float *) ctx->ewald_f[0],
		    (float *) ctx->ewald_f[1], (float *) ctx->ewald_f[2], (float *) ctx->ewald_f[3], ctx->ewald_raw);
	} else {
		const double *r = (const double *) tmp;
		k_ewald_from_raw<double><<<TVG_CNT(ctx, nb), 256, 0, ctx->stream>>>(
		    ctx->cfg.boxsize, r, r + npt, r + 2 * npt, r + 3 * npt, (double *) ctx->ewald_f[0],
		    (double *) ctx->ewald_f[1], (double *) ctx->ewald_f[2], (double *) ctx->ewald_f[3],
		    ctx->ewald_raw);
	}
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
	cudaFree(tmp);
	TVG_CUDA(ctx, e);
	ctx->have_ewald = true;
	return TVG_OK;
}

template <typename F>
__global__ void k_ewald_raw_float(const double *raw, F *out, int comp, int n)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (F) raw[4 * i + comp];
}

extern "C" int tvg_download_ewald_table(tvg_context *ctx, void *fx, void *fy, void *fz, void *fp)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_ewald) return tvg_fail(ctx, TVG_E_STATE, "ewald table not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	const int npt = N_EW1 * N_EW1 * N_EW1;
	void *outs[4] = { fx, fy, fz, fp };
	void *tmp = nullptr;
	TVG_CUDA(ctx, cudaMalloc(&tmp, tvg_fsize(ctx) * npt));
	for (int c = 0; c < 4; c++) {
		if (!outs[c]) continue;
		if (ctx->cfg.float_bytes == 4)
			k_ewald_raw_float<float><<<TVG_CNT(ctx, tvg_blocks(npt, 256)), 256, 0, ctx->stream>>>(ctx->ewald_raw,
			                                                                          (float *) tmp, c, npt);
		else
			k_ewald_raw_float<double><<<TVG_CNT(ctx, tvg_blocks(npt, 256)), 256, 0, ctx->stream>>>(ctx->ewald_raw,
			                                                                           (double *) tmp, c, npt);
		cudaError_t e = cudaMemcpyAsync(outs[c], tmp, tvg_fsize(ctx) * npt, cudaMemcpyDeviceToHost,
		                                ctx->stream);
		if (e != cudaSuccess) { cudaFree(tmp); TVG_CUDA(ctx, e); }
	}
	cudaError_t e = cudaStreamSynchronize(ctx->stream);
	cudaFree(tmp);
	TVG_CUDA(ctx, e);
	return TVG_OK;
}
