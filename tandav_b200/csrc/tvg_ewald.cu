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
// judge of the learned correction.
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
