// tvg_ewald_mlp.cu -- the learned Ewald correction: a 3 -> 64 -> 64 -> 3
// network (tanh) on the symmetry-folded octant that stands in for the
// interpolation of the lattice-minus-image force T(x) (the quantity of the
// reference's Ewald table, Gravity/periodic.c:35-113, 352-461).
//
// Model: x in [0, 1/2]^3 (box units, the folded octant; the other octants
// follow from the symmetries T_a(.., -x_b, ..) = -T_a if a = b, +T_a
// otherwise), v = 4 x - 1, and
//     T(x) = 4 pi x / 3 + S(x) + C . m(v) + s N(v)
// (tvg_ewald_mlp.cuh): the linear background term, the seven nearest lattice
// images, a cubic least-squares fit, and the network N on what is left,
// scaled by that rest's rms s. Without S and the fit the same network reached
// 5.6e-3 rms in T; with them, 1.4e-4 (FP64 fits of 2^15 points, 6000 Adam
// steps). Parameters, 4672 floats:
//     W1[64][3] @0, b1[64] @192, W2[64][64] @256, b2[64] @4352,
//     W3[3][64] @4416, b3[3] @4608 (the network, 4611, trained);
//     C[3][20] @4611, s @4671 (fitted).
//
// Training (own kernels): 2^20 seeded points uniform on the octant, FP64
// targets T(x) by the Ewald sum of the table generator (tvg_ewald_sum.cuh)
// minus the analytic part; the normal equations of the cubic fit summed in
// FP64 (fixed-order block sums) and solved on the host (Cholesky); then the
// network's FP32 minibatch mean-square loss on the normalised rest: one
// thread per sample runs forward and backward, gradients are summed over the
// warp by shuffles into one slot per warp, then over the slots in fixed order
// (deterministic), then Adam.
//
// Inference: BF16 weights (rounded once after training), FP32 arithmetic and
// accumulation. The exact FP64 table (the reference's 65^3 nodes) validates
// it: tvg_ewald_mlp_validate measures the max and rms error there, and the
// walk refuses the learned correction when the max error is above the limit
// the caller gives.
#include <math.h>

#include <cmath>
#include <stdlib.h>

#include <vector>

#include "tvg_internal.cuh"
#include "tvg_ewald_sum.cuh"
#include "tvg_ewald_mlp.cuh"

// ------------------------------------------------------------ data

__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

__device__ __forceinline__ double u01(uint64_t r) { return (double) (r >> 11) * (1.0 / 9007199254740992.0); }

// points uniform on [0, 1/2]^3 (FP32-representable) and, in FP64, what the
// analytic part leaves of T there
__global__ void k_mlp_data(int64_t n, uint64_t seed, float *x, double *yraw)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	double p[3], f[3], a[3], pot;
	for (int d = 0; d < 3; d++)
		p[d] = (double) (float) (0.5 * u01(splitmix64(seed ^ (uint64_t) (3 * i + d) * 0x2545F4914F6CDD1Dull)));
	ewald_point(p, f, &pot);
	mlp_analytic(p, a);
	for (int d = 0; d < 3; d++) {
		x[3 * i + d] = (float) p[d];
		yraw[3 * i + d] = f[d] - a[d];
	}
}

// normal equations of the cubic fit: entry e < 210 is G_ij = sum m_i m_j
// (i <= j, row by row), e < 270 is b_ai = sum y_a m_i, e < 273 is sum y_a^2;
// block (e, c) sums the samples of chunk c in a fixed order
#define LSQ_NE 273
#define LSQ_CHUNKS 64
__global__ void __launch_bounds__(128)
k_mlp_lsq(int64_t n, const float *__restrict__ x, const double *__restrict__ yraw, double *part)
{
	const int e = blockIdx.x, c = blockIdx.y;
	int kind, i = 0, j = 0, a = 0;
	if (e < 210) {
		kind = 0;
		int r = e;
		while (r >= MLP_NMONO - i) { r -= MLP_NMONO - i; i++; }
		j = i + r;
	} else if (e < 270) {
		kind = 1;
		a = (e - 210) / MLP_NMONO;
		i = (e - 210) % MLP_NMONO;
	} else {
		kind = 2;
		a = e - 270;
	}
	const int64_t lo = n * c / LSQ_CHUNKS, hi = n * (c + 1) / LSQ_CHUNKS;
	double acc = 0;
	for (int64_t q = lo + threadIdx.x; q < hi; q += blockDim.x) {
		const double v[3] = { 4.0 * x[3 * q] - 1.0, 4.0 * x[3 * q + 1] - 1.0, 4.0 * x[3 * q + 2] - 1.0 };
		double m[MLP_NMONO];
		mlp_monomials<double>(v, m);
		if (kind == 0) acc += m[i] * m[j];
		else if (kind == 1) acc += yraw[3 * q + a] * m[i];
		else acc += yraw[3 * q + a] * yraw[3 * q + a];
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
	__shared__ double ws[4];
	if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
	__syncthreads();
	if (threadIdx.x == 0) part[(int64_t) e * LSQ_CHUNKS + c] = ((ws[0] + ws[1]) + ws[2]) + ws[3];
}

// network targets: (what the analytic part and the fit leave) / s, with the
// FP32 coefficients inference uses
__global__ void k_mlp_target(int64_t n, const float *__restrict__ x, const double *__restrict__ yraw,
                             const float *__restrict__ prm, float *y)
{
	const int64_t q = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (q >= n) return;
	const double v[3] = { 4.0 * x[3 * q] - 1.0, 4.0 * x[3 * q + 1] - 1.0, 4.0 * x[3 * q + 2] - 1.0 };
	double m[MLP_NMONO];
	mlp_monomials<double>(v, m);
	const double inv_s = 1.0 / (double) prm[MLP_SCALE];
	for (int a = 0; a < 3; a++) {
		double r = yraw[3 * q + a];
		for (int k = 0; k < MLP_NMONO; k++) r -= (double) prm[MLP_POLY + MLP_NMONO * a + k] * m[k];
		y[3 * q + a] = (float) (r * inv_s);
	}
}

// ------------------------------------------------------------ training

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
	for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
	return v;
}

// the warp's sum of v for parameter e lands in slot[e] (lane e % 32 writes)
__device__ __forceinline__ void put(float *slot, int e, float v)
{
	const float s = warp_sum(v);
	if ((threadIdx.x & 31) == (e & 31)) slot[e] = s;
}

// forward + backward of one sample per thread; per-warp gradient slots and
// per-warp loss sums. Samples past n contribute zero.
__global__ void __launch_bounds__(128)
k_mlp_grad(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
           const float *__restrict__ prm, float inv_norm, float *slots, float *loss_slots)
{
	__shared__ float P[MLP_NPARAM];
	for (int e = threadIdx.x; e < MLP_NPARAM; e += blockDim.x) P[e] = prm[e];
	__syncthreads();
	const float *W1 = P + MLP_W1, *B1 = P + MLP_B1, *W2 = P + MLP_W2, *B2 = P + MLP_B2,
	            *W3 = P + MLP_W3, *B3 = P + MLP_B3;
	const int64_t s = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	const bool have = s < n;
	const int64_t gw = s >> 5;
	float *slot = slots + gw * MLP_NNET;
	float v[3] = { 0.f, 0.f, 0.f }, t[3] = { 0.f, 0.f, 0.f };
	if (have) {
		for (int d = 0; d < 3; d++) {
			v[d] = 4.f * x[3 * s + d] - 1.f;
			t[d] = y[3 * s + d];
		}
	}
	float a1[MLP_H];
#pragma unroll
	for (int j = 0; j < MLP_H; j++)
		a1[j] = tanhf(B1[j] + W1[3 * j] * v[0] + W1[3 * j + 1] * v[1] + W1[3 * j + 2] * v[2]);
	float out[3] = { B3[0], B3[1], B3[2] };
	for (int j = 0; j < MLP_H; j++) {
		float z = B2[j];
#pragma unroll
		for (int i = 0; i < MLP_H; i++) z = fmaf(W2[MLP_H * j + i], a1[i], z);
		const float a2 = tanhf(z);
		out[0] = fmaf(W3[j], a2, out[0]);
		out[1] = fmaf(W3[MLP_H + j], a2, out[1]);
		out[2] = fmaf(W3[2 * MLP_H + j], a2, out[2]);
	}
	float dy[3], l = 0.f;
	for (int d = 0; d < 3; d++) {
		const float r = have ? out[d] - t[d] : 0.f;
		l += r * r;
		dy[d] = 2.f * r * inv_norm;
	}
	l = warp_sum(l);
	if ((threadIdx.x & 31) == 0) loss_slots[gw] = l;
	put(slot, MLP_B3 + 0, dy[0]);
	put(slot, MLP_B3 + 1, dy[1]);
	put(slot, MLP_B3 + 2, dy[2]);
	float dh1[MLP_H];
#pragma unroll
	for (int i = 0; i < MLP_H; i++) dh1[i] = 0.f;
	for (int j = 0; j < MLP_H; j++) {
		float z = B2[j];
#pragma unroll
		for (int i = 0; i < MLP_H; i++) z = fmaf(W2[MLP_H * j + i], a1[i], z);
		const float a2 = tanhf(z);
		const float dh2 = W3[j] * dy[0] + W3[MLP_H + j] * dy[1] + W3[2 * MLP_H + j] * dy[2];
		const float dz2 = dh2 * (1.f - a2 * a2);
		put(slot, MLP_W3 + j, dy[0] * a2);
		put(slot, MLP_W3 + MLP_H + j, dy[1] * a2);
		put(slot, MLP_W3 + 2 * MLP_H + j, dy[2] * a2);
		put(slot, MLP_B2 + j, dz2);
#pragma unroll
		for (int i = 0; i < MLP_H; i++) {
			put(slot, MLP_W2 + MLP_H * j + i, dz2 * a1[i]);
			dh1[i] = fmaf(W2[MLP_H * j + i], dz2, dh1[i]);
		}
	}
#pragma unroll
	for (int j = 0; j < MLP_H; j++) {
		const float dz1 = dh1[j] * (1.f - a1[j] * a1[j]);
		put(slot, MLP_B1 + j, dz1);
		put(slot, MLP_W1 + 3 * j, dz1 * v[0]);
		put(slot, MLP_W1 + 3 * j + 1, dz1 * v[1]);
		put(slot, MLP_W1 + 3 * j + 2, dz1 * v[2]);
	}
}

// sum of the warp slots in slot order (deterministic)
__global__ void k_mlp_sum(int nslots, const float *__restrict__ slots, const float *__restrict__ lslots,
                          float *grad, float *loss)
{
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e < MLP_NNET) {
		float g = 0.f;
		for (int w = 0; w < nslots; w++) g += slots[(int64_t) w * MLP_NNET + e];
		grad[e] = g;
	}
	if (e == MLP_NNET) {
		double l = 0;
		for (int w = 0; w < nslots; w++) l += lslots[w];
		*loss = (float) l;
	}
}

// Adam (Kingma & Ba 2015)
__global__ void k_mlp_adam(float *prm, const float *__restrict__ grad, float *m, float *v, float lr,
                           float c1, float c2)
{
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= MLP_NNET) return;
	const float g = grad[e];
	m[e] = 0.9f * m[e] + 0.1f * g;
	v[e] = 0.999f * v[e] + 0.001f * g * g;
	prm[e] -= lr * (m[e] * c1) / (sqrtf(v[e] * c2) + 1e-8f);
}

__global__ void k_mlp_to_bf16(const float *__restrict__ prm, __nv_bfloat16 *out)
{
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e < MLP_NPARAM) out[e] = __float2bfloat16_rn(prm[e]);
}

// forward only: per-warp sums of the network's squared residual (in units
// of s^2)
__global__ void __launch_bounds__(128)
k_mlp_loss(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
           const float *__restrict__ prm, float *loss_slots)
{
	__shared__ float P[MLP_NPARAM];
	for (int e = threadIdx.x; e < MLP_NPARAM; e += blockDim.x) P[e] = prm[e];
	__syncthreads();
	const int64_t s = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	float l = 0.f;
	if (s < n) {
		float v[3], out[3];
		for (int d = 0; d < 3; d++) v[d] = 4.f * x[3 * s + d] - 1.f;
		mlp_net(P, v, out);
		for (int d = 0; d < 3; d++) {
			const float r = out[d] - y[3 * s + d];
			l += r * r;
		}
	}
	l = warp_sum(l);
	if ((threadIdx.x & 31) == 0) loss_slots[s >> 5] = l;
}

// ------------------------------------------------------------ inference

// T(x) for points of the octant by the walk's evaluation (mlp_forward_warp:
// BF16 network on the tensor cores, FP32 elsewhere)
__global__ void __launch_bounds__(128)
k_mlp_eval(int64_t n, const double *__restrict__ x, const __nv_bfloat16 *__restrict__ w,
           const float *__restrict__ f32, double *t)
{
	__shared__ float P[MLP_NPARAM];
	__shared__ uint32_t W2b[MLP_H * MLP_H / 2];
	mlp_load_shared(w, f32, P, W2b);
	__syncthreads();
	const int64_t s = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	const bool have = s < n;          // every lane of a warp takes part
	float xs[3] = { 0.f, 0.f, 0.f }, out[3];
	if (have)
		for (int d = 0; d < 3; d++) xs[d] = (float) x[3 * s + d];
	mlp_forward_warp(P, W2b, xs, out);
	if (have)
		for (int d = 0; d < 3; d++) t[3 * s + d] = (double) out[d];
}

// ------------------------------------------------------------ host

// one gradient / loss slot per launched warp (blocks of 128 threads): the
// warps past n write zeros into their own slots
static inline int64_t mlp_slots(int64_t n) { return ((n + 127) / 128) * 4; }

static int dmalloc(tvg_context *ctx, void **p, size_t b)
{
	if (*p) return TVG_OK;
	TVG_CUDA(ctx, cudaMalloc(p, b));
	return TVG_OK;
}

static void init_params(std::vector<float> &p, uint64_t seed)
{
	// Glorot-uniform weights, zero biases, from a seeded host generator
	uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
	auto next = [&]() {
		st ^= st << 13; st ^= st >> 7; st ^= st << 17;
		return (double) (st >> 11) * (1.0 / 9007199254740992.0);
	};
	p.assign(MLP_NPARAM, 0.f);
	const double l1 = sqrt(6.0 / (3 + MLP_H)), l2 = sqrt(6.0 / (2 * MLP_H)), l3 = sqrt(6.0 / (MLP_H + 3));
	for (int e = 0; e < 3 * MLP_H; e++) p[MLP_W1 + e] = (float) ((2 * next() - 1) * l1);
	for (int e = 0; e < MLP_H * MLP_H; e++) p[MLP_W2 + e] = (float) ((2 * next() - 1) * l2);
	for (int e = 0; e < 3 * MLP_H; e++) p[MLP_W3 + e] = (float) ((2 * next() - 1) * l3);
}

// the cubic fit from the summed normal equations (k_mlp_lsq): Cholesky in
// FP64 for the three components; the coefficients are stored as FP32 and s is
// the rms of what they leave (evaluated with the FP32 coefficients)
static int fit_cubic(tvg_context *ctx, const std::vector<double> &part, int64_t ns,
                     std::vector<float> &p0)
{
	const int M = MLP_NMONO;
	double sum[LSQ_NE];
	for (int e = 0; e < LSQ_NE; e++) {
		double t = 0;
		for (int c = 0; c < LSQ_CHUNKS; c++) t += part[(size_t) e * LSQ_CHUNKS + c];
		sum[e] = t;
	}
	double G[M][M], L[M][M] = {};
	int e = 0;
	for (int i = 0; i < M; i++)
		for (int j = i; j < M; j++, e++) G[i][j] = G[j][i] = sum[e];
	for (int i = 0; i < M; i++) {
		for (int j = 0; j <= i; j++) {
			double t = G[i][j];
			for (int k = 0; k < j; k++) t -= L[i][k] * L[j][k];
			if (i == j) {
				if (!(t > 0)) return tvg_fail(ctx, TVG_E_CUDA, "mlp fit: normal equations not positive definite");
				L[i][i] = sqrt(t);
			} else {
				L[i][j] = t / L[j][j];
			}
		}
	}
	double r2 = 0;
	for (int a = 0; a < 3; a++) {
		double z[M], c[M];
		for (int i = 0; i < M; i++) {
			double t = sum[210 + M * a + i];
			for (int k = 0; k < i; k++) t -= L[i][k] * z[k];
			z[i] = t / L[i][i];
		}
		for (int i = M - 1; i >= 0; i--) {
			double t = z[i];
			for (int k = i + 1; k < M; k++) t -= L[k][i] * c[k];
			c[i] = t / L[i][i];
		}
		double cf[M], gc = 0, bc = 0;
		for (int i = 0; i < M; i++) {
			p0[MLP_POLY + M * a + i] = (float) c[i];
			cf[i] = (double) (float) c[i];
		}
		for (int i = 0; i < M; i++) {
			bc += cf[i] * sum[210 + M * a + i];
			for (int j = 0; j < M; j++) gc += cf[i] * G[i][j] * cf[j];
		}
		r2 += sum[270 + a] - 2 * bc + gc;
	}
	const double sc = sqrt(r2 / (3.0 * (double) ns));
	p0[MLP_SCALE] = (sc > 1e-30 && std::isfinite(sc)) ? (float) sc : 1.f;
	return TVG_OK;
}

static int ensure_mlp(tvg_context *ctx)
{
	TVG_CHECK(dmalloc(ctx, (void **) &ctx->mlp_prm, 4 * MLP_NPARAM));
	TVG_CHECK(dmalloc(ctx, (void **) &ctx->mlp_bf16, 2 * MLP_NPARAM));
	return TVG_OK;
}

static int refresh_bf16(tvg_context *ctx)
{
	k_mlp_to_bf16<<<TVG_CNT(ctx, (MLP_NPARAM + 255) / 256), 256, 0, ctx->stream>>>(ctx->mlp_prm, (__nv_bfloat16 *) ctx->mlp_bf16);
	TVG_CUDA(ctx, cudaGetLastError());
	ctx->have_mlp = true;
	ctx->mlp_ok = false;          // until validated
	return TVG_OK;
}

// one gradient of the mean-square loss over n samples (device arrays)
static int grad_batch(tvg_context *ctx, int64_t n, const float *x, const float *y, float *grad,
                      float *loss, float *slots, float *lslots)
{
	const int nslots = (int) mlp_slots(n);
	k_mlp_grad<<<TVG_CNT(ctx, tvg_blocks(n, 128)), 128, 0, ctx->stream>>>(
	    n, x, y, ctx->mlp_prm, 1.f / (3.f * (float) n), slots, lslots);
	TVG_CUDA(ctx, cudaGetLastError());
	k_mlp_sum<<<TVG_CNT(ctx, (MLP_NNET + 1 + 255) / 256), 256, 0, ctx->stream>>>(nslots, slots, lslots,
	                                                                             grad, loss);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

extern "C" int tvg_ewald_mlp_train(tvg_context *ctx, const tvg_mlp_train_config *cfg,
                                   float *final_loss)
{
	if (!ctx || !cfg) return TVG_E_BADINPUT;
	if (cfg->n_samples < 32 || cfg->batch < 32 || cfg->batch > cfg->n_samples || cfg->steps < 0)
		return tvg_fail(ctx, TVG_E_BADINPUT, "mlp train: need 32 <= batch <= n_samples, steps >= 0");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	TVG_CHECK(ensure_mlp(ctx));
	const int64_t ns = cfg->n_samples, nb = cfg->batch;
	float *x = nullptr, *y = nullptr, *slots = nullptr, *lslots = nullptr, *grad = nullptr,
	      *m = nullptr, *v = nullptr, *loss = nullptr, *yraw_f = nullptr, *part_f = nullptr;
	std::vector<void *> bufs;
	auto alloc = [&](float **p, size_t b) -> int {
		cudaError_t e = cudaMalloc((void **) p, b);
		if (e != cudaSuccess) {
			cudaGetLastError();
			return tvg_fail(ctx, TVG_E_NOMEM, "mlp train: cudaMalloc(%zu) failed", b);
		}
		bufs.push_back(*p);
		return TVG_OK;
	};
	int rc = TVG_OK;
	const int nslots = (int) mlp_slots(nb);
	if ((rc = alloc(&x, 12 * (size_t) ns)) || (rc = alloc(&y, 12 * (size_t) ns))
	    || (rc = alloc(&slots, 4 * (size_t) nslots * MLP_NPARAM)) || (rc = alloc(&lslots, 4 * (size_t) nslots))
	    || (rc = alloc(&grad, 4 * MLP_NPARAM)) || (rc = alloc(&m, 4 * MLP_NPARAM))
	    || (rc = alloc(&v, 4 * MLP_NPARAM)) || (rc = alloc(&loss, 4))
	    || (rc = alloc(&yraw_f, 24 * (size_t) ns)) || (rc = alloc(&part_f, 8 * LSQ_NE * LSQ_CHUNKS))) {
		for (void *b : bufs) cudaFree(b);
		return rc;
	}
	double *yraw = (double *) yraw_f, *part = (double *) part_f;
	auto done = [&](int r) {
		cudaStreamSynchronize(s);
		for (void *b : bufs) cudaFree(b);
		return r;
	};
	k_mlp_data<<<TVG_CNT(ctx, tvg_blocks(ns, 128)), 128, 0, s>>>(ns, cfg->seed, x, yraw);
	if (cudaGetLastError() != cudaSuccess) return done(tvg_fail(ctx, TVG_E_CUDA, "mlp data launch"));
	if (!cfg->resume) {
		// the cubic fit of what the analytic part leaves, then the network's
		// initial weights (a resumed training keeps both)
		std::vector<float> p0;
		init_params(p0, cfg->seed);
		k_mlp_lsq<<<TVG_CNT(ctx, dim3(LSQ_NE, LSQ_CHUNKS)), 128, 0, s>>>(ns, x, yraw, part);
		if (cudaGetLastError() != cudaSuccess) return done(tvg_fail(ctx, TVG_E_CUDA, "mlp lsq launch"));
		std::vector<double> hp((size_t) LSQ_NE * LSQ_CHUNKS);
		if (cudaMemcpyAsync(hp.data(), part, 8 * hp.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess
		    || cudaStreamSynchronize(s) != cudaSuccess)
			return done(tvg_fail(ctx, TVG_E_CUDA, "mlp lsq copy"));
		if ((rc = fit_cubic(ctx, hp, ns, p0))) return done(rc);
		if (cudaMemcpyAsync(ctx->mlp_prm, p0.data(), 4 * MLP_NPARAM, cudaMemcpyHostToDevice, s) != cudaSuccess)
			return done(tvg_fail(ctx, TVG_E_CUDA, "mlp train: upload failed"));
	}
	k_mlp_target<<<TVG_CNT(ctx, tvg_blocks(ns, 128)), 128, 0, s>>>(ns, x, yraw, ctx->mlp_prm, y);
	if (cudaGetLastError() != cudaSuccess) return done(tvg_fail(ctx, TVG_E_CUDA, "mlp target launch"));
	cudaMemsetAsync(m, 0, 4 * MLP_NPARAM, s);
	cudaMemsetAsync(v, 0, 4 * MLP_NPARAM, s);
	const int64_t nbatches = ns / nb;
	for (int st = 0; st < cfg->steps; st++) {
		// cosine decay from lr to lr_final
		const double f = cfg->steps > 1 ? (double) st / (cfg->steps - 1) : 0.0;
		const float lr = (float) (cfg->lr_final + 0.5 * (cfg->lr - cfg->lr_final) * (1.0 + cos(M_PI * f)));
		const int64_t off = (st % nbatches) * nb;
		rc = grad_batch(ctx, nb, x + 3 * off, y + 3 * off, grad, loss, slots, lslots);
		if (rc) return done(rc);
		const float c1 = (float) (1.0 / (1.0 - pow(0.9, st + 1))), c2 = (float) (1.0 / (1.0 - pow(0.999, st + 1)));
		k_mlp_adam<<<TVG_CNT(ctx, (MLP_NNET + 255) / 256), 256, 0, s>>>(ctx->mlp_prm, grad, m, v, lr, c1, c2);
		if (cudaGetLastError() != cudaSuccess) return done(tvg_fail(ctx, TVG_E_CUDA, "mlp adam launch"));
	}
	// mean-square residual of the trained FP32 weights over all samples
	float *lall = nullptr;
	if ((rc = alloc(&lall, 4 * (size_t) mlp_slots(ns)))) return done(rc);
	k_mlp_loss<<<TVG_CNT(ctx, tvg_blocks(ns, 128)), 128, 0, s>>>(ns, x, y, ctx->mlp_prm, lall);
	if (cudaGetLastError() != cudaSuccess) return done(tvg_fail(ctx, TVG_E_CUDA, "mlp loss launch"));
	std::vector<float> lw((size_t) mlp_slots(ns));
	float sc = 1.f;
	if (cudaMemcpyAsync(lw.data(), lall, 4 * lw.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess
	    || cudaMemcpyAsync(&sc, ctx->mlp_prm + MLP_SCALE, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
		return done(tvg_fail(ctx, TVG_E_CUDA, "mlp loss copy"));
	cudaStreamSynchronize(s);
	double tot = 0;
	for (float q : lw) tot += q;
	// in units of T^2
	if (final_loss) *final_loss = (float) (tot / (3.0 * (double) ns) * (double) sc * (double) sc);
	rc = refresh_bf16(ctx);
	return done(rc);
}

extern "C" int tvg_ewald_mlp_weights(tvg_context *ctx, float *params, int32_t set)
{
	if (!ctx || !params) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (set) {
		TVG_CHECK(ensure_mlp(ctx));
		TVG_CUDA(ctx, cudaMemcpy(ctx->mlp_prm, params, 4 * MLP_NPARAM, cudaMemcpyHostToDevice));
		TVG_CHECK(refresh_bf16(ctx));
		TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
		return TVG_OK;
	}
	if (!ctx->have_mlp) return tvg_fail(ctx, TVG_E_STATE, "mlp: no weights");
	TVG_CUDA(ctx, cudaMemcpy(params, ctx->mlp_prm, 4 * MLP_NPARAM, cudaMemcpyDeviceToHost));
	return TVG_OK;
}

extern "C" int tvg_ewald_mlp_grad(tvg_context *ctx, int64_t n, const float *x, const float *y,
                                  float *grad, float *loss)
{
	if (!ctx || !x || !y || !grad || n < 1) return TVG_E_BADINPUT;
	if (!ctx->have_mlp) return tvg_fail(ctx, TVG_E_STATE, "mlp: no weights");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	const int nslots = (int) mlp_slots(n);
	float *dx, *dy, *sl, *ll, *g, *l;
	TVG_CUDA(ctx, cudaMalloc((void **) &dx, 12 * (size_t) n));
	TVG_CUDA(ctx, cudaMalloc((void **) &dy, 12 * (size_t) n));
	TVG_CUDA(ctx, cudaMalloc((void **) &sl, 4 * (size_t) nslots * MLP_NPARAM));
	TVG_CUDA(ctx, cudaMalloc((void **) &ll, 4 * (size_t) nslots));
	TVG_CUDA(ctx, cudaMalloc((void **) &g, 4 * MLP_NPARAM + 4));
	l = g + MLP_NPARAM;
	cudaMemsetAsync(g, 0, 4 * MLP_NPARAM + 4, s);      // the fitted entries have no gradient
	cudaMemcpyAsync(dx, x, 12 * (size_t) n, cudaMemcpyHostToDevice, s);
	cudaMemcpyAsync(dy, y, 12 * (size_t) n, cudaMemcpyHostToDevice, s);
	int rc = grad_batch(ctx, n, dx, dy, g, l, sl, ll);
	if (rc == TVG_OK) {
		cudaMemcpyAsync(grad, g, 4 * MLP_NPARAM, cudaMemcpyDeviceToHost, s);
		if (loss) cudaMemcpyAsync(loss, l, 4, cudaMemcpyDeviceToHost, s);
		if (cudaStreamSynchronize(s) != cudaSuccess) rc = tvg_fail(ctx, TVG_E_CUDA, "mlp grad copy");
	}
	cudaFree(dx); cudaFree(dy); cudaFree(sl); cudaFree(ll); cudaFree(g);
	return rc;
}

extern "C" int tvg_ewald_mlp_eval(tvg_context *ctx, int64_t n, const double *x, double *t)
{
	if (!ctx || !x || !t || n < 1) return TVG_E_BADINPUT;
	if (!ctx->have_mlp) return tvg_fail(ctx, TVG_E_STATE, "mlp: no weights");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	double *dx, *dt;
	TVG_CUDA(ctx, cudaMalloc((void **) &dx, 24 * (size_t) n));
	TVG_CUDA(ctx, cudaMalloc((void **) &dt, 24 * (size_t) n));
	cudaMemcpyAsync(dx, x, 24 * (size_t) n, cudaMemcpyHostToDevice, ctx->stream);
	k_mlp_eval<<<TVG_CNT(ctx, tvg_blocks(n, 128)), 128, 0, ctx->stream>>>(n, dx, (const __nv_bfloat16 *) ctx->mlp_bf16,
	                                                                      ctx->mlp_prm, dt);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpyAsync(t, dt, 24 * (size_t) n, cudaMemcpyDeviceToHost, ctx->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
	cudaFree(dx);
	cudaFree(dt);
	if (e != cudaSuccess) return tvg_fail(ctx, TVG_E_CUDA, "mlp eval: %s", cudaGetErrorString(e));
	return TVG_OK;
}

// errors of the walk's evaluation of the model at the 65^3 nodes of the
// exact FP64 table
__global__ void __launch_bounds__(128)
k_mlp_validate(const double *__restrict__ raw, const __nv_bfloat16 *__restrict__ w,
            const float *__restrict__ f32, double *err)
{
	__shared__ float P[MLP_NPARAM];
	__shared__ uint32_t W2b[MLP_H * MLP_H / 2];
	mlp_load_shared(w, f32, P, W2b);
	__syncthreads();
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	const bool have = idx < 65 * 65 * 65;      // every lane of a warp takes part
	const int id = have ? idx : 0;
	const int i = id / (65 * 65), j = (id / 65) % 65, k = id % 65;
	const float xs[3] = { 0.5f * i / 64.f, 0.5f * j / 64.f, 0.5f * k / 64.f };
	float out[3];
	mlp_forward_warp(P, W2b, xs, out);
	if (!have) return;
	double e2 = 0;
	for (int d = 0; d < 3; d++) {
		const double r = (double) out[d] - raw[4 * idx + d];
		e2 += r * r;
	}
	err[idx] = sqrt(e2);
}

extern "C" int tvg_ewald_mlp_validate(tvg_context *ctx, double max_allowed, double *max_err,
                                   double *rms_err)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_mlp) return tvg_fail(ctx, TVG_E_STATE, "mlp: no weights");
	if (!ctx->have_ewald || !ctx->ewald_raw)
		return tvg_fail(ctx, TVG_E_STATE, "mlp validate: exact Ewald table not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	const int npt = 65 * 65 * 65;
	double *d;
	TVG_CUDA(ctx, cudaMalloc((void **) &d, 8 * (size_t) npt));
	k_mlp_validate<<<TVG_CNT(ctx, (npt + 127) / 128), 128, 0, ctx->stream>>>(ctx->ewald_raw, (const __nv_bfloat16 *) ctx->mlp_bf16,
	                                                                       ctx->mlp_prm, d);
	std::vector<double> h(npt);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, 8 * (size_t) npt, cudaMemcpyDeviceToHost, ctx->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
	cudaFree(d);
	if (e != cudaSuccess) return tvg_fail(ctx, TVG_E_CUDA, "mlp validate: %s", cudaGetErrorString(e));
	double mx = 0, s2 = 0;
	for (double q : h) { mx = q > mx ? q : mx; s2 += q * q; }
	if (max_err) *max_err = mx;
	if (rms_err) *rms_err = sqrt(s2 / npt);
	ctx->mlp_max_err = mx;
	ctx->mlp_ok = mx <= max_allowed;
	return TVG_OK;
}
