// tvg_ewald_mlp.cuh -- layout and forward pass of the learned Ewald
// correction (tvg_ewald_mlp.cu). On the folded octant x in [0, 1/2]^3 (box
// units), with v = 4 x - 1:
//     T(x) = 4 pi x / 3 + S(x) + C . m(v) + s N(v),
//     S(x) = -sum_{n in {0,1}^3, n != 0} (x - n) / |x - n|^3,
//     N(v) = W3 tanh(W2 tanh(W1 v + b1) + b2) + b3,
// where 4 pi x / 3 is the uniform background's linear term at the origin,
// S the seven lattice images nearest to the octant (they carry the steep part
// of T near the faces and corners), m(v) the 20 monomials of degree <= 3 with
// coefficients C fitted by least squares to what those two leave, and N the
// 3 -> 64 -> 64 -> 3 network trained on the rest divided by its rms s.
#pragma once

#include <cuda_bf16.h>

#define MLP_H 64
#define MLP_W1 0
#define MLP_B1 (MLP_W1 + 3 * MLP_H)
#define MLP_W2 (MLP_B1 + MLP_H)
#define MLP_B2 (MLP_W2 + MLP_H * MLP_H)
#define MLP_W3 (MLP_B2 + MLP_H)
#define MLP_B3 (MLP_W3 + 3 * MLP_H)
#define MLP_NNET (MLP_B3 + 3)               /* trained network parameters */
#define MLP_NMONO 20
#define MLP_POLY MLP_NNET                   /* C[3][20], fitted */
#define MLP_SCALE (MLP_POLY + 3 * MLP_NMONO) /* s */
#define MLP_NPARAM (MLP_SCALE + 1)
#define MLP_LIN 4.18879020478639098         /* 4 pi / 3 */

// the monomials of degree <= 3 of v, by degree then lexicographically:
// 1, v0, v1, v2, v0^2, v0v1, v0v2, v1^2, v1v2, v2^2, v0^3, v0^2v1, v0^2v2,
// v0v1^2, v0v1v2, v0v2^2, v1^3, v1^2v2, v1v2^2, v2^3
template <typename R>
__host__ __device__ __forceinline__ void mlp_monomials(const R v[3], R m[MLP_NMONO])
{
	const R a = v[0], b = v[1], c = v[2];
	m[0] = 1; m[1] = a; m[2] = b; m[3] = c;
	m[4] = a * a; m[5] = a * b; m[6] = a * c; m[7] = b * b; m[8] = b * c; m[9] = c * c;
	m[10] = m[4] * a; m[11] = m[4] * b; m[12] = m[4] * c; m[13] = a * m[7]; m[14] = m[5] * c;
	m[15] = a * m[9]; m[16] = m[7] * b; m[17] = m[7] * c; m[18] = b * m[9]; m[19] = m[9] * c;
}

// 4 pi x / 3 + S(x): the analytic part of the model, in FP64 (training
// targets)
__device__ __forceinline__ void mlp_analytic(const double x[3], double out[3])
{
	for (int d = 0; d < 3; d++) out[d] = MLP_LIN * x[d];
	for (int n = 1; n < 8; n++) {
		const double d0 = x[0] - (n & 1), d1 = x[1] - ((n >> 1) & 1), d2 = x[2] - ((n >> 2) & 1);
		const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
		const double i3 = 1.0 / (r2 * sqrt(r2));
		out[0] -= d0 * i3;
		out[1] -= d1 * i3;
		out[2] -= d2 * i3;
	}
}

// N(v), the network alone, from FP32 parameters P; FP32 arithmetic
__device__ __forceinline__ void mlp_net(const float *P, const float v[3], float o[3])
{
	float a1[MLP_H];
#pragma unroll
	for (int j = 0; j < MLP_H; j++)
		a1[j] = tanhf(P[MLP_B1 + j] + P[MLP_W1 + 3 * j] * v[0] + P[MLP_W1 + 3 * j + 1] * v[1]
		              + P[MLP_W1 + 3 * j + 2] * v[2]);
	float o0 = P[MLP_B3], o1 = P[MLP_B3 + 1], o2 = P[MLP_B3 + 2];
	for (int j = 0; j < MLP_H; j++) {
		float z = P[MLP_B2 + j];
#pragma unroll
		for (int i = 0; i < MLP_H; i++) z = fmaf(P[MLP_W2 + MLP_H * j + i], a1[i], z);
		const float a2 = tanhf(z);
		o0 = fmaf(P[MLP_W3 + j], a2, o0);
		o1 = fmaf(P[MLP_W3 + MLP_H + j], a2, o1);
		o2 = fmaf(P[MLP_W3 + 2 * MLP_H + j], a2, o2);
	}
	o[0] = o0;
	o[1] = o1;
	o[2] = o2;
}

// the walk's and the validation's copy of the parameters: network in BF16 (as
// inference uses it), the fitted polynomial and the scale in FP32
__device__ __forceinline__ float mlp_param(const __nv_bfloat16 *w, const float *f32, int e)
{
	return e < MLP_NNET ? __bfloat162float(w[e]) : f32[e];
}

// ------------------------------------------- warp evaluation (tensor cores)
//
// N(v) for the 32 points of a warp, one per lane; every lane of the warp
// calls (lanes without a point pass any v and ignore the result). Layer 1 and
// the tanh run per lane, producing the activations directly in the A-fragment
// layout of mma.sync.m16n8k16 (rows = points, columns = hidden units); layer
// 2 is 2 x 8 x 4 BF16 MMAs with FP32 accumulation (W2 as BF16 pairs in
// shared memory, row n of W2 = column n of B); layer 3 sums each lane's 16
// units and reduces over the 4 lanes of a row group. Activations are rounded
// to BF16 and tanh is the hardware approximation (tanh.approx.f32): the
// network's output is multiplied by s ~ 1e-3, so their error stays ~1e-5 of
// T. W2b: MLP_H * MLP_H / 2 words, W2b[(n * MLP_H + k) / 2] = (W2[n][k],
// W2[n][k + 1]) for even k.
__device__ __forceinline__ float mlp_tanh_approx(float x)
{
	float y;
	asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
	return y;
}

__device__ __forceinline__ uint32_t mlp_pack_bf16(float lo, float hi)
{
	const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
	return *reinterpret_cast<const uint32_t *>(&h);
}

__device__ __forceinline__ void mlp_net_warp(const float *P, const uint32_t *W2b, const float v[3],
                                             float o[3])
{
	const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
	// the four points whose rows this lane holds: g, g + 8, g + 16, g + 24
	float pv[4][3];
#pragma unroll
	for (int q = 0; q < 4; q++)
#pragma unroll
		for (int c = 0; c < 3; c++) pv[q][c] = __shfl_sync(0xFFFFFFFFu, v[c], g + 8 * q);
	// layer 1 into A fragments: a[mt][ks][r], mt = m tile (points 16 mt + ..),
	// ks = k step (units 16 ks + ..)
	uint32_t a[2][4][4];
#pragma unroll
	for (int ks = 0; ks < 4; ks++) {
#pragma unroll
		for (int half = 0; half < 2; half++) {
			const int u0 = 16 * ks + 2 * t + 8 * half, u1 = u0 + 1;
			const float w00 = P[MLP_W1 + 3 * u0], w01 = P[MLP_W1 + 3 * u0 + 1], w02 = P[MLP_W1 + 3 * u0 + 2];
			const float w10 = P[MLP_W1 + 3 * u1], w11 = P[MLP_W1 + 3 * u1 + 1], w12 = P[MLP_W1 + 3 * u1 + 2];
			const float b0 = P[MLP_B1 + u0], b1 = P[MLP_B1 + u1];
#pragma unroll
			for (int q = 0; q < 4; q++) {
				const float z0 = fmaf(w00, pv[q][0], fmaf(w01, pv[q][1], fmaf(w02, pv[q][2], b0)));
				const float z1 = fmaf(w10, pv[q][0], fmaf(w11, pv[q][1], fmaf(w12, pv[q][2], b1)));
				// q = 0, 1: tile 0 rows g, g + 8; q = 2, 3: tile 1
				a[q >> 1][ks][(q & 1) + 2 * half] = mlp_pack_bf16(mlp_tanh_approx(z0), mlp_tanh_approx(z1));
			}
		}
	}
	float out[4][3];
#pragma unroll
	for (int q = 0; q < 4; q++) out[q][0] = out[q][1] = out[q][2] = 0.f;
#pragma unroll
	for (int nt = 0; nt < 8; nt++) {
		const int n0 = 8 * nt + 2 * t;        // this lane's accumulator columns n0, n0 + 1
		float acc[2][4];
#pragma unroll
		for (int mt = 0; mt < 2; mt++) {
			acc[mt][0] = acc[mt][2] = P[MLP_B2 + n0];
			acc[mt][1] = acc[mt][3] = P[MLP_B2 + n0 + 1];
		}
#pragma unroll
		for (int ks = 0; ks < 4; ks++) {
			// B fragment: column n = 8 nt + g, rows k = 16 ks + 2 t (+1), + 8 (+9)
			const int n = 8 * nt + g, k0 = 16 * ks + 2 * t;
			const uint32_t b0 = W2b[(n * MLP_H + k0) >> 1], b1 = W2b[(n * MLP_H + k0 + 8) >> 1];
#pragma unroll
			for (int mt = 0; mt < 2; mt++)
				asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
				             "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
				             : "+f"(acc[mt][0]), "+f"(acc[mt][1]), "+f"(acc[mt][2]), "+f"(acc[mt][3])
				             : "r"(a[mt][ks][0]), "r"(a[mt][ks][1]), "r"(a[mt][ks][2]), "r"(a[mt][ks][3]),
				               "r"(b0), "r"(b1));
		}
		// acc[mt][0..1]: row g + 16 mt, columns n0, n0 + 1; acc[mt][2..3]: row g + 8 + 16 mt
		const float w3[3][2] = { { P[MLP_W3 + n0], P[MLP_W3 + n0 + 1] },
		                         { P[MLP_W3 + MLP_H + n0], P[MLP_W3 + MLP_H + n0 + 1] },
		                         { P[MLP_W3 + 2 * MLP_H + n0], P[MLP_W3 + 2 * MLP_H + n0 + 1] } };
#pragma unroll
		for (int mt = 0; mt < 2; mt++)
#pragma unroll
			for (int hr = 0; hr < 2; hr++) {
				const int q = 2 * mt + hr;
				const float h0 = mlp_tanh_approx(acc[mt][2 * hr]), h1 = mlp_tanh_approx(acc[mt][2 * hr + 1]);
#pragma unroll
				for (int c = 0; c < 3; c++) out[q][c] = fmaf(w3[c][0], h0, fmaf(w3[c][1], h1, out[q][c]));
			}
	}
	// sum over the 4 lanes of the row group, then lane L takes point L
#pragma unroll
	for (int q = 0; q < 4; q++)
#pragma unroll
		for (int c = 0; c < 3; c++) {
			out[q][c] += __shfl_xor_sync(0xFFFFFFFFu, out[q][c], 1);
			out[q][c] += __shfl_xor_sync(0xFFFFFFFFu, out[q][c], 2);
		}
	const int src = (lane & 7) << 2, slot = lane >> 3;
#pragma unroll
	for (int c = 0; c < 3; c++) {
		float r = 0.f;
#pragma unroll
		for (int q = 0; q < 4; q++) {
			const float x = __shfl_sync(0xFFFFFFFFu, out[q][c], src);
			r = slot == q ? x : r;
		}
		o[c] = r + P[MLP_B3 + c];
	}
}

// T at x for the warp's 32 points (every lane calls): mlp_net_warp plus the
// analytic part (4 pi x / 3 and the seven images, FP32) and the fitted cubic
__device__ __forceinline__ void mlp_forward_warp(const float *P, const uint32_t *W2b, const float x[3],
                                                 float out[3])
{
	const float v[3] = { 4.f * x[0] - 1.f, 4.f * x[1] - 1.f, 4.f * x[2] - 1.f };
	float o[3];
	mlp_net_warp(P, W2b, v, o);
	const float s = P[MLP_SCALE];
	float t[3] = { s * o[0], s * o[1], s * o[2] };
	float m[MLP_NMONO];
	mlp_monomials<float>(v, m);
#pragma unroll
	for (int k = 0; k < MLP_NMONO; k++) {
		t[0] = fmaf(P[MLP_POLY + k], m[k], t[0]);
		t[1] = fmaf(P[MLP_POLY + MLP_NMONO + k], m[k], t[1]);
		t[2] = fmaf(P[MLP_POLY + 2 * MLP_NMONO + k], m[k], t[2]);
	}
#pragma unroll
	for (int n = 1; n < 8; n++) {
		const float d0 = x[0] - (float) (n & 1), d1 = x[1] - (float) ((n >> 1) & 1),
		            d2 = x[2] - (float) ((n >> 2) & 1);
		const float ri = rsqrtf(fmaf(d0, d0, fmaf(d1, d1, d2 * d2)));
		const float i3 = ri * ri * ri;
		t[0] = fmaf(-d0, i3, t[0]);
		t[1] = fmaf(-d1, i3, t[1]);
		t[2] = fmaf(-d2, i3, t[2]);
	}
	out[0] = fmaf((float) MLP_LIN, x[0], t[0]);
	out[1] = fmaf((float) MLP_LIN, x[1], t[1]);
	out[2] = fmaf((float) MLP_LIN, x[2], t[2]);
}

// parameters for the warp evaluation into shared memory (block-wide): P in
// FP32 (network from BF16), W2b the BF16 pairs of W2
__device__ __forceinline__ void mlp_load_shared(const __nv_bfloat16 *w, const float *f32, float *P,
                                                uint32_t *W2b)
{
	for (int e = threadIdx.x; e < MLP_NPARAM; e += blockDim.x) P[e] = mlp_param(w, f32, e);
	const uint32_t *w2 = reinterpret_cast<const uint32_t *>(w + MLP_W2);
	for (int e = threadIdx.x; e < MLP_H * MLP_H / 2; e += blockDim.x) W2b[e] = w2[e];
}
