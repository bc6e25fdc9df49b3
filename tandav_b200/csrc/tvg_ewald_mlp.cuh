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

// T at x (octant) from FP32 parameters P (shared memory); FP32 arithmetic
__device__ __forceinline__ void mlp_forward(const float *P, const float x[3], float out[3])
{
	const float v[3] = { 4.f * x[0] - 1.f, 4.f * x[1] - 1.f, 4.f * x[2] - 1.f };
	float o[3];
	mlp_net(P, v, o);
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

// the walk's and the judge's copy of the parameters: network in BF16 (as
// inference uses it), the fitted polynomial and the scale in FP32
__device__ __forceinline__ float mlp_param(const __nv_bfloat16 *w, const float *f32, int e)
{
	return e < MLP_NNET ? __bfloat162float(w[e]) : f32[e];
}
