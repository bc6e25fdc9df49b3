// tvg_ewald_mlp.cuh -- layout and forward pass of the learned Ewald
// correction (tvg_ewald_mlp.cu): T(x) = 4 pi x / 3 + W3 tanh(W2 tanh(W1 v + b1)
// + b2) + b3 with v = 4 x - 1, x on the folded octant [0, 1/2]^3 (box units).
#pragma once

#include <cuda_bf16.h>

#define MLP_H 64
#define MLP_W1 0
#define MLP_B1 (MLP_W1 + 3 * MLP_H)
#define MLP_W2 (MLP_B1 + MLP_H)
#define MLP_B2 (MLP_W2 + MLP_H * MLP_H)
#define MLP_W3 (MLP_B2 + MLP_H)
#define MLP_B3 (MLP_W3 + 3 * MLP_H)
#define MLP_NPARAM (MLP_B3 + 3)
#define MLP_LIN 4.18879020478639098f      /* 4 pi / 3 */

// T at x (octant) from FP32 parameters P (shared memory); FP32 arithmetic
__device__ __forceinline__ void mlp_forward(const float *P, const float x[3], float out[3])
{
	const float v0 = 4.f * x[0] - 1.f, v1 = 4.f * x[1] - 1.f, v2 = 4.f * x[2] - 1.f;
	float a1[MLP_H];
#pragma unroll
	for (int j = 0; j < MLP_H; j++)
		a1[j] = tanhf(P[MLP_B1 + j] + P[MLP_W1 + 3 * j] * v0 + P[MLP_W1 + 3 * j + 1] * v1
		              + P[MLP_W1 + 3 * j + 2] * v2);
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
	out[0] = MLP_LIN * x[0] + o0;
	out[1] = MLP_LIN * x[1] + o1;
	out[2] = MLP_LIN * x[2] + o2;
}
