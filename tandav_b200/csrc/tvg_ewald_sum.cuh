// tvg_ewald_sum.cuh -- the lattice-minus-image force T(x) of a unit mass
// (box units, G = 1) by Ewald summation in FP64, shared by the table
// generators and the training data of the learned correction.
//
// compute_ewald_force / compute_ewald_potential (Gravity/periodic.c:352-461):
// the force of the periodic lattice minus the nearest image, after Hernquist,
// Bouchet & Suto (1991, eqs. 2.14-2.16), alpha = 2, real-space images and
// k-space vectors with |n|, |h| <= 4 per axis.
#pragma once

__device__ inline void ewald_point(const double x[3], double f[3], double *pot)
{
	const double alpha = 2.0, pi = 3.14159265358979323846;
	f[0] = f[1] = f[2] = 0;
	if (x[0] == 0 && x[1] == 0 && x[2] == 0) {
		*pot = 2.8372975;                     // periodic.c:419
		return;
	}
	const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
	const double r3 = r * r * r;
	for (int k = 0; k < 3; k++) f[k] = x[k] / r3;
	double s1 = 0, s2 = 0;
	for (int a = -4; a < 5; a++)
		for (int b = -4; b < 5; b++)
			for (int c = -4; c < 5; c++) {
				const double d0 = x[0] - a, d1 = x[1] - b, d2 = x[2] - c;
				const double rr = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
				const double ar = alpha * rr;
				const double val = erfc(ar) + 2 * alpha * rr / sqrt(pi) * exp(-(ar * ar));
				const double q = rr * rr * rr;
				f[0] -= d0 / q * val;
				f[1] -= d1 / q * val;
				f[2] -= d2 / q * val;
				s1 += erfc(ar) / rr;
			}
	for (int a = -4; a < 5; a++)
		for (int b = -4; b < 5; b++)
			for (int c = -4; c < 5; c++) {
				const int h2 = a * a + b * b + c * c;
				if (h2 == 0) continue;
				const double hx = x[0] * a + x[1] * b + x[2] * c;
				const double e = exp(-pi * pi * h2 / (alpha * alpha));
				const double val = 2.0 / h2 * e * sin(2 * pi * hx);
				f[0] -= a * val;
				f[1] -= b * val;
				f[2] -= c * val;
				s2 += 1.0 / (pi * h2) * e * cos(2 * pi * hx);
			}
	*pot = pi / (alpha * alpha) - s1 - s2 + 1.0 / r;
}

