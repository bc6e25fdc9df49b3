/*
 * tv_oracle.c -- CPU restatement of the Tandav gravity hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see tv_oracle.h). The CUDA product never links
 * this file; tests compare the CUDA path against it, and it is itself pinned
 * against the real reference built by oracle/Makefile.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "tv_oracle.h"

typedef __uint128_t u128;

/*
 * Peano-Hilbert keys, peano.c:122-276 (Skilling 2004, "Programming the
 * Hilbert curve", AIP Conf. Proc. 707, 381). The coordinates are first
 * scaled to 63-bit integers in double precision exactly as the reference
 * does ((p - origin) * 2^63 / size, truncated), then converted to the
 * Hilbert "transpose" form, then interleaved: level k (k = 0..42) is bit
 * 63-k of (X0, X1, X2). The standard key holds level k at bits
 * 130-3k..128-3k (levels 1..42), the reversed key holds level k at bits
 * 3k+2..3k (levels 0..41 complete, level 42 truncated).
 */
static void hilbert_transpose(uint64_t X[3])
{
	for (uint64_t q = 1ULL << 63; q > 1; q >>= 1) {
		const uint64_t mask = q - 1;
		for (int i = 0; i < 3; i++) {
			if (X[i] & q) {
				X[0] ^= mask;                      /* invert low bits of X0 */
			} else {
				uint64_t t = (X[0] ^ X[i]) & mask;   /* exchange low bits */
				X[0] ^= t;
				X[i] ^= t;
			}
		}
	}
	X[1] ^= X[0];                                    /* Gray encode */
	X[2] ^= X[1];
	uint64_t parity_above = 0;                       /* bit b: parity of X2 bits > b */
	for (uint64_t q = 1ULL << 63; q > 1; q >>= 1)
		if (X[2] & q) parity_above ^= q - 1;
	for (int i = 0; i < 3; i++) X[i] ^= parity_above;
}

static void ph_keys_from_coords(double px, double py, double pz, const double origin[3],
                                double size, u128 *std_key, u128 *rev_key)
{
	const double fac = (double) (1ULL << 63) / size;
	uint64_t X[3] = { (uint64_t) ((px - origin[0]) * fac), (uint64_t) ((py - origin[1]) * fac),
	                  (uint64_t) ((pz - origin[2]) * fac) };
	hilbert_transpose(X);
	u128 s = 0, r = 0;
	for (int k = 1; k <= 42; k++) {
		int b = 63 - k;
		u128 trip = (u128) ((((X[0] >> b) & 1) << 2) | (((X[1] >> b) & 1) << 1) | ((X[2] >> b) & 1));
		s |= trip << (128 - 3 * k);
		if (k <= 41) r |= trip << (3 * k);
		else r |= (trip & 3) << 126;               /* level 42: only 2 bits fit */
	}
	*std_key = s;
	*rev_key = r;
}

#define FLOAT float
#define SFX _f32
#include "tv_oracle_float.inc"
#undef FLOAT
#undef SFX
#define FLOAT double
#define SFX _f64
#include "tv_oracle_float.inc"
#undef FLOAT
#undef SFX

void tvo_peano_keys(int64_t n, int32_t fsize, const void *x, const void *y, const void *z,
                    const double origin[3], double size, uint64_t *std_key, uint64_t *rev_key)
{
	if (fsize == 4) keys_f32(n, x, y, z, origin, size, std_key, rev_key);
	else keys_f64(n, x, y, z, origin, size, std_key, rev_key);
}

static const uint64_t *Sort_Keys;

static int cmp_index_by_key(const void *a, const void *b)
{
	uint32_t i = *(const uint32_t *) a, j = *(const uint32_t *) b;
	uint64_t hi = Sort_Keys[2 * i], hj = Sort_Keys[2 * j];
	if (hi != hj) return hi < hj ? -1 : 1;
	uint64_t li = Sort_Keys[2 * i + 1], lj = Sort_Keys[2 * j + 1];
	if (li != lj) return li < lj ? -1 : 1;
	return i < j ? -1 : (i > j);                      /* ties: input order */
}

void tvo_sort_keys(int64_t n, const uint64_t *key, uint32_t *perm)
{
	for (int64_t i = 0; i < n; i++) perm[i] = (uint32_t) i;
	Sort_Keys = key;
	qsort(perm, (size_t) n, sizeof(uint32_t), cmp_index_by_key);
	Sort_Keys = NULL;
}

int32_t tvo_top_nodes(int64_t n, int32_t fsize, const uint64_t *std_key, const void *x,
                      const void *y, const void *z, const double origin[3], double size,
                      tvo_topnode *out)
{
	if (fsize == 4) return top_nodes_f32(n, std_key, x, y, z, origin, size, out);
	return top_nodes_f64(n, std_key, x, y, z, origin, size, out);
}

int64_t tvo_tree_build(int64_t n, int32_t fsize, const uint64_t *rev_key, const void *x,
                       const void *y, const void *z, const void *mass, double domain_size,
                       tvo_topnode *top, int32_t ntop, void *tree, int64_t tree_cap,
                       int32_t *tree_parent, int32_t vector_size)
{
	/* particles equal in all 42 levels would be dumped into a level-41 node
	 * (tree_build.c:337-342); the restatement follows that path too.
	 * vector_size: the reference's compile-time VECTOR_SIZE (64 by default) */
	if (fsize == 4)
		return tree_build_f32(n, rev_key, x, y, z, mass, domain_size, top, ntop, tree, tree_cap,
		                      tree_parent, vector_size);
	return tree_build_f64(n, rev_key, x, y, z, mass, domain_size, top, ntop, tree, tree_cap,
	                      tree_parent, vector_size);
}

void tvo_walk_gravity(int64_t n, int32_t fsize, const void *x, const void *y, const void *z,
                      const void *mass, const void *last_acc, const tvo_topnode *top,
                      int32_t ntop, const void *tree, const tvo_walk_params *prm, double *acc,
                      double *cost)
{
	tvo_walk_gravity_pot(n, fsize, x, y, z, mass, last_acc, top, ntop, tree, prm, acc, cost, NULL);
}

void tvo_walk_gravity_pot(int64_t n, int32_t fsize, const void *x, const void *y, const void *z,
                          const void *mass, const void *last_acc, const tvo_topnode *top,
                          int32_t ntop, const void *tree, const tvo_walk_params *prm, double *acc,
                          double *cost, double *pot)
{
	if (fsize == 4)
		walk_all_f32(n, x, y, z, mass, last_acc, top, ntop, tree, prm, NULL, NULL, NULL, NULL, 0,
		             acc, cost, pot);
	else
		walk_all_f64(n, x, y, z, mass, last_acc, top, ntop, tree, prm, NULL, NULL, NULL, NULL, 0,
		             acc, cost, pot);
}

void tvo_walk_ewald(int64_t n, int32_t fsize, const void *x, const void *y, const void *z,
                    const void *mass, const void *last_acc, const tvo_topnode *top, int32_t ntop,
                    const void *tree, const tvo_walk_params *prm, const void *fx, const void *fy,
                    const void *fz, double *acc, double *cost)
{
	tvo_walk_ewald_pot(n, fsize, x, y, z, mass, last_acc, top, ntop, tree, prm, fx, fy, fz, NULL, acc,
	                   cost, NULL);
}

void tvo_walk_ewald_pot(int64_t n, int32_t fsize, const void *x, const void *y, const void *z,
                        const void *mass, const void *last_acc, const tvo_topnode *top, int32_t ntop,
                        const void *tree, const tvo_walk_params *prm, const void *fx, const void *fy,
                        const void *fz, const void *fp, double *acc, double *cost, double *pot)
{
	if (fsize == 4)
		walk_all_f32(n, x, y, z, mass, last_acc, top, ntop, tree, prm, fx, fy, fz, fp, 1, acc, cost,
		             pot);
	else
		walk_all_f64(n, x, y, z, mass, last_acc, top, ntop, tree, prm, fx, fy, fz, fp, 1, acc, cost,
		             pot);
}

/*
 * Ewald correction force (Hernquist, Bouchet & Suto 1991, eqs. 2.14b/2.16;
 * Gravity/periodic.c:352-414) in box units: the force of the infinite
 * lattice minus the nearest image, alpha = 2.
 */
static void ewald_force_at(const double x[3], int nreal, int nk, double f[3])
{
	const double alpha = 2.0;
	f[0] = f[1] = f[2] = 0;
	double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
	if (r == 0) return;
	for (int k = 0; k < 3; k++) f[k] = x[k] / (r * r * r);
	for (int a = -nreal; a <= nreal; a++)
		for (int b = -nreal; b <= nreal; b++)
			for (int c = -nreal; c <= nreal; c++) {
				double d[3] = { x[0] - a, x[1] - b, x[2] - c };
				double rr = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
				double val = erfc(alpha * rr) + 2 * alpha * rr / sqrt(M_PI) * exp(-((alpha * rr) * (alpha * rr)));
				double r3 = rr * rr * rr;
				for (int k = 0; k < 3; k++) f[k] -= d[k] / r3 * val;
			}
	for (int a = -nk; a <= nk; a++)
		for (int b = -nk; b <= nk; b++)
			for (int c = -nk; c <= nk; c++) {
				int h2 = a * a + b * b + c * c;
				if (h2 == 0) continue;
				double hx = x[0] * a + x[1] * b + x[2] * c;
				double val = 2.0 / h2 * exp(-M_PI * M_PI * h2 / (alpha * alpha)) * sin(2 * M_PI * hx);
				f[0] -= a * val;
				f[1] -= b * val;
				f[2] -= c * val;
			}
}

static double ewald_potential_at(const double x[3], int nreal, int nk)
{
	const double alpha = 2.0;
	if (x[0] == 0 && x[1] == 0 && x[2] == 0) return 2.8372975;   /* periodic.c:419 */
	double s1 = 0, s2 = 0;
	for (int a = -nreal; a <= nreal; a++)
		for (int b = -nreal; b <= nreal; b++)
			for (int c = -nreal; c <= nreal; c++) {
				double d[3] = { x[0] - a, x[1] - b, x[2] - c };
				double rr = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
				s1 += erfc(alpha * rr) / rr;
			}
	for (int a = -nk; a <= nk; a++)
		for (int b = -nk; b <= nk; b++)
			for (int c = -nk; c <= nk; c++) {
				int h2 = a * a + b * b + c * c;
				if (h2 == 0) continue;
				double hx = x[0] * a + x[1] * b + x[2] * c;
				s2 += 1.0 / (M_PI * h2) * exp(-M_PI * M_PI * h2 / (alpha * alpha)) * cos(2 * M_PI * hx);
			}
	return M_PI / (alpha * alpha) - s1 - s2 + 1.0 / sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
}

void tvo_ewald_table(int32_t n_ewald, double *fx, double *fy, double *fz, double *fp)
{
	const int m = n_ewald + 1;
	#pragma omp parallel for schedule(dynamic) collapse(2)
	for (int i = 0; i < m; i++)
		for (int j = 0; j < m; j++)
			for (int k = 0; k < m; k++) {
				size_t idx = ((size_t) i * m + j) * m + k;
				double x[3] = { 0.5 * i / n_ewald, 0.5 * j / n_ewald, 0.5 * k / n_ewald };
				double f[3] = { 0, 0, 0 };
				if (i || j || k) ewald_force_at(x, 4, 4, f);
				fx[idx] = f[0];
				fy[idx] = f[1];
				fz[idx] = f[2];
				if (fp) fp[idx] = ewald_potential_at(x, 4, 4);
			}
}

void tvo_ewald_force(int64_t m, const double *x, int32_t nreal, int32_t nk, double *f)
{
	#pragma omp parallel for schedule(dynamic, 16)
	for (int64_t i = 0; i < m; i++) ewald_force_at(&x[3 * i], nreal, nk, &f[3 * i]);
}

/* Catmull-Rom style 4-point Lagrange weights for a uniform grid. */
static inline void lagrange4(double t, double w[4])
{
	w[0] = -t * (t - 1) * (t - 2) / 6;
	w[1] = (t + 1) * (t - 1) * (t - 2) / 2;
	w[2] = -(t + 1) * t * (t - 2) / 2;
	w[3] = (t + 1) * t * (t - 1) / 6;
}

/* Odd/even symmetry of the correction across each axis: component d is odd
 * in x_d and even in the other coordinates. Look up at |x| with sign fold. */
static void corr_lookup(const double *tab, int n, const double u_box[3], double f[3])
{
	double a[3];
	int sgn[3];
	for (int k = 0; k < 3; k++) { a[k] = fabs(u_box[k]); sgn[k] = u_box[k] < 0 ? -1 : 1; }
	const int m = n + 1;
	int base[3];
	double w[3][4];
	for (int k = 0; k < 3; k++) {
		double g = a[k] * 2 * n;             /* grid spacing 0.5 / n in box units */
		int i = (int) g;
		if (i > n - 2) i = n - 2;
		if (i < 1) i = 1;
		base[k] = i - 1;
		lagrange4(g - i, w[k]);
	}
	f[0] = f[1] = f[2] = 0;
	for (int p = 0; p < 4; p++)
		for (int q = 0; q < 4; q++)
			for (int r = 0; r < 4; r++) {
				int ii = base[0] + p, jj = base[1] + q, kk = base[2] + r;
				size_t idx = (((size_t) ii * m + jj) * m + kk) * 3;
				double wt = w[0][p] * w[1][q] * w[2][r];
				f[0] += wt * tab[idx];
				f[1] += wt * tab[idx + 1];
				f[2] += wt * tab[idx + 2];
			}
	for (int k = 0; k < 3; k++) f[k] *= sgn[k];
}

void tvo_direct(int64_t n, const double *pos, const double *mass, int64_t nt,
                const int64_t *targets, double gravity, double softening, double box,
                const double *corr_table, int32_t corr_n, double *acc)
{
	const double h = -41.0 / 32.0 * softening;     /* tree_build.c:136 */
	const double h2 = h * h, h3 = h * h * h;
	#pragma omp parallel for schedule(dynamic, 4)
	for (int64_t t = 0; t < nt; t++) {
		const int64_t i = targets[t];
		double a[3] = { 0, 0, 0 };
		const double xi[3] = { pos[i], pos[n + i], pos[2 * n + i] };
		for (int64_t j = 0; j < n; j++) {
			if (j == i) continue;
			double d[3] = { pos[j] - xi[0], pos[n + j] - xi[1], pos[2 * n + j] - xi[2] };
			if (box > 0)
				for (int k = 0; k < 3; k++) {
					if (d[k] > 0.5 * box) d[k] -= box;
					else if (d[k] < -0.5 * box) d[k] += box;
				}
			double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
			if (r2 == 0) continue;
			double fac;
			if (r2 < h2) {
				double u2 = r2 / h2;
				fac = gravity * mass[j] * (175 - u2 * (294 - u2 * 135)) / (16 * h3);
			} else {
				fac = gravity * mass[j] / (r2 * sqrt(r2));
			}
			for (int k = 0; k < 3; k++) a[k] += fac * d[k];
			if (box > 0 && corr_table) {
				double u[3] = { d[0] / box, d[1] / box, d[2] / box }, f[3];
				corr_lookup(corr_table, corr_n, u, f);
				/* Ewald_Correction sign convention: -sign(d) * table(|d|) */
				for (int k = 0; k < 3; k++) a[k] += -gravity * mass[j] * f[k] / (box * box);
			}
		}
		acc[t] = a[0];
		acc[nt + t] = a[1];
		acc[2 * nt + t] = a[2];
	}
}
