/*
 * Self-written replacements for the three GSL facilities the reference
 * calls: natural cubic splines (comoving.c kick/drift tables), adaptive
 * quadrature (the same tables) and an index heapsort (sort.c self-test).
 * Written from the mathematics; accurate to ~1e-12 relative on the smooth
 * integrands used, not bit-identical to GSL. Test infrastructure only.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "gsl/gsl_spline.h"
#include "gsl/gsl_integration.h"
#include "gsl/gsl_heapsort.h"

static const gsl_interp_type cspline_type = { 1 };
const gsl_interp_type *gsl_interp_cspline = &cspline_type;

struct gsl_spline { size_t n; double *x, *y, *m; };   /* m = second derivatives */
struct gsl_interp_accel { size_t last; };

gsl_spline *gsl_spline_alloc(const gsl_interp_type *t, size_t n)
{
	(void) t;
	gsl_spline *s = calloc(1, sizeof(*s));
	s->n = n;
	s->x = calloc(n, sizeof(double));
	s->y = calloc(n, sizeof(double));
	s->m = calloc(n, sizeof(double));
	return s;
}

/* Natural spline: m_0 = m_{n-1} = 0, tridiagonal system for the interior. */
int gsl_spline_init(gsl_spline *s, const double *x, const double *y, size_t n)
{
	memcpy(s->x, x, n * sizeof(double));
	memcpy(s->y, y, n * sizeof(double));
	double *c = calloc(n, sizeof(double)), *d = calloc(n, sizeof(double));
	s->m[0] = s->m[n - 1] = 0;
	for (size_t i = 1; i + 1 < n; i++) {
		double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
		double a = h0, b = 2 * (h0 + h1), cc = h1;
		double r = 6 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
		if (i > 1) { b -= a * c[i - 1]; r -= a * d[i - 1]; }
		c[i] = cc / b;
		d[i] = r / b;
	}
	for (size_t i = n - 2; i >= 1; i--) {
		s->m[i] = d[i] - c[i] * s->m[i + 1];
		if (i == 1) break;
	}
	free(c); free(d);
	return 0;
}

double gsl_spline_eval(const gsl_spline *s, double xv, gsl_interp_accel *a)
{
	size_t lo = 0, hi = s->n - 1;
	while (hi - lo > 1) {
		size_t mid = (lo + hi) / 2;
		if (s->x[mid] > xv) hi = mid; else lo = mid;
	}
	if (a) a->last = lo;
	double h = s->x[hi] - s->x[lo];
	double A = (s->x[hi] - xv) / h, B = (xv - s->x[lo]) / h;
	return A * s->y[lo] + B * s->y[hi]
	     + ((A * A * A - A) * s->m[lo] + (B * B * B - B) * s->m[hi]) * h * h / 6.0;
}

void gsl_spline_free(gsl_spline *s) { if (!s) return; free(s->x); free(s->y); free(s->m); free(s); }
gsl_interp_accel *gsl_interp_accel_alloc(void) { return calloc(1, sizeof(gsl_interp_accel)); }
void gsl_interp_accel_free(gsl_interp_accel *a) { free(a); }

struct gsl_integration_workspace { size_t limit; };
gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n)
{
	gsl_integration_workspace *w = calloc(1, sizeof(*w));
	w->limit = n;
	return w;
}
void gsl_integration_workspace_free(gsl_integration_workspace *w) { free(w); }

/* 10-point Gauss-Legendre nodes/weights by Newton iteration on P_10. */
#define GL_N 10
static double gl_x[GL_N], gl_w[GL_N];
static int gl_ready = 0;

static void gl_setup(void)
{
	for (int i = 0; i < GL_N; i++) {
		double z = cos(M_PI * (i + 0.75) / (GL_N + 0.5)), pp = 0;
		for (int it = 0; it < 100; it++) {
			double p0 = 1, p1 = 0;
			for (int k = 1; k <= GL_N; k++) {
				double p2 = p1; p1 = p0;
				p0 = ((2.0 * k - 1) * z * p1 - (k - 1.0) * p2) / k;
			}
			pp = GL_N * (z * p0 - p1) / (z * z - 1);
			double dz = p0 / pp;
			z -= dz;
			if (fabs(dz) < 1e-16) break;
		}
		gl_x[i] = z;
		gl_w[i] = 2 / ((1 - z * z) * pp * pp);
	}
	gl_ready = 1;
}

static double gl_rule(const gsl_function *f, double a, double b)
{
	double c = 0.5 * (a + b), h = 0.5 * (b - a), s = 0;
	for (int i = 0; i < GL_N; i++)
		s += gl_w[i] * f->function(c + h * gl_x[i], f->params);
	return s * h;
}

static double gl_adapt(const gsl_function *f, double a, double b, double whole,
                       double tol, int depth, double *err)
{
	double c = 0.5 * (a + b);
	double l = gl_rule(f, a, c), r = gl_rule(f, c, b);
	double diff = fabs(l + r - whole);
	if (diff <= tol || depth > 40) { *err += diff; return l + r; }
	return gl_adapt(f, a, c, l, 0.5 * tol, depth + 1, err)
	     + gl_adapt(f, c, b, r, 0.5 * tol, depth + 1, err);
}

int gsl_integration_qag(const gsl_function *f, double a, double b, double epsabs,
                        double epsrel, size_t limit, int key,
                        gsl_integration_workspace *w, double *result, double *abserr)
{
	(void) limit; (void) key; (void) w;
	if (!gl_ready) gl_setup();
	double whole = gl_rule(f, a, b);
	double tol = fmax(epsabs, 1e-3 * epsrel * fabs(whole));
	double err = 0;
	*result = gl_adapt(f, a, b, whole, tol, 0, &err);
	*abserr = err;
	return 0;
}

/* Index heapsort: perm[] orders data ascending under cmp. */
int gsl_heapsort_index(size_t *perm, const void *data, size_t n, size_t size,
                       int (*cmp)(const void *, const void *))
{
	const char *d = data;
	for (size_t i = 0; i < n; i++) perm[i] = i;
	if (n < 2) return 0;
#define KEY(i) (d + perm[i] * size)
	for (size_t start = n / 2; start-- > 0;) {
		size_t root = start;
		for (;;) {
			size_t child = 2 * root + 1;
			if (child >= n) break;
			if (child + 1 < n && cmp(KEY(child), KEY(child + 1)) < 0) child++;
			if (cmp(KEY(root), KEY(child)) >= 0) break;
			size_t t = perm[root]; perm[root] = perm[child]; perm[child] = t;
			root = child;
		}
	}
	for (size_t end = n - 1; end > 0; end--) {
		size_t t = perm[0]; perm[0] = perm[end]; perm[end] = t;
		size_t root = 0;
		for (;;) {
			size_t child = 2 * root + 1;
			if (child >= end) break;
			if (child + 1 < end && cmp(KEY(child), KEY(child + 1)) < 0) child++;
			if (cmp(KEY(root), KEY(child)) >= 0) break;
			size_t u = perm[root]; perm[root] = perm[child]; perm[child] = u;
			root = child;
		}
	}
#undef KEY
	return 0;
}
