/*
 * Interface of the GSL cubic spline as the reference's comoving.c uses it:
 * natural cubic spline through (x_i, y_i), evaluated with an accelerator.
 * Implemented in gsl_min.c from the textbook tridiagonal formulation.
 */
#ifndef TV_ORACLE_GSL_SPLINE_H
#define TV_ORACLE_GSL_SPLINE_H
#include <stddef.h>
typedef struct gsl_spline gsl_spline;
typedef struct gsl_interp_accel gsl_interp_accel;
typedef struct gsl_interp_type { int kind; } gsl_interp_type;
extern const gsl_interp_type *gsl_interp_cspline;
gsl_spline *gsl_spline_alloc(const gsl_interp_type *t, size_t n);
int gsl_spline_init(gsl_spline *s, const double *x, const double *y, size_t n);
double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a);
void gsl_spline_free(gsl_spline *s);
gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
#endif
