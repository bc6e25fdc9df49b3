/*
 * Interface of the GSL adaptive quadrature as the reference's comoving.c uses
 * it. gsl_min.c implements it as adaptive Gauss-Legendre bisection to the
 * requested relative tolerance (not GSL's own Gauss-Kronrod rule).
 */
#ifndef TV_ORACLE_GSL_INTEGRATION_H
#define TV_ORACLE_GSL_INTEGRATION_H
#include <stddef.h>
typedef struct { double (*function)(double x, void *params); void *params; } gsl_function;
typedef struct gsl_integration_workspace gsl_integration_workspace;
#define GSL_INTEG_GAUSS41 4
gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace *w);
int gsl_integration_qag(const gsl_function *f, double a, double b, double epsabs,
                        double epsrel, size_t limit, int key,
                        gsl_integration_workspace *w, double *result, double *abserr);
#endif
