/*
 * GSL integration shim -- TEST INFRASTRUCTURE (oracle only).
 *
 * gsl_integration_qag is provided as a globally adaptive bisection
 * quadrature on 20-point Gauss-Legendre panels (shim_gsl.c), driven to a
 * tolerance 1000x tighter than the caller asks, so it returns the converged
 * integral that GSL's QUADPACK Gauss-Kronrod rules also converge to for the
 * smooth integrands of cola.c:273 and power.c:191,216.  The Kronrod rule
 * selector `key` is accepted and ignored.
 */
#ifndef ORACLE_SHIM_GSL_INTEGRATION_H
#define ORACLE_SHIM_GSL_INTEGRATION_H
#include <stddef.h>

typedef struct { double (*function)(double x, void* params); void* params; } gsl_function;
typedef struct { size_t limit; } gsl_integration_workspace;

enum { GSL_INTEG_GAUSS15 = 1, GSL_INTEG_GAUSS21 = 2, GSL_INTEG_GAUSS31 = 3,
       GSL_INTEG_GAUSS41 = 4, GSL_INTEG_GAUSS51 = 5, GSL_INTEG_GAUSS61 = 6 };

gsl_integration_workspace* gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace* w);
int gsl_integration_qag(const gsl_function* f, double a, double b,
                        double epsabs, double epsrel, size_t limit, int key,
                        gsl_integration_workspace* workspace,
                        double* result, double* abserr);
#endif
