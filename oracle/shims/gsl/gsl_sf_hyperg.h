/*
 * GSL hypergeometric-function shim -- TEST INFRASTRUCTURE (oracle only).
 * gsl_sf_hyperg_2F1(a,b,c,x) for |x| < 1: Gauss series, with Pfaff's
 * transformation 2F1(a,b;c;x) = (1-x)^(-a) 2F1(a,c-b;c;x/(x-1)) for x < 0
 * (Abramowitz & Stegun 15.3.4), as used by cola.c:169-179.
 */
#ifndef ORACLE_SHIM_GSL_SF_HYPERG_H
#define ORACLE_SHIM_GSL_SF_HYPERG_H
double gsl_sf_hyperg_2F1(double a, double b, double c, double x);
#endif
