/*
 * GSL random-number-generator shim -- TEST INFRASTRUCTURE (oracle only).
 *
 * Provides gsl_rng_ranlxd1, the double-precision RANLUX generator that lpt.c
 * uses for the Gaussian initial field (lpt.c:172-233).  Implementation in
 * shim_gsl.c: Luscher's second-generation RANLUX (M. Luscher, Comput. Phys.
 * Commun. 79 (1994) 100) in its 48-bit form -- the base-2^24 subtract-with-
 * borrow generator with lags (10, 24), taken two words at a time, is the
 * base-2^48 subtract-with-borrow generator with lags (5, 12).  Luxury level 1
 * runs 202 such steps per block of 12 delivered numbers; seeding fills the
 * 12 words from a 31-bit shift-register sequence of the seed.
 * Bit-compatibility with GSL's own gsl_rng_ranlxd1 could not be checked in
 * this container (no GSL): this RNG is "parity unpinned".
 */
#ifndef ORACLE_SHIM_GSL_RNG_H
#define ORACLE_SHIM_GSL_RNG_H

typedef struct { const char* name; unsigned int luxury; } gsl_rng_type;
typedef struct {
  const gsl_rng_type* type;
  double x[12];
  double carry;
  int ir, jr, ir_old;
  unsigned int pr;
} gsl_rng;

extern const gsl_rng_type* gsl_rng_ranlxd1;
extern const gsl_rng_type* gsl_rng_ranlxd2;

gsl_rng* gsl_rng_alloc(const gsl_rng_type* T);
void gsl_rng_set(gsl_rng* r, unsigned long int seed);
double gsl_rng_uniform(gsl_rng* r);
void gsl_rng_free(gsl_rng* r);

#endif
