// 2LPT initial displacements on the GPU (lpt.c:145-578).
#pragma once
#include "cosmo.h"

struct cg_lpt_out;

// Generate the nc^3 particles of one realization into a host array of
// reference Particle structs (56 B each, lattice order, ids 1..nc^3).
// dplus = D(a_init)/D(1) from power.c's GrowthFactor.  Returns 0 or a CG_E*
// code (message in cg_last_error()).
int lpt_generate(int nc, double boxsize, int seed, double omega_m, double a_init, double dplus,
                 const PowerTable& power, void* particles_host);

// Release the device buffers kept between lpt_generate calls.
void lpt_dropin_release();

// Host RANLUX (48-bit, luxury 202): the generator of lpt.c:172-233.
struct Ranlux48 {
  double x[12];
  double carry;
  int ir, jr, ir_old;
  int pr;
  void seed(unsigned long s);
  double uniform();
};
