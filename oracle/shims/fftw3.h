/*
 * FFTW3 single-precision API shim -- TEST INFRASTRUCTURE (oracle only).
 *
 * Provides the subset of the FFTW3f / FFTW3f-MPI interface that the
 * reference's pm.c and lpt.c call, implemented on a project-written
 * mixed-radix (2/3/4/5) Stockham FFT that computes each 1-D transform in
 * double precision (shim_fftw.c).  Semantics follow the FFTW3 manual:
 *   - transforms are unnormalised;
 *   - r2c stores n2/2+1 complex values per row over a real row padded to
 *     2*(n2/2+1) floats (in-place layout, FFTW manual "Multi-dimensional
 *     DFTs of real data");
 *   - c2r of a multi-dimensional half spectrum is c2c over the leading
 *     dimensions followed by a 1-D c2r over the last one, which uses only the
 *     real parts of its k=0 and k=n2/2 inputs (the half-complex convention);
 *   - FFTW_MPI_TRANSPOSED_OUT / _IN exchange the first two dimensions of the
 *     complex array ([n1][n0][n2/2+1]), as FFTW-MPI does on one process.
 * This is not FFTW: timings taken with it are labelled "shim-FFT, not FFTW".
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#include <stddef.h>
#include <stdio.h>   /* the real fftw3.h includes it (FILE* wisdom API); comm.c relies on that */

typedef float fftwf_complex[2];
typedef struct oracle_fftw_plan_s* fftwf_plan;

#define FFTW_MEASURE  (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_IN  (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)

fftwf_complex* fftwf_alloc_complex(size_t n);
float* fftwf_alloc_real(size_t n);
void fftwf_free(void* p);
void fftwf_destroy_plan(fftwf_plan p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);

#endif
