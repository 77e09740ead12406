/* FFTW3f-MPI API shim (one process) -- TEST INFRASTRUCTURE; see fftw3.h. */
#ifndef ORACLE_SHIM_FFTW3_MPI_H
#define ORACLE_SHIM_FFTW3_MPI_H

#include "mpi.h"
#include "fftw3.h"

void fftwf_mpi_init(void);
void fftwf_mpi_cleanup(void);

ptrdiff_t fftwf_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                  MPI_Comm comm,
                                  ptrdiff_t* local_n0, ptrdiff_t* local_0_start);
ptrdiff_t fftwf_mpi_local_size_3d_transposed(
    ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm,
    ptrdiff_t* local_n0, ptrdiff_t* local_0_start,
    ptrdiff_t* local_n1, ptrdiff_t* local_1_start);

fftwf_plan fftwf_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     float* in, fftwf_complex* out,
                                     MPI_Comm comm, unsigned flags);
fftwf_plan fftwf_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     fftwf_complex* in, float* out,
                                     MPI_Comm comm, unsigned flags);
void fftwf_mpi_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_mpi_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);

#endif
