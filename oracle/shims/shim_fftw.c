/*
 * FFTW3f(-MPI) shim implementation -- TEST INFRASTRUCTURE (see fftw3.h).
 *
 * 1-D transforms: self-sorting (Stockham) mixed-radix FFT, radices 4, 2, 3, 5
 * and a generic odd radix, computed in double precision with a twiddle table
 * e^{-2 pi i k/n} built in double (Cooley & Tukey 1965; Stockham 1966; the
 * autosort form follows Van Loan, "Computational Frameworks for the FFT",
 * 1992, ch. 1.7).  3-D real transforms are separable: z (the contiguous,
 * last dimension) is done as a real transform, y and x as complex ones.  The
 * intermediate 3-D array is single precision, as in FFTW single precision.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "fftw3-mpi.h"

#define SHIM_PI 3.14159265358979323846264338327950288

/* ---------------------------------------------------------------- 1-D FFT */

typedef struct {
  int n;
  int nf;
  int fac[40];
  double* tw;   /* tw[2k], tw[2k+1] = cos, sin of -2 pi k / n */
} fft1d;

static fft1d* fft1d_make(int n)
{
  fft1d* p = (fft1d*)calloc(1, sizeof(fft1d));
  p->n = n;
  int m = n;
  while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
  while (m % 3 == 0) { p->fac[p->nf++] = 3; m /= 3; }
  while (m % 5 == 0) { p->fac[p->nf++] = 5; m /= 5; }
  for (int f = 7; m > 1; f += 2)
    while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
  p->tw = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  for (int k = 0; k < n; k++) {
    double a = -2.0 * SHIM_PI * (double)k / (double)n;
    p->tw[2 * k] = cos(a);
    p->tw[2 * k + 1] = sin(a);
  }
  return p;
}

static void fft1d_free(fft1d* p)
{
  if (p) { free(p->tw); free(p); }
}

/* In-place transform of x (n interleaved complex doubles) using work (same
 * size).  sign = -1 forward (e^{-i..}), +1 backward; unnormalised. */
static void fft1d_exec(const fft1d* p, double* x, double* work, int sign)
{
  const int n = p->n;
  if (n == 1) return;
  double* src = x;
  double* dst = work;
  int ns = 1;
  for (int s = 0; s < p->nf; s++) {
    const int r = p->fac[s];
    const int m = n / r;           /* input stride between butterfly legs */
    const int twstep = n / (ns * r);
    for (int j = 0; j < m; j++) {
      const int jm = j % ns;
      double vr[64], vi[64];
      for (int k = 0; k < r; k++) {
        double ar = src[2 * (j + k * m)], ai = src[2 * (j + k * m) + 1];
        if (k && jm) {
          int t = (jm * k * twstep) % n;
          double wr = p->tw[2 * t], wi = -sign * p->tw[2 * t + 1];
          double br = ar * wr - ai * wi;
          double bi = ar * wi + ai * wr;
          ar = br; ai = bi;
        }
        vr[k] = ar; vi[k] = ai;
      }
      double or_[64], oi[64];
      if (r == 2) {
        or_[0] = vr[0] + vr[1]; oi[0] = vi[0] + vi[1];
        or_[1] = vr[0] - vr[1]; oi[1] = vi[0] - vi[1];
      } else if (r == 4) {
        double s0r = vr[0] + vr[2], s0i = vi[0] + vi[2];
        double d0r = vr[0] - vr[2], d0i = vi[0] - vi[2];
        double s1r = vr[1] + vr[3], s1i = vi[1] + vi[3];
        double d1r = vr[1] - vr[3], d1i = vi[1] - vi[3];
        /* multiply d1 by (sign * i) */
        double jd1r = -sign * d1i, jd1i = sign * d1r;
        or_[0] = s0r + s1r; oi[0] = s0i + s1i;
        or_[2] = s0r - s1r; oi[2] = s0i - s1i;
        or_[1] = d0r + jd1r; oi[1] = d0i + jd1i;
        or_[3] = d0r - jd1r; oi[3] = d0i - jd1i;
      } else {
        const int rs = n / r;
        for (int q = 0; q < r; q++) {
          double sr = 0.0, si = 0.0;
          for (int k = 0; k < r; k++) {
            int t = ((q * k) % r) * rs;
            double wr = p->tw[2 * t], wi = -sign * p->tw[2 * t + 1];
            sr += vr[k] * wr - vi[k] * wi;
            si += vr[k] * wi + vi[k] * wr;
          }
          or_[q] = sr; oi[q] = si;
        }
      }
      const int base = (j / ns) * ns * r + jm;
      for (int q = 0; q < r; q++) {
        dst[2 * (base + q * ns)] = or_[q];
        dst[2 * (base + q * ns) + 1] = oi[q];
      }
    }
    double* t = src; src = dst; dst = t;
    ns *= r;
  }
  if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

/* ------------------------------------------------------------- 3-D plans */

enum { KIND_R2C = 1, KIND_C2R = 2 };

struct oracle_fftw_plan_s {
  int kind;
  int n0, n1, n2;
  unsigned flags;
};

fftwf_complex* fftwf_alloc_complex(size_t n)
{
  return (fftwf_complex*)malloc(sizeof(fftwf_complex) * (n ? n : 1));
}
float* fftwf_alloc_real(size_t n) { return (float*)malloc(sizeof(float) * (n ? n : 1)); }
void fftwf_free(void* p) { free(p); }
void fftwf_destroy_plan(fftwf_plan p) { free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftwf_mpi_init(void) {}
void fftwf_mpi_cleanup(void) {}

ptrdiff_t fftwf_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                  MPI_Comm comm,
                                  ptrdiff_t* local_n0, ptrdiff_t* local_0_start)
{
  (void)comm;
  *local_n0 = n0;
  *local_0_start = 0;
  return n0 * n1 * n2;
}

ptrdiff_t fftwf_mpi_local_size_3d_transposed(
    ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm,
    ptrdiff_t* local_n0, ptrdiff_t* local_0_start,
    ptrdiff_t* local_n1, ptrdiff_t* local_1_start)
{
  (void)comm;
  *local_n0 = n0; *local_0_start = 0;
  *local_n1 = n1; *local_1_start = 0;
  return n0 * n1 * n2;
}

static fftwf_plan make_plan(int kind, ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                            unsigned flags)
{
  fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
  p->kind = kind;
  p->n0 = (int)n0; p->n1 = (int)n1; p->n2 = (int)n2;
  p->flags = flags;
  return p;
}

fftwf_plan fftwf_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     float* in, fftwf_complex* out,
                                     MPI_Comm comm, unsigned flags)
{
  (void)in; (void)out; (void)comm;
  return make_plan(KIND_R2C, n0, n1, n2, flags);
}

fftwf_plan fftwf_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     fftwf_complex* in, float* out,
                                     MPI_Comm comm, unsigned flags)
{
  (void)in; (void)out; (void)comm;
  return make_plan(KIND_C2R, n0, n1, n2, flags);
}

/* Complex c2c along dimension 0 (stride s0) or 1 (stride s1) of a float
 * complex array t[n0][n1][nh], in blocks of KB columns of the last index. */
#define KB 8

static void pass_dim(float* t, int n0, int n1, int nh, int dim, int sign)
{
  const int nlen = dim == 0 ? n0 : n1;
  const int nother = dim == 0 ? n1 : n0;
  const size_t sl = dim == 0 ? (size_t)n1 * nh : (size_t)nh;  /* stride along line */
  const size_t so = dim == 0 ? (size_t)nh : (size_t)n1 * nh;  /* stride of other dim */
  const int nblk = (nh + KB - 1) / KB;
  fft1d* p = fft1d_make(nlen);
#pragma omp parallel
  {
    double* buf = (double*)malloc(sizeof(double) * 2 * (size_t)nlen * KB);
    double* work = (double*)malloc(sizeof(double) * 2 * (size_t)nlen);
#pragma omp for schedule(static)
    for (long task = 0; task < (long)nother * nblk; task++) {
      const int o = (int)(task / nblk);
      const int k0 = (int)(task % nblk) * KB;
      const int kb = nh - k0 < KB ? nh - k0 : KB;
      for (int i = 0; i < nlen; i++) {
        const float* src = t + 2 * ((size_t)o * so + (size_t)i * sl + k0);
        for (int b = 0; b < kb; b++) {
          buf[2 * ((size_t)b * nlen + i)] = src[2 * b];
          buf[2 * ((size_t)b * nlen + i) + 1] = src[2 * b + 1];
        }
      }
      for (int b = 0; b < kb; b++)
        fft1d_exec(p, buf + 2 * (size_t)b * nlen, work, sign);
      for (int i = 0; i < nlen; i++) {
        float* dst = t + 2 * ((size_t)o * so + (size_t)i * sl + k0);
        for (int b = 0; b < kb; b++) {
          dst[2 * b] = (float)buf[2 * ((size_t)b * nlen + i)];
          dst[2 * b + 1] = (float)buf[2 * ((size_t)b * nlen + i) + 1];
        }
      }
    }
    free(buf);
    free(work);
  }
  fft1d_free(p);
}

void fftwf_mpi_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out)
{
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2;
  const int nh = n2 / 2 + 1;
  const size_t rowr = 2 * (size_t)nh;   /* padded real row */
  float* t = (float*)malloc(sizeof(float) * 2 * (size_t)n0 * n1 * nh);
  fft1d* pz = fft1d_make(n2);
#pragma omp parallel
  {
    double* line = (double*)malloc(sizeof(double) * 2 * (size_t)n2);
    double* work = (double*)malloc(sizeof(double) * 2 * (size_t)n2);
#pragma omp for schedule(static)
    for (long r = 0; r < (long)n0 * n1; r++) {
      const float* src = in + (size_t)r * rowr;
      for (int z = 0; z < n2; z++) { line[2 * z] = src[z]; line[2 * z + 1] = 0.0; }
      fft1d_exec(pz, line, work, -1);
      float* dst = t + 2 * (size_t)r * nh;
      for (int k = 0; k < nh; k++) {
        dst[2 * k] = (float)line[2 * k];
        dst[2 * k + 1] = (float)line[2 * k + 1];
      }
    }
    free(line);
    free(work);
  }
  fft1d_free(pz);
  pass_dim(t, n0, n1, nh, 1, -1);
  pass_dim(t, n0, n1, nh, 0, -1);
  float* o = (float*)out;
  if (p->flags & FFTW_MPI_TRANSPOSED_OUT) {
#pragma omp parallel for schedule(static)
    for (long yx = 0; yx < (long)n1 * n0; yx++) {
      const int y = (int)(yx / n0), x = (int)(yx % n0);
      memcpy(o + 2 * (size_t)yx * nh, t + 2 * ((size_t)x * n1 + y) * nh,
             sizeof(float) * 2 * nh);
    }
  } else {
    memcpy(o, t, sizeof(float) * 2 * (size_t)n0 * n1 * nh);
  }
  free(t);
}

void fftwf_mpi_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out)
{
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2;
  const int nh = n2 / 2 + 1;
  const size_t rowr = 2 * (size_t)nh;
  float* t = (float*)malloc(sizeof(float) * 2 * (size_t)n0 * n1 * nh);
  const float* i_ = (const float*)in;
  if (p->flags & FFTW_MPI_TRANSPOSED_IN) {
#pragma omp parallel for schedule(static)
    for (long xy = 0; xy < (long)n0 * n1; xy++) {
      const int x = (int)(xy / n1), y = (int)(xy % n1);
      memcpy(t + 2 * (size_t)xy * nh, i_ + 2 * ((size_t)y * n0 + x) * nh,
             sizeof(float) * 2 * nh);
    }
  } else {
    memcpy(t, i_, sizeof(float) * 2 * (size_t)n0 * n1 * nh);
  }
  pass_dim(t, n0, n1, nh, 0, +1);
  pass_dim(t, n0, n1, nh, 1, +1);
  fft1d* pz = fft1d_make(n2);
#pragma omp parallel
  {
    double* line = (double*)malloc(sizeof(double) * 2 * (size_t)n2);
    double* work = (double*)malloc(sizeof(double) * 2 * (size_t)n2);
#pragma omp for schedule(static)
    for (long r = 0; r < (long)n0 * n1; r++) {
      const float* src = t + 2 * (size_t)r * nh;
      /* Half-complex convention: Im of k=0 and (even n2) k=n2/2 unused. */
      for (int k = 0; k < nh; k++) {
        line[2 * k] = src[2 * k];
        line[2 * k + 1] = src[2 * k + 1];
      }
      line[1] = 0.0;
      if (n2 % 2 == 0) line[2 * (n2 / 2) + 1] = 0.0;
      for (int k = nh; k < n2; k++) {
        line[2 * k] = line[2 * (n2 - k)];
        line[2 * k + 1] = -line[2 * (n2 - k) + 1];
      }
      fft1d_exec(pz, line, work, +1);
      float* dst = out + (size_t)r * rowr;
      for (int z = 0; z < n2; z++) dst[z] = (float)line[2 * z];
    }
    free(line);
    free(work);
  }
  fft1d_free(pz);
  free(t);
}
