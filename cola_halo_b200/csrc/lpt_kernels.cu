// Second-order Lagrangian perturbation theory initial conditions on the GPU
// (lpt.c:145-578 on one process).
//
//  1. seed table: one RANLUX stream on the host (lpt.c:172-207)
//  2. modes: one thread per (kx, ky) column seeds its own RANLUX stream with
//     the table entry and draws phase / amplitude for kz = 0..N/2-1
//     (lpt.c:219-351), writing the Zel'dovich displacement spectra
//  3. gradients i k_j psi_i, six c2r (lpt.c:358-403)
//  4. second-order source in real space, r2c (lpt.c:409-427)
//  5. 2LPT displacement spectra -i k/k^2 S, c2r (lpt.c:440-503)
//  6. particles on the lattice (lpt.c:532-561)
// Spectra use the mesh layout [kz][kx][ky]; real grids [x][y][z].
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../../include/colagpu.h"
#include "internal.h"
#include "lpt.h"

extern int cg_set_error_from_lpt(int code, const char* msg);

namespace {

constexpr int T = CG_THREADS;
constexpr double kUlp48 = 1.0 / 281474976710656.0;   // 2^-48

// ------------------------------------------------------------- RANLUX-48
// Luscher's RANLUX in 48-bit form: x_k = x_{k-5} - x_{k-12} - c (mod 1) on
// 12 words held as doubles in [0,1); 202 steps per block of 12 delivered
// numbers (luxury level 1); seeding from a 31-bit shift register
// b(n+31) = b(n) xor b(n+18) of the seed's bits.
struct DevRanlux {
  double x[12];
  double carry;
  int ir, jr, ir_old;
};

__host__ __device__ inline void rlx_seed(double* x, double* carry, int* ir, int* jr, int* ir_old,
                                         unsigned long s) {
  if (s == 0) s = 1;
  int bits[31];
  unsigned long v = s & 0xFFFFFFFFUL;
  for (int k = 0; k < 31; k++) { bits[k] = (int)(v & 1UL); v >>= 1; }
  int ib = 0, jb = 18;
  for (int w = 0; w < 12; w++) {
    double acc = 0.0;
    for (int l = 0; l < 48; l++) {
      acc = 2.0 * acc + (double)(bits[ib] ^ 1);
      bits[ib] ^= bits[jb];
      ib = ib == 30 ? 0 : ib + 1;
      jb = jb == 30 ? 0 : jb + 1;
    }
    x[w] = acc * kUlp48;
  }
  *carry = 0.0;
  *ir = 11;
  *jr = 7;
  *ir_old = 0;
}

__host__ __device__ inline void rlx_refill(double* x, double* carry, int* ir, int* jr, int* ir_old,
                                           int pr) {
  int i = *ir, j = *jr;
  double c = *carry;
  for (int k = 0; k < pr; k++) {
    double y = x[j] - x[i] - c;
    if (y < 0.0) { c = kUlp48; y += 1.0; }
    else c = 0.0;
    x[i] = y;
    i = i == 11 ? 0 : i + 1;
    j = j == 11 ? 0 : j + 1;
  }
  *ir = i;
  *jr = j;
  *ir_old = i;
  *carry = c;
}

__host__ __device__ inline double rlx_uniform(double* x, double* carry, int* ir, int* jr,
                                              int* ir_old, int pr) {
  *ir = *ir == 11 ? 0 : *ir + 1;
  if (*ir == *ir_old) rlx_refill(x, carry, ir, jr, ir_old, pr);
  return x[*ir];
}

// --------------------------------------------------------------- modes
// PowerSpec (power.c:120-151) on a device copy of the table.
__device__ double power_spec(double k, const double* __restrict__ logk,
                             const double* __restrict__ logD, int n, double norm) {
  const double lk = log10(k);
  if (lk < logk[0] || lk > logk[n - 1]) return 0.0;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (hi + lo) / 2;
    if (lk < logk[mid]) hi = mid;
    else lo = mid;
  }
  const double u = (lk - logk[lo]) / (logk[hi] - logk[lo]);
  const double ld = (1 - u) * logD[lo] + u * logD[hi];
  return norm * pow(10.0, ld) / (4.0 * M_PI * k * k * k);
}

__device__ __forceinline__ double kvec_of(int i, int N, double kf) {
  return (i < N / 2 ? (double)i : -(double)(N - i)) * kf;
}

// lpt.c:219-351: modes of column (i, j); cd_a[k][i][j] for k < N/2.
__global__ void __launch_bounds__(T) k_modes(int N, double box, const unsigned* __restrict__ seeds,
                                             const double* __restrict__ logk,
                                             const double* __restrict__ logD, int ntab,
                                             double norm, float2* __restrict__ c0,
                                             float2* __restrict__ c1, float2* __restrict__ c2) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * N) return;
  const int i = (int)(t / N), j = (int)(t % N);
  double x[12], carry;
  int ir, jr, ir_old;
  rlx_seed(x, &carry, &ir, &jr, &ir_old, seeds[(size_t)i * N + j]);
  const double kf = 2 * M_PI / box;
  const double fac = pow(2 * M_PI / box, 1.5);
  float2* cd[3] = {c0, c1, c2};
  const size_t plane = (size_t)N * N;
  for (int k = 0; k < N / 2; k++) {
    const double phase = rlx_uniform(x, &carry, &ir, &jr, &ir_old, 202) * 2 * M_PI;
    double ampl;
    do {
      ampl = rlx_uniform(x, &carry, &ir, &jr, &ir_old, 202);
    } while (ampl == 0.0);
    if (i == N / 2 || j == N / 2 || k == N / 2) continue;
    if (i == 0 && j == 0 && k == 0) continue;
    const double kv[3] = {kvec_of(i, N, kf), kvec_of(j, N, kf), kvec_of(k, N, kf)};
    const double kmag2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
    const double kmag = sqrt(kmag2);
    double p = power_spec(kmag, logk, logD, ntab, norm);
    p *= -log(ampl);
    const double delta = fac * sqrt(p);
    double sp, cp;
    sincos(phase, &sp, &cp);
    if (k > 0) {
      for (int a = 0; a < 3; a++)
        cd[a][k * plane + (size_t)i * N + j] =
            make_float2((float)(-kv[a] / kmag2 * delta * sp), (float)(kv[a] / kmag2 * delta * cp));
    } else if (i == 0) {
      if (j >= N / 2) continue;
      const int jj = N - j;
      for (int a = 0; a < 3; a++) {
        cd[a][(size_t)i * N + j] =
            make_float2((float)(-kv[a] / kmag2 * delta * sp), (float)(kv[a] / kmag2 * delta * cp));
        cd[a][(size_t)i * N + jj] =
            make_float2((float)(-kv[a] / kmag2 * delta * sp), (float)(-kv[a] / kmag2 * delta * cp));
      }
    } else {
      if (i >= N / 2) continue;
      const int ii = N - i;
      const int jj = j == 0 ? 0 : N - j;
      for (int a = 0; a < 3; a++) {
        cd[a][(size_t)i * N + j] =
            make_float2((float)(-kv[a] / kmag2 * delta * sp), (float)(kv[a] / kmag2 * delta * cp));
        cd[a][(size_t)ii * N + jj] =
            make_float2((float)(-kv[a] / kmag2 * delta * sp), (float)(-kv[a] / kmag2 * delta * cp));
      }
    }
  }
}

// lpt.c:358-398: i k_j psi_i for (0,0) (0,1) (0,2) (1,1) (1,2) (2,2).
struct Spec6 { float2* p[6]; };
__global__ void __launch_bounds__(T) k_gradients(int N, double kf, const float2* __restrict__ c0,
                                                 const float2* __restrict__ c1,
                                                 const float2* __restrict__ c2, Spec6 g) {
  const size_t total = (size_t)(N / 2 + 1) * N * N;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(t / ((size_t)N * N));
    const int i = (int)((t / N) % N);
    const int j = (int)(t % N);
    const double kx = kvec_of(i, N, kf), ky = kvec_of(j, N, kf), kz = kvec_of(k, N, kf);
    const float2 a = c0[t], b = c1[t], c = c2[t];
    g.p[0][t] = make_float2((float)(-(double)a.y * kx), (float)((double)a.x * kx));
    g.p[1][t] = make_float2((float)(-(double)a.y * ky), (float)((double)a.x * ky));
    g.p[2][t] = make_float2((float)(-(double)a.y * kz), (float)((double)a.x * kz));
    g.p[3][t] = make_float2((float)(-(double)b.y * ky), (float)((double)b.x * ky));
    g.p[4][t] = make_float2((float)(-(double)b.y * kz), (float)((double)b.x * kz));
    g.p[5][t] = make_float2((float)(-(double)c.y * kz), (float)((double)c.x * kz));
  }
}

// lpt.c:409-422 (float arithmetic in the reference's order).
struct Real6 { float* p[6]; };
__global__ void __launch_bounds__(T) k_source(size_t n, Real6 d, float* __restrict__ src) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const float d0 = d.p[0][t], d1 = d.p[1][t], d2 = d.p[2][t];
    const float d3 = d.p[3][t], d4 = d.p[4][t], d5 = d.p[5][t];
    float s = __fmul_rn(d0, __fadd_rn(d3, d5));
    s = __fadd_rn(s, __fmul_rn(d3, d5));
    s = __fsub_rn(s, __fmul_rn(d1, d1));
    s = __fsub_rn(s, __fmul_rn(d2, d2));
    s = __fsub_rn(s, __fmul_rn(d4, d4));
    src[t] = s;
  }
}

// lpt.c:440-494: cdisp2_a = -i k_a / k^2 S.
__global__ void __launch_bounds__(T) k_disp2(int N, double kf, const float2* __restrict__ S,
                                             float2* __restrict__ o0, float2* __restrict__ o1,
                                             float2* __restrict__ o2) {
  const size_t total = (size_t)(N / 2 + 1) * N * N;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(t / ((size_t)N * N));
    const int i = (int)((t / N) % N);
    const int j = (int)(t % N);
    const double kv[3] = {kvec_of(i, N, kf), kvec_of(j, N, kf), kvec_of(k, N, kf)};
    const double kmag2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
    const float2 s = S[t];
    float2* o[3] = {o0, o1, o2};
    for (int a = 0; a < 3; a++) {
      if (kmag2 > 0.0)
        o[a][t] = make_float2((float)((double)s.y * kv[a] / kmag2),
                              (float)(-(double)s.x * kv[a] / kmag2));
      else
        o[a][t] = make_float2(0.0f, 0.0f);
    }
  }
}

// lpt.c:532-561: lattice positions plus displacements; Particle AoS out.
struct PFull { float x[3]; float dx1[3]; float dx2[3]; float v[3]; long long id; };
struct Real3c { const float* p[3]; };
__global__ void __launch_bounds__(T) k_particles(int N, float dx, Real3c dis, Real3c dis2,
                                                 double nmesh3_inv, double dplus, double D2,
                                                 double D20, PFull* __restrict__ out) {
  const size_t n = (size_t)N * N * N;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / ((size_t)N * N));
    const int j = (int)((t / N) % N);
    const int k = (int)(t % N);
    const float q[3] = {__fmul_rn(__fadd_rn((float)i, 0.5f), dx),
                        __fmul_rn(__fadd_rn((float)j, 0.5f), dx),
                        __fmul_rn(__fadd_rn((float)k, 0.5f), dx)};
    PFull p;
    const double c37 = 3.0 / 7.0;
    for (int a = 0; a < 3; a++) {
      const float d1 = dis.p[a][t];
      const float d2 = (float)__dmul_rn(nmesh3_inv, (double)dis2.p[a][t]);
      // x + dis*Dplus - 3.0/7.0*D20*dis2*D2, left to right
      const double t2 = __dmul_rn(__dmul_rn(__dmul_rn(c37, D20), (double)d2), D2);
      p.x[a] = (float)__dsub_rn(__dadd_rn((double)q[a], __dmul_rn((double)d1, dplus)), t2);
      p.dx1[a] = d1;
      p.dx2[a] = (float)__dmul_rn(__dmul_rn(-c37, D20), (double)d2);
      p.v[a] = 0.0f;
    }
    p.id = (long long)t + 1;
    out[t] = p;
  }
}

// ------------------------------------------------------------ buffers
struct LptBuffers {
  int N = 0;
  MeshFFT fft{};
  float2* cd[3] = {};
  float2* gs[6] = {};
  float* gr[6] = {};
  unsigned* seeds = nullptr;
  double* tab = nullptr;
  int ntab = 0;
  void* aos = nullptr;
  cudaStream_t st = nullptr;
};
LptBuffers g_lpt;

void release() {
  if (g_lpt.st) cudaStreamSynchronize(g_lpt.st);
  for (int a = 0; a < 3; a++) cudaFree(g_lpt.cd[a]);
  for (int a = 0; a < 6; a++) { cudaFree(g_lpt.gs[a]); cudaFree(g_lpt.gr[a]); }
  cudaFree(g_lpt.seeds);
  cudaFree(g_lpt.tab);
  cudaFree(g_lpt.aos);
  mesh_fft_free(&g_lpt.fft);
  if (g_lpt.st) cudaStreamDestroy(g_lpt.st);
  g_lpt = LptBuffers();
}

cudaError_t ensure(int N) {
  if (g_lpt.N == N) return cudaSuccess;
  release();
  cudaError_t e = cudaStreamCreateWithFlags(&g_lpt.st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = mesh_fft_alloc(&g_lpt.fft, N);
  const size_t sb = sizeof(float2) * (size_t)(N / 2 + 1) * N * N;
  const size_t rb = sizeof(float) * (size_t)N * N * N;
  for (int a = 0; a < 3 && e == cudaSuccess; a++) e = cudaMalloc(&g_lpt.cd[a], sb);
  for (int a = 0; a < 6 && e == cudaSuccess; a++) e = cudaMalloc(&g_lpt.gs[a], sb);
  for (int a = 0; a < 6 && e == cudaSuccess; a++) e = cudaMalloc(&g_lpt.gr[a], rb);
  if (e == cudaSuccess) e = cudaMalloc(&g_lpt.seeds, sizeof(unsigned) * (size_t)N * N);
  if (e == cudaSuccess) e = cudaMalloc(&g_lpt.aos, 56 * (size_t)N * N * N);
  if (e != cudaSuccess) {
    release();
    return e;
  }
  g_lpt.N = N;
  return cudaSuccess;
}

}  // namespace

// ------------------------------------------------------------ host RNG
void Ranlux48::seed(unsigned long s) {
  pr = 202;
  rlx_seed(x, &carry, &ir, &jr, &ir_old, s);
}
double Ranlux48::uniform() { return rlx_uniform(x, &carry, &ir, &jr, &ir_old, pr); }

void lpt_dropin_release() { release(); }

// lpt.c:177-207
static void seed_table(int N, int seed, std::vector<unsigned>& st) {
  Ranlux48 r;
  r.seed((unsigned long)seed);
  st.assign((size_t)N * N, 0u);
  auto draw = [&]() { return (unsigned)(0x7fffffff * r.uniform()); };
  for (int i = 0; i < N / 2; i++) {
    for (int j = 0; j < i; j++) st[(size_t)i * N + j] = draw();
    for (int j = 0; j < i + 1; j++) st[(size_t)j * N + i] = draw();
    for (int j = 0; j < i; j++) st[(size_t)(N - 1 - i) * N + j] = draw();
    for (int j = 0; j < i + 1; j++) st[(size_t)(N - 1 - j) * N + i] = draw();
    for (int j = 0; j < i; j++) st[(size_t)i * N + (N - 1 - j)] = draw();
    for (int j = 0; j < i + 1; j++) st[(size_t)j * N + (N - 1 - i)] = draw();
    for (int j = 0; j < i; j++) st[(size_t)(N - 1 - i) * N + (N - 1 - j)] = draw();
    for (int j = 0; j < i + 1; j++) st[(size_t)(N - 1 - j) * N + (N - 1 - i)] = draw();
  }
}

int lpt_generate(int nc, double boxsize, int seed, double omega_m, double a_init, double dplus,
                 const PowerTable& power, void* particles_host) {
  const int N = nc;
  if (!pm_supported_mesh(N))
    return cg_set_error_from_lpt(CG_EUNSUPPORTED, "2LPT grid size not built into this library");
  cudaError_t e = ensure(N);
  if (e != cudaSuccess) return cg_set_error_from_lpt(CG_ENOMEM, cudaGetErrorString(e));
  cudaStream_t st = g_lpt.st;
  std::vector<unsigned> seeds;
  seed_table(N, seed, seeds);
  const int ntab = (int)power.logk.size();
  std::vector<double> tab(2 * (size_t)ntab);
  for (int i = 0; i < ntab; i++) {
    tab[i] = power.logk[i];
    tab[ntab + i] = power.logD[i];
  }
  if (ntab != g_lpt.ntab) {
    cudaFree(g_lpt.tab);
    g_lpt.tab = nullptr;
    e = cudaMalloc(&g_lpt.tab, sizeof(double) * 2 * ntab);
    if (e != cudaSuccess) return cg_set_error_from_lpt(CG_ENOMEM, cudaGetErrorString(e));
    g_lpt.ntab = ntab;
  }
  const size_t sb = sizeof(float2) * (size_t)(N / 2 + 1) * N * N;
  const size_t nreal = (size_t)N * N * N;
  const double kf = 2 * M_PI / boxsize;
  e = cudaMemcpyAsync(g_lpt.seeds, seeds.data(), sizeof(unsigned) * seeds.size(),
                      cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g_lpt.tab, tab.data(), sizeof(double) * tab.size(),
                        cudaMemcpyHostToDevice, st);
  for (int a = 0; a < 3 && e == cudaSuccess; a++) e = cudaMemsetAsync(g_lpt.cd[a], 0, sb, st);
  if (e != cudaSuccess) return cg_set_error_from_lpt(CG_ECUDA, cudaGetErrorString(e));
  // 2. modes
  {
    const long long cols = (long long)N * N;
    prof_mark(st, CG_ST_LPT);
    k_modes<<<(int)((cols + T - 1) / T), T, 0, st>>>(N, boxsize, g_lpt.seeds, g_lpt.tab,
                                                      g_lpt.tab + ntab, ntab, power.norm,
                                                      g_lpt.cd[0], g_lpt.cd[1], g_lpt.cd[2]);
  }
  // 3. gradients and six c2r
  Spec6 g6;
  for (int a = 0; a < 6; a++) g6.p[a] = g_lpt.gs[a];
  prof_mark(st, CG_ST_LPT);
  k_gradients<<<grid_for((long long)(N / 2 + 1) * N * N), T, 0, st>>>(N, kf, g_lpt.cd[0],
                                                                     g_lpt.cd[1], g_lpt.cd[2], g6);
  for (int a = 0; a < 6; a++) mesh_c2r(&g_lpt.fft, g_lpt.gs[a], g_lpt.gr[a], st);
  // 4. source (into gr[3]) and r2c (into gs[0])
  Real6 r6;
  for (int a = 0; a < 6; a++) r6.p[a] = g_lpt.gr[a];
  prof_mark(st, CG_ST_LPT);
  k_source<<<grid_for((long long)nreal), T, 0, st>>>(nreal, r6, g_lpt.gr[3]);
  mesh_r2c(&g_lpt.fft, g_lpt.gr[3], g_lpt.gs[0], st);
  // 5. 2LPT spectra into gs[1..3]
  prof_mark(st, CG_ST_LPT);
  k_disp2<<<grid_for((long long)(N / 2 + 1) * N * N), T, 0, st>>>(N, kf, g_lpt.gs[0], g_lpt.gs[1],
                                                                 g_lpt.gs[2], g_lpt.gs[3]);
  // c2r: ZA -> gr[0..2], 2LPT -> gr[3..5]
  for (int a = 0; a < 3; a++) {
    mesh_c2r(&g_lpt.fft, g_lpt.cd[a], g_lpt.gr[a], st);
    mesh_c2r(&g_lpt.fft, g_lpt.gs[1 + a], g_lpt.gr[3 + a], st);
  }
  // 6. particles
  const double om = omega_m;
  const double omega = om / (om + (1.0 - om) * a_init * a_init * a_init);
  const double D2 = dplus * dplus * pow(omega / om, -1.0 / 143.0);   // lpt.c:522-524
  const double D20 = pow(om, -1.0 / 143.0);
  const float dx = (float)(boxsize / N);
  Real3c dis = {{g_lpt.gr[0], g_lpt.gr[1], g_lpt.gr[2]}};
  Real3c dis2 = {{g_lpt.gr[3], g_lpt.gr[4], g_lpt.gr[5]}};
  prof_mark(st, CG_ST_LPT);
  k_particles<<<grid_for((long long)nreal), T, 0, st>>>(N, dx, dis, dis2,
                                                        1.0 / pow((double)N, 3.0), dplus, D2,
                                                        D20, (PFull*)g_lpt.aos);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(particles_host, g_lpt.aos, 56 * nreal, cudaMemcpyDefault, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cg_set_error_from_lpt(CG_ECUDA, cudaGetErrorString(e));
  return CG_OK;
}
