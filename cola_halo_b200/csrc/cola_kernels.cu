// COLA kick / drift / periodic wrap / snapshot on structure-of-arrays
// particle state, and the AoS <-> SoA conversions for the reference's
// Particle layout.  Per-particle arithmetic reproduces the reference's
// single/double precision mix and operation order (intrinsics prevent FMA
// contraction), so results are bit-identical to cola.c given the same inputs
// and coefficients.
#include <cuda_runtime.h>
#include <stddef.h>

#include "internal.h"

namespace {

constexpr int T = CG_THREADS;

struct P3 { float* p[3]; };
struct C3 { const float* p[3]; };

P3 mk(float* const a[3]) { return P3{{a[0], a[1], a[2]}}; }
C3 mkc(const float* const a[3]) { return C3{{a[0], a[1], a[2]}}; }

// move.c:34-41: one-shot periodic wrap of each coordinate.
__global__ void __launch_bounds__(T) k_wrap(P3 x, long long n, float L) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    // the three loads first: the component arrays may alias as far as the
    // compiler knows, so a store would hold back the next load
    float v[3];
#pragma unroll
    for (int a = 0; a < 3; a++) v[a] = x.p[a][i];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (v[a] < 0.0f) x.p[a][i] = __fadd_rn(v[a], L);
      else if (v[a] >= L) x.p[a][i] = __fsub_rn(v[a], L);
    }
  }
}

// cola.c:105-111
//   ax = (float)((-1.5 * (double)Om) * (double)f - (double)(dx1*q1 + dx2*q2))
//   v += ax * dda
__device__ __forceinline__ float kick_acc(float f, float d1, float d2, double c, float q1,
                                          float q2) {
  const float s = __fadd_rn(__fmul_rn(d1, q1), __fmul_rn(d2, q2));
  return __double2float_rn(__dsub_rn(__dmul_rn(c, (double)f), (double)s));
}

__global__ void __launch_bounds__(T) k_kick(P3 v, C3 f, C3 dx1, C3 dx2, long long n,
                                            double c, float dda, float q1, float q2) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    float fv[3], d1[3], d2[3], vv[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      fv[a] = f.p[a][i];
      d1[a] = dx1.p[a][i];
      d2[a] = dx2.p[a][i];
      vv[a] = v.p[a][i];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float ax = kick_acc(fv[a], d1[a], d2[a], c, q1, q2);
      v.p[a][i] = __fadd_rn(vv[a], __fmul_rn(ax, dda));
    }
  }
}

// cola.c:142-149:  x += v*dyyy + (dx1*da1 + dx2*da2)
__global__ void __launch_bounds__(T) k_drift(P3 x, C3 v, C3 dx1, C3 dx2, long long n,
                                             float dyyy, float da1, float da2) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    float xv[3], vv[3], d1[3], d2[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      xv[a] = x.p[a][i];
      vv[a] = v.p[a][i];
      d1[a] = dx1.p[a][i];
      d2[a] = dx2.p[a][i];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float lpt = __fadd_rn(__fmul_rn(d1[a], da1), __fmul_rn(d2[a], da2));
      const float step = __fadd_rn(__fmul_rn(vv[a], dyyy), lpt);
      x.p[a][i] = __fadd_rn(xv[a], step);
    }
  }
}

// cola_kick then cola_drift of the same particle in one pass (the kick's
// new velocity feeds the drift, as in the two calls): reads x, v, f, dx1,
// dx2 once and writes x and v once.  The arithmetic is k_kick's followed by
// k_drift's, so the results are bit-identical to the two kernels.
__global__ void __launch_bounds__(T) k_kick_drift(P3 x, P3 v, C3 f, C3 dx1, C3 dx2, long long n,
                                                  double c, float dda, float q1, float q2,
                                                  float dyyy, float da1, float da2) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    // all 15 loads first (the arrays may alias as far as the compiler
    // knows, so stores would otherwise hold back the next component's loads)
    float xv[3], vv[3], fv[3], d1[3], d2[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      xv[a] = x.p[a][i];
      vv[a] = v.p[a][i];
      fv[a] = f.p[a][i];
      d1[a] = dx1.p[a][i];
      d2[a] = dx2.p[a][i];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float ax = kick_acc(fv[a], d1[a], d2[a], c, q1, q2);
      vv[a] = __fadd_rn(vv[a], __fmul_rn(ax, dda));
      const float lpt = __fadd_rn(__fmul_rn(d1[a], da1), __fmul_rn(d2[a], da2));
      xv[a] = __fadd_rn(xv[a], __fadd_rn(__fmul_rn(vv[a], dyyy), lpt));
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      v.p[a][i] = vv[a];
      x.p[a][i] = xv[a];
    }
  }
}

// Reference ParticleMinimum (particle.h:29-33): float x[3], v[3]; long long id.
struct PMin { float x[3]; float v[3]; long long id; };
// Reference Particle (particle.h:8-14).
struct PFull { float x[3]; float dx1[3]; float dx2[3]; float v[3]; long long id; };
static_assert(sizeof(PMin) == 32, "ParticleMinimum is 32 bytes");
static_assert(sizeof(PFull) == 56, "Particle is 56 bytes");

// cola.c:388-410
__global__ void __launch_bounds__(T) k_snapshot(C3 x, C3 v, C3 f, C3 dx1, C3 dx2, long long n,
                                                double c, float dda, float q1, float q2,
                                                float Dv, float Dv2, float dyyy, float da1,
                                                float da2, float vfac,
                                                const long long* __restrict__ id,
                                                const int* __restrict__ orig,
                                                PMin* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    PMin o;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float d1 = dx1.p[a][i], d2 = dx2.p[a][i], vv = v.p[a][i];
      const float ax = kick_acc(f.p[a][i], d1, d2, c, q1, q2);
      // vfac*(v + ax*dda + (dx1*Dv + dx2*Dv2)*1)
      float s = __fadd_rn(vv, __fmul_rn(ax, dda));
      s = __fadd_rn(s, __fadd_rn(__fmul_rn(d1, Dv), __fmul_rn(d2, Dv2)));
      o.v[a] = __fmul_rn(vfac, s);
      // x + v*dyyy + 1*(dx1*da1 + dx2*da2)
      const float p = __fadd_rn(x.p[a][i], __fmul_rn(vv, dyyy));
      o.x[a] = __fadd_rn(p, __fadd_rn(__fmul_rn(d1, da1), __fmul_rn(d2, da2)));
    }
    o.id = id[i];
    out[orig ? orig[i] : i] = o;
  }
}

// set_noncola_initial (cola.c:297-338): positions as they are, 2LPT
// velocities vfac (dx1 Dv + dx2 Dv2) in float, in the caller's order
__global__ void __launch_bounds__(T) k_initial_snapshot(C3 x, C3 dx1, C3 dx2, long long n,
                                                        float vfac, float Dv, float Dv2,
                                                        const long long* __restrict__ id,
                                                        const int* __restrict__ orig,
                                                        PMin* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    PMin o;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float d1 = dx1.p[a][i], d2 = dx2.p[a][i];
      o.v[a] = __fmul_rn(vfac, __fadd_rn(__fmul_rn(d1, Dv), __fmul_rn(d2, Dv2)));
      o.x[a] = x.p[a][i];
    }
    o.id = id[i];
    out[orig ? orig[i] : i] = o;
  }
}

__global__ void __launch_bounds__(T) k_aos_to_soa(const PFull* __restrict__ in, long long n,
                                                  P3 x, P3 dx1, P3 dx2, P3 v,
                                                  long long* __restrict__ id,
                                                  int* __restrict__ orig) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    const PFull p = in[i];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      x.p[a][i] = p.x[a];
      dx1.p[a][i] = p.dx1[a];
      dx2.p[a][i] = p.dx2[a];
      v.p[a][i] = p.v[a];
    }
    id[i] = p.id;
    if (orig) orig[i] = (int)i;
  }
}

__global__ void __launch_bounds__(T) k_soa_to_aos(PFull* __restrict__ out, long long n, C3 x,
                                                  C3 dx1, C3 dx2, C3 v,
                                                  const long long* __restrict__ id,
                                                  const int* __restrict__ orig) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    PFull p;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      p.x[a] = x.p[a][i];
      p.dx1[a] = dx1.p[a][i];
      p.dx2[a] = dx2.p[a][i];
      p.v[a] = v.p[a][i];
    }
    p.id = id[i];
    out[orig ? orig[i] : i] = p;
  }
}

}  // namespace

cudaError_t dev_wrap(float* const x[3], long long n, float L, cudaStream_t st) {
  prof_mark(st, CG_ST_WRAP);
  if (n > 0) k_wrap<<<grid_for(n), T, 0, st>>>(mk(x), n, L);
  return cudaGetLastError();
}

cudaError_t dev_kick(float* const v[3], const float* const f[3], const float* const dx1[3],
                      const float* const dx2[3], long long n, float omega_m, float dda,
                      float q1, float q2, cudaStream_t st) {
  const double c = -1.5 * (double)omega_m;      // cola.c:105  -1.5*Om (double)
  prof_mark(st, CG_ST_KICK);
  if (n > 0) k_kick<<<grid_for(n), T, 0, st>>>(mk(v), mkc(f), mkc(dx1), mkc(dx2), n, c, dda, q1, q2);
  return cudaGetLastError();
}

cudaError_t dev_drift(float* const x[3], const float* const v[3], const float* const dx1[3],
                       const float* const dx2[3], long long n, float dyyy, float da1,
                       float da2, cudaStream_t st) {
  prof_mark(st, CG_ST_DRIFT);
  if (n > 0) k_drift<<<grid_for(n), T, 0, st>>>(mk(x), mkc(v), mkc(dx1), mkc(dx2), n, dyyy, da1, da2);
  return cudaGetLastError();
}

cudaError_t dev_kick_drift(float* const x[3], float* const v[3], const float* const f[3],
                           const float* const dx1[3], const float* const dx2[3], long long n,
                           float omega_m, float dda, float q1, float q2, float dyyy, float da1,
                           float da2, cudaStream_t st) {
  const double c = -1.5 * (double)omega_m;
  prof_mark(st, CG_ST_KICK_DRIFT);
  if (n > 0)
    k_kick_drift<<<grid_for(n), T, 0, st>>>(mk(x), mk(v), mkc(f), mkc(dx1), mkc(dx2), n, c, dda,
                                            q1, q2, dyyy, da1, da2);
  return cudaGetLastError();
}

cudaError_t dev_snapshot(const float* const x[3], const float* const v[3],
                          const float* const f[3], const float* const dx1[3],
                          const float* const dx2[3], long long n, float omega_m, float dda,
                          float q1, float q2, float Dv, float Dv2, float dyyy, float da1,
                          float da2, float vfac, const long long* id, const int* orig,
                          void* out_aos, cudaStream_t st) {
  const double c = -1.5 * (double)omega_m;
  prof_mark(st, CG_ST_SNAPSHOT);
  if (n > 0)
    k_snapshot<<<grid_for(n), T, 0, st>>>(mkc(x), mkc(v), mkc(f), mkc(dx1), mkc(dx2), n, c,
                                          dda, q1, q2, Dv, Dv2, dyyy, da1, da2, vfac, id,
                                          orig, reinterpret_cast<PMin*>(out_aos));
  return cudaGetLastError();
}

cudaError_t dev_initial_snapshot(const ParticleSoA* s, float vfac, float Dv, float Dv2,
                                 void* out_aos, cudaStream_t st) {
  prof_mark(st, CG_ST_SNAPSHOT);
  if (s->n > 0)
    k_initial_snapshot<<<grid_for(s->n), T, 0, st>>>(mkc(s->x), mkc(s->dx1), mkc(s->dx2), s->n,
                                                     vfac, Dv, Dv2, s->id, s->orig,
                                                     reinterpret_cast<PMin*>(out_aos));
  return cudaGetLastError();
}

cudaError_t particles_aos_to_soa(const void* aos, ParticleSoA* s, cudaStream_t st) {
  prof_mark(st, CG_ST_OTHER);
  if (s->n > 0)
    k_aos_to_soa<<<grid_for(s->n), T, 0, st>>>(reinterpret_cast<const PFull*>(aos), s->n,
                                               mk(s->x), mk(s->dx1), mk(s->dx2), mk(s->v), s->id,
                                               s->orig);
  return cudaGetLastError();
}

cudaError_t particles_soa_to_aos(void* aos, const ParticleSoA* s, cudaStream_t st) {
  prof_mark(st, CG_ST_OTHER);
  if (s->n > 0)
    k_soa_to_aos<<<grid_for(s->n), T, 0, st>>>(reinterpret_cast<PFull*>(aos), s->n,
                                               mkc(s->x), mkc(s->dx1), mkc(s->dx2), mkc(s->v),
                                               s->id, s->orig);
  return cudaGetLastError();
}
