// Cell order of the particle arrays.
//
// The reference keeps its particles in the order 2LPT created them (the
// Lagrangian lattice) for the whole run.  As structure forms, particles from
// distant lattice sites gather in the same halo, so a warp's 32 particles
// no longer touch neighbouring mesh cells.  The CIC deposit's atomics and
// the interpolation's gathers then miss in L2, and both slow down several
// times between the first and the last steps.  Sorting the particles by a
// grid of about eight particles per cell restores the locality of the
// initial lattice.  The sort is a counting sort: the bin of each particle with its
// count, a prefix sum over the bins, and one scatter of every per-particle
// array (forces included, so that no call order depends on the sort) into a
// second set of arrays.  orig[] follows the particles, so every
// output can be put back in the caller's order.
#include <cuda_runtime.h>
#include <math.h>

#include "internal.h"
#include "scan.cuh"

namespace {

constexpr int T = CG_THREADS;

struct P3 { float* p[3]; };
struct C3 { const float* p[3]; };

// bin (ix nb + iy) nb + iz of each particle, its count, and the particle's
// rank among the bin's arrivals
__global__ void __launch_bounds__(T) k_sort_bin(C3 x, long long n, float scale, int nb,
                                                unsigned* __restrict__ key,
                                                unsigned* __restrict__ rank,
                                                unsigned* __restrict__ cnt) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int v = (int)(x.p[a][i] * scale);   // NaN converts to 0
      c[a] = v < 0 ? 0 : (v >= nb ? nb - 1 : v);
    }
    const unsigned k = (unsigned)(((long long)c[0] * nb + c[1]) * nb + c[2]);
    key[i] = k;
    // one atomic per distinct bin of the warp: in cell order most of a
    // warp's particles share a bin, and same-address atomics serialise
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, k);
    const int leader = __ffs(peers) - 1;
    const int lane = threadIdx.x & 31;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(cnt + k, (unsigned)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    rank[i] = base + (unsigned)__popc(peers & ((1u << lane) - 1u));
  }
}

// particle i to slot start[bin] + rank: no atomics, one float3 group at a
// time (loads of the next group overlap the stores of this one)
__device__ __forceinline__ void move3(const C3& in, const P3& out, long long i, unsigned j) {
  const float a = in.p[0][i], b = in.p[1][i], c = in.p[2][i];
  out.p[0][j] = a;
  out.p[1][j] = b;
  out.p[2][j] = c;
}

__global__ void __launch_bounds__(T) k_sort_scatter(
    C3 x, C3 v, C3 d1, C3 d2, C3 f, const long long* __restrict__ id,
    const int* __restrict__ orig, long long n, const unsigned* __restrict__ key,
    const unsigned* __restrict__ rank, const unsigned* __restrict__ start, P3 xo, P3 vo,
    P3 d1o, P3 d2o, P3 fo, long long* __restrict__ ido, int* __restrict__ origo) {
  // one particle per thread: the 34 array pointers are read from the
  // parameter bank where they are used instead of living in registers
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= n) return;
  const unsigned j = start[key[i]] + rank[i];
  move3(x, xo, i, j);
  move3(v, vo, i, j);
  move3(d1, d1o, i, j);
  move3(d2, d2o, i, j);
  move3(f, fo, i, j);
  ido[j] = id[i];
  origo[j] = orig[i];
}

// f back to the caller's order: fo[orig[i]] = f[i]
__global__ void __launch_bounds__(T) k_unsort_forces(C3 f, const int* __restrict__ orig,
                                                     long long n, P3 fo) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    const int j = orig[i];
    if (j < 0 || (long long)j >= n) continue;
#pragma unroll
    for (int a = 0; a < 3; a++) fo.p[a][j] = f.p[a][i];
  }
}

template <class A>
void release(A*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace

void particle_order_free(ParticleOrder* o) {
  release(o->alloc);
  release(o->alloc_id);
  release(o->alloc_orig);
  release(o->key);
  release(o->cnt);
  release(o->bsum);
  *o = ParticleOrder{};
}

namespace {
// Bins per side for n particles: about eight particles per bin (a bin is
// then two lattice spacings on a side, six mesh cells at a PM factor of 3),
// at most 1024 per side.
int bins_per_side(long long n) {
  int nb = (int)llround(cbrt((double)n) / 2.0);
  if (nb < 1) nb = 1;
  if (nb > 1024) nb = 1024;
  return nb;
}

cudaError_t order_alloc(ParticleOrder* o, long long cap) {
  const size_t c = (size_t)cap;
  cudaError_t e = cudaMalloc(&o->alloc, sizeof(float) * 15 * c);
  if (e == cudaSuccess) e = cudaMalloc(&o->alloc_id, sizeof(long long) * c);
  if (e == cudaSuccess) e = cudaMalloc(&o->alloc_orig, sizeof(int) * c);
  if (e == cudaSuccess) e = cudaMalloc(&o->key, sizeof(unsigned) * 2 * c);   // key, rank
  if (e != cudaSuccess) {
    particle_order_free(o);
    return e;
  }
  for (int a = 0; a < 3; a++) {
    o->x[a] = o->alloc + (0 + a) * c;
    o->v[a] = o->alloc + (3 + a) * c;
    o->dx1[a] = o->alloc + (6 + a) * c;
    o->dx2[a] = o->alloc + (9 + a) * c;
    o->f[a] = o->alloc + (12 + a) * c;
  }
  o->id = o->alloc_id;
  o->orig = o->alloc_orig;
  o->cap = cap;
  return cudaSuccess;
}

cudaError_t order_bins(ParticleOrder* o, long long nbins) {
  if (o->nbins >= nbins) return cudaSuccess;
  release(o->cnt);
  release(o->bsum);
  o->nbins = 0;
  cudaError_t e = cudaMalloc(&o->cnt, sizeof(unsigned) * (size_t)nbins);
  if (e == cudaSuccess)
    e = cudaMalloc(&o->bsum, sizeof(unsigned) * (size_t)cgscan::scratch_entries(nbins));
  if (e != cudaSuccess) return e;
  o->nbins = nbins;
  return cudaSuccess;
}
}  // namespace

cudaError_t particle_order_reserve(ParticleOrder* o, long long cap) {
  cudaError_t e = cudaSuccess;
  if (!o->alloc) e = order_alloc(o, cap);
  else if (o->cap < cap) return cudaErrorInvalidValue;
  const long long nb = bins_per_side(cap);
  if (e == cudaSuccess) e = order_bins(o, nb * nb * nb);
  return e;
}

cudaError_t particles_sort_cells(ParticleSoA* s, ParticleOrder* o, float L, cudaStream_t st) {
  const long long n = s->n;
  if (n < 2 || !(L > 0.0f)) return cudaSuccess;
  if (n > 0x7fffffffLL || !s->orig) return cudaErrorInvalidValue;
  const int nb = bins_per_side(n);
  const long long nbins = (long long)nb * nb * nb;
  cudaError_t e = cudaSuccess;
  if (!o->alloc && (e = order_alloc(o, s->cap)) != cudaSuccess) return e;
  if (n > o->cap) return cudaErrorInvalidValue;
  if ((e = order_bins(o, nbins)) != cudaSuccess) return e;
  e = cudaMemsetAsync(o->cnt, 0, sizeof(unsigned) * (size_t)nbins, st);
  if (e != cudaSuccess) return e;
  const C3 x{{s->x[0], s->x[1], s->x[2]}};
  const float scale = (float)nb / L;
  prof_mark(st, CG_ST_SORT);
  unsigned* rank = o->key + o->cap;
  k_sort_bin<<<grid_for(n), T, 0, st>>>(x, n, scale, nb, o->key, rank, o->cnt);
  cgscan::exclusive(o->cnt, o->cnt, nbins, o->bsum, nullptr, CG_ST_SORT, st);
  const C3 v{{s->v[0], s->v[1], s->v[2]}};
  const C3 d1{{s->dx1[0], s->dx1[1], s->dx1[2]}};
  const C3 d2{{s->dx2[0], s->dx2[1], s->dx2[2]}};
  const C3 f{{s->f[0], s->f[1], s->f[2]}};
  const P3 fo{{o->f[0], o->f[1], o->f[2]}};
  const P3 xo{{o->x[0], o->x[1], o->x[2]}};
  const P3 vo{{o->v[0], o->v[1], o->v[2]}};
  const P3 d1o{{o->dx1[0], o->dx1[1], o->dx1[2]}};
  const P3 d2o{{o->dx2[0], o->dx2[1], o->dx2[2]}};
  prof_mark(st, CG_ST_SORT);
  k_sort_scatter<<<(unsigned)((n + T - 1) / T), T, 0, st>>>(x, v, d1, d2, f, s->id, s->orig, n,
                                                            o->key, rank,
                                                            o->cnt, xo, vo, d1o, d2o, fo, o->id,
                                                            o->orig);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // the sorted arrays become the working set; the old ones the scratch of
  // the next sort
  for (int a = 0; a < 3; a++) {
    float* t = s->x[a]; s->x[a] = o->x[a]; o->x[a] = t;
    t = s->v[a]; s->v[a] = o->v[a]; o->v[a] = t;
    t = s->dx1[a]; s->dx1[a] = o->dx1[a]; o->dx1[a] = t;
    t = s->dx2[a]; s->dx2[a] = o->dx2[a]; o->dx2[a] = t;
    t = s->f[a]; s->f[a] = o->f[a]; o->f[a] = t;
  }
  long long* ti = s->id; s->id = o->id; o->id = ti;
  int* to = s->orig; s->orig = o->orig; o->orig = to;
  return cudaSuccess;
}

cudaError_t particles_unsort_forces(ParticleSoA* s, ParticleOrder* o, cudaStream_t st) {
  if (s->n < 1 || !s->orig || !o->alloc) return cudaSuccess;
  const C3 f{{s->f[0], s->f[1], s->f[2]}};
  const P3 fo{{o->f[0], o->f[1], o->f[2]}};
  prof_mark(st, CG_ST_SORT);
  k_unsort_forces<<<grid_for(s->n), T, 0, st>>>(f, s->orig, s->n, fo);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  for (int a = 0; a < 3; a++) {
    float* t = s->f[a];
    s->f[a] = o->f[a];
    o->f[a] = t;
  }
  return cudaSuccess;
}
