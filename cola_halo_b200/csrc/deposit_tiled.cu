// Cell-sorted CIC deposit with shared-memory tile accumulation.
//
// The same contributions as PtoMesh (pm.c:209-276) plus the buffer copy of
// send_buffer_positions (pm.c:437-445) -- identical weights, float
// arithmetic and bounds -- but each mesh cell is written once, by the CTA
// that owns its 16^3 tile:
//   1. k_bin     key = home tile * 8 + boundary class of each particle; the
//                class bits say whether the particle's cloud reaches the
//                next tile in x, y, z.  Bin counts with warp-aggregated
//                atomics (one atomic per distinct key in a warp).
//   2. scan      exclusive prefix sum of the bin counts.
//   3. k_scatter particle positions into bin order (warp-aggregated slot
//                reservation).
//   4. k_tile    one CTA per tile gathers its own particles and the boundary
//                classes of its 7 lower neighbours, accumulates their
//                contributions inside the tile in shared memory (float
//                atomics), and stores delta = -1 + sum for all 4096 cells.
// No fill pass and no global atomics on the mesh.
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace {

constexpr int TS = 16;                 // tile edge (cells)
constexpr int TCELLS = TS * TS * TS;   // 4096
constexpr int T = CG_THREADS;
constexpr unsigned kInvalid = 0xFFFFFFFFu;

struct CicT {
  int i0, i1, j0, j1, k0, k1;
  float d1, d2, d3, t1, t2, t3;
  bool ok;
};

// pm.c:230-258 (same expressions as the atomic deposit)
__device__ __forceinline__ CicT cic_t(float px, float py, float pz, int N, float scale) {
  CicT c;
  const float X = __fmul_rn(px, scale);
  const float Y = __fmul_rn(py, scale);
  const float Z = __fmul_rn(pz, scale);
  c.ok = isfinite(X) && isfinite(Y) && isfinite(Z);
  const int iI = (int)floorf(X);
  int J = __float2int_rz(Y);
  int K = __float2int_rz(Z);
  c.d1 = __fsub_rn(X, (float)iI);
  c.d2 = __fsub_rn(Y, (float)J);
  c.d3 = __fsub_rn(Z, (float)K);
  c.t1 = __fsub_rn(1.0f, c.d1);
  c.t2 = __fsub_rn(1.0f, c.d2);
  c.t3 = __fsub_rn(1.0f, c.d3);
  if (J >= N) J = 0;
  if (K >= N) K = 0;
  if (J < 0 || K < 0) c.ok = false;
  c.i0 = iI;
  c.i1 = iI + 1;
  c.j0 = J;
  c.j1 = J + 1 >= N ? 0 : J + 1;
  c.k0 = K;
  c.k1 = K + 1 >= N ? 0 : K + 1;
  return c;
}

// Add the contributions of one CIC cloud that land in tile (ox, oy, oz).
__device__ __forceinline__ void add_in_tile(float* s, const CicT& c, int N, float wpar, int ox,
                                            int oy, int oz) {
  const float T2W = __fmul_rn(c.t2, wpar);
  const float D2W = __fmul_rn(c.d2, wpar);
  const int is[2] = {c.i0, c.i1};
  const float wx[2] = {c.t1, c.d1};
  const int js[2] = {c.j0, c.j1};
  const float wy[2] = {T2W, D2W};
  const int ks[2] = {c.k0, c.k1};
  const float wz[2] = {c.t3, c.d3};
#pragma unroll
  for (int a = 0; a < 2; a++) {
    const int i = is[a];
    if (i < 0 || i >= N) continue;
    const int li = i - ox;
    if (li < 0 || li >= TS) continue;
#pragma unroll
    for (int b = 0; b < 2; b++) {
      const int lj = js[b] - oy;
      if (lj < 0 || lj >= TS) continue;
#pragma unroll
      for (int d = 0; d < 2; d++) {
        const int lk = ks[d] - oz;
        if (lk < 0 || lk >= TS) continue;
        // weight (w_z * w_x) * w_y as in pm.c:264-275
        atomicAdd(s + (li * TS + lj) * TS + lk, __fmul_rn(__fmul_rn(wz[d], wx[a]), wy[b]));
      }
    }
  }
}

__device__ __forceinline__ unsigned key_of(float px, float py, float pz, int N, float scale,
                                           int NT) {
  const CicT c = cic_t(px, py, pz, N, scale);
  if (!c.ok) return kInvalid;
  // x = L exactly lands in cell N: only its buffer copy (cells 0, 1) counts
  const int cx = c.i0 >= N ? c.i0 - N : (c.i0 < 0 ? 0 : c.i0);
  const unsigned tile = ((unsigned)(cx / TS) * NT + c.j0 / TS) * NT + c.k0 / TS;
  const unsigned cls = ((cx % TS) == TS - 1 ? 1u : 0u) | ((c.j0 % TS) == TS - 1 ? 2u : 0u) |
                       ((c.k0 % TS) == TS - 1 ? 4u : 0u);
  return tile * 8u + cls;
}

// Warp-aggregated atomic add of 1 to counts[key]: lanes with the same key
// elect one leader; returns this lane's rank among them and the leader's
// old value through *base.
__device__ __forceinline__ unsigned agg_inc(unsigned* counts, unsigned key, unsigned active,
                                            unsigned* base) {
  const unsigned peers = __match_any_sync(active, key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  const unsigned rank = __popc(peers & ((1u << lane) - 1));
  unsigned b = 0;
  if (lane == leader) b = atomicAdd(counts + key, (unsigned)__popc(peers));
  *base = __shfl_sync(peers, b, leader);
  return rank;
}

__global__ void __launch_bounds__(T) k_bin(const float* __restrict__ x0,
                                           const float* __restrict__ x1,
                                           const float* __restrict__ x2, long long n, int N,
                                           float scale, int NT, unsigned* __restrict__ keys,
                                           unsigned* __restrict__ counts,
                                           unsigned* __restrict__ err) {
  const long long stride = (long long)gridDim.x * T;
  for (long long base = (long long)blockIdx.x * T; base < n; base += stride) {
    const long long i = base + threadIdx.x;
    const bool in = i < n;
    const unsigned active = __ballot_sync(0xffffffffu, in);
    if (!in) continue;
    const float px = x0[i], py = x1[i], pz = x2[i];
    const unsigned key = key_of(px, py, pz, N, scale, NT);
    keys[i] = key;
    if (key == kInvalid) {
      atomicOr(err, isfinite(px) && isfinite(py) && isfinite(pz) ? CG_ERR_BAD_CELL
                                                                  : CG_ERR_NONFINITE);
    }
    const unsigned valid = __ballot_sync(active, key != kInvalid);
    if (key != kInvalid) {
      unsigned b;
      agg_inc(counts, key, valid, &b);
    }
  }
}

__global__ void __launch_bounds__(T) k_scatter(const float* __restrict__ x0,
                                               const float* __restrict__ x1,
                                               const float* __restrict__ x2, long long n,
                                               const unsigned* __restrict__ keys,
                                               const unsigned* __restrict__ offsets,
                                               unsigned* __restrict__ cursor,
                                               float4* __restrict__ sorted) {
  const long long stride = (long long)gridDim.x * T;
  for (long long base = (long long)blockIdx.x * T; base < n; base += stride) {
    const long long i = base + threadIdx.x;
    const bool in = i < n;
    const unsigned active = __ballot_sync(0xffffffffu, in);
    if (!in) continue;
    const unsigned key = keys[i];
    const unsigned valid = __ballot_sync(active, key != kInvalid);
    if (key == kInvalid) continue;
    unsigned b;
    const unsigned rank = agg_inc(cursor, key, valid, &b);
    sorted[offsets[key] + b + rank] = make_float4(x0[i], x1[i], x2[i], 0.0f);
  }
}

// --------------------------------------------------------------- scan
constexpr int SCAN_B = 1024;   // elements per block (256 threads x 4)

__global__ void __launch_bounds__(256) k_scan_blocks(const unsigned* __restrict__ in,
                                                     unsigned* __restrict__ out, int n,
                                                     unsigned* __restrict__ block_sums) {
  __shared__ unsigned s[256];
  const int base = blockIdx.x * SCAN_B + threadIdx.x * 4;
  unsigned v[4], sum = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    v[q] = base + q < n ? in[base + q] : 0u;
    sum += v[q];
  }
  s[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 256; off <<= 1) {
    const unsigned t = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  unsigned run = s[threadIdx.x] - sum;   // exclusive prefix of this thread
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (base + q < n) out[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == 255) block_sums[blockIdx.x] = s[255];
}

__global__ void __launch_bounds__(1024) k_scan_sums(unsigned* __restrict__ sums, int nb) {
  __shared__ unsigned s[1024];
  unsigned carry = 0;
  for (int c0 = 0; c0 < nb; c0 += 1024) {
    const int i = c0 + threadIdx.x;
    const unsigned v = i < nb ? sums[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const unsigned t = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) sums[i] = carry + s[threadIdx.x] - v;
    const unsigned total = s[1023];
    __syncthreads();
    carry += total;
  }
}

__global__ void __launch_bounds__(256) k_scan_add(unsigned* __restrict__ out, int n,
                                                  const unsigned* __restrict__ block_sums) {
  const int base = blockIdx.x * SCAN_B + threadIdx.x * 4;
  const unsigned add = block_sums[blockIdx.x];
#pragma unroll
  for (int q = 0; q < 4; q++)
    if (base + q < n) out[base + q] += add;
}

// ------------------------------------------------------------ tile CTA
__global__ void __launch_bounds__(T) k_tile(const float4* __restrict__ sorted,
                                            const unsigned* __restrict__ offsets,
                                            const unsigned* __restrict__ counts, int N, int NT,
                                            float scale, float wpar, float x_right,
                                            float shiftx, float* __restrict__ dens) {
  __shared__ float s[TCELLS];
  const int tile = blockIdx.x;
  const int tx = tile / (NT * NT), ty = (tile / NT) % NT, tz = tile % NT;
  const int ox = tx * TS, oy = ty * TS, oz = tz * TS;
  for (int i = threadIdx.x; i < TCELLS; i += T) s[i] = 0.0f;
  __syncthreads();
  // own tile (all classes), then the lower neighbours' boundary classes
#pragma unroll 1
  for (int nb = 0; nb < 8; nb++) {
    const int ax = nb & 1, ay = (nb >> 1) & 1, az = (nb >> 2) & 1;
    const int ntx = ax ? (tx == 0 ? NT - 1 : tx - 1) : tx;
    const int nty = ay ? (ty == 0 ? NT - 1 : ty - 1) : ty;
    const int ntz = az ? (tz == 0 ? NT - 1 : tz - 1) : tz;
    const unsigned nt = ((unsigned)ntx * NT + nty) * NT + ntz;
#pragma unroll 1
    for (int cls = 0; cls < 8; cls++) {
      if ((cls & nb) != nb) continue;            // class must reach this tile
      const unsigned bin = nt * 8u + cls;
      const unsigned b0 = offsets[bin], b1 = b0 + counts[bin];
      for (unsigned p = b0 + threadIdx.x; p < b1; p += T) {
        const float4 q = sorted[p];
        const CicT c = cic_t(q.x, q.y, q.z, N, scale);
        add_in_tile(s, c, N, wpar, ox, oy, oz);
        if (q.x > x_right) {
          const CicT g = cic_t(__fadd_rn(q.x, shiftx), q.y, q.z, N, scale);
          if (g.ok) add_in_tile(s, g, N, wpar, ox, oy, oz);
        }
      }
    }
  }
  __syncthreads();
  // delta = -1 + sum  (pm.c:221-224); rows of 16 z cells are 64 B
  for (int i = threadIdx.x; i < TCELLS; i += T) {
    const int li = i / (TS * TS), lj = (i / TS) % TS, lk = i % TS;
    dens[((size_t)(ox + li) * N + (oy + lj)) * N + oz + lk] = __fadd_rn(-1.0f, s[i]);
  }
}

}  // namespace

cudaError_t pm_deposit_tiled(PmPlan* p, const float* const x[3], long long n, cudaStream_t st) {
  const int N = p->N;
  if (N % TS) return cudaErrorNotSupported;
  const int NT = N / TS;
  const long long ntiles = (long long)NT * NT * NT;
  const long long nbins = ntiles * 8;
  cudaError_t e;
  if (p->sort_cap < n || !p->bins) {
    // the sort buffers are sized on first use; a stream being captured into
    // a graph cannot allocate, so the caller takes the atomic deposit there
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
      return cudaErrorNotSupported;
    cudaFree(p->keys);
    cudaFree(p->sorted);
    p->keys = nullptr;
    p->sorted = nullptr;
    p->sort_cap = 0;
    if ((e = cudaMalloc(&p->keys, sizeof(unsigned) * (size_t)(n > 0 ? n : 1))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p->sorted, sizeof(float4) * (size_t)(n > 0 ? n : 1))) != cudaSuccess) return e;
    if (!p->bins) {
      const long long nblk = (nbins + SCAN_B - 1) / SCAN_B;
      if ((e = cudaMalloc(&p->bins, sizeof(unsigned) * (size_t)(3 * nbins + nblk))) != cudaSuccess)
        return e;
    }
    p->sort_cap = n;
  }
  unsigned* counts = p->bins;
  unsigned* offsets = p->bins + nbins;
  unsigned* cursor = p->bins + 2 * nbins;
  unsigned* bsums = p->bins + 3 * nbins;
  const int nblk = (int)((nbins + SCAN_B - 1) / SCAN_B);
  cudaMemsetAsync(counts, 0, sizeof(unsigned) * nbins, st);
  cudaMemsetAsync(cursor, 0, sizeof(unsigned) * nbins, st);
  if (n > 0) {
    prof_mark(st, CG_ST_DEPOSIT);
    k_bin<<<grid_for(n), T, 0, st>>>(x[0], x[1], x[2], n, N, p->scale, NT, p->keys, counts, p->err);
  }
  prof_mark(st, CG_ST_DEPOSIT);
  k_scan_blocks<<<nblk, 256, 0, st>>>(counts, offsets, (int)nbins, bsums);
  prof_mark(st, CG_ST_DEPOSIT);
  k_scan_sums<<<1, 1024, 0, st>>>(bsums, nblk);
  prof_mark(st, CG_ST_DEPOSIT);
  k_scan_add<<<nblk, 256, 0, st>>>(offsets, (int)nbins, bsums);
  if (n > 0) {
    prof_mark(st, CG_ST_DEPOSIT);
    k_scatter<<<grid_for(n), T, 0, st>>>(x[0], x[1], x[2], n, p->keys, offsets, cursor, p->sorted);
  }
  prof_mark(st, CG_ST_DEPOSIT);
  k_tile<<<(unsigned)ntiles, T, 0, st>>>(p->sorted, offsets, counts, N, NT, p->scale, p->wpar,
                                         p->x_right, p->shiftx, p->dens);
  return cudaGetLastError();
}
