// Particle-mesh force on one B200: CIC deposit, 3-D r2c, Green's function /
// spectral gradient, three 3-D c2r, CIC interpolation.
//
// Reference: pm.c:209-412 (PtoMesh, compute_density_k, compute_force_mesh,
// force_at_particle_locations) and pm.c:416-532 (buffer particles), on one
// process.  The x-direction periodicity that the reference obtains from
// buffer particles is restated exactly: a particle with x > x_right also
// acts through a copy at x - L, with that copy's own CIC weights.
//
// Mesh layouts in HBM
//   real   R[x][y][z]        N^3 floats, z contiguous, no padding
//   half   S[kz][kx][ky]     (N/2+1) N N complex floats, ky contiguous
// Transform passes of the force (each one read + one write of a mesh):
//   FZ     r2c along z of R, transposed store into S      (+ density sum)
//   FX     forward c2c along kx (stride N), in place
//   GREEN  forward c2c along ky (contiguous lines), Green/gradient, inverse
//          c2c along ky -> the y spectrum and the shared x/z spectrum
//          (one read, two writes)
//   FX     inverse c2c along kx per component (x and z scale the shared
//          spectrum by n_x / n_z as they load it)
//   ZI     c2r along z of G_a, transposed load, store R_a
// The plain 3-D transforms (mesh_r2c / mesh_c2r) run FZ, FY, FX and back.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <type_traits>
#include <vector>
#include <mutex>

#include "fft_core.cuh"
#include "internal.h"
#include "scan.cuh"

using cgfft::cplx;

// TMA maps of the x pass for tk columns per CTA (encoded on demand).
bool x_maps_for(PmPlan* p, int tk);

namespace {

constexpr int T = CG_THREADS;
constexpr int TY = 16;   // z-lines per CTA in FZ / ZI
constexpr int BY = 8;    // y-lines per CTA in FY

// ------------------------------------------------------------------ fill
__global__ void k_fill(float4* __restrict__ p, size_t n4, float v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < n4; i += stride) p[i] = make_float4(v, v, v, v);
}

// ------------------------------------------------------------ CIC index
// pm.c:230-258: cell and weights of one position (float arithmetic, no FMA).
struct Cic {
  int i0, i1, j0, j1, k0, k1;
  float d1, d2, d3, t1, t2, t3;
  bool ok;
};

__device__ __forceinline__ Cic cic_index(float px, float py, float pz, int N, float scale) {
  Cic c;
  const float X = __fmul_rn(px, scale);
  const float Y = __fmul_rn(py, scale);
  const float Z = __fmul_rn(pz, scale);
  c.ok = isfinite(X) && isfinite(Y) && isfinite(Z);
  int iI = (int)floorf(X);
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
  if (J < 0 || K < 0) c.ok = false;   // the reference assumes y, z >= 0
  c.i0 = iI;
  c.i1 = iI + 1;
  c.j0 = J;
  c.j1 = J + 1 >= N ? 0 : J + 1;
  c.k0 = K;
  c.k1 = K + 1 >= N ? 0 : K + 1;
  return c;
}

__device__ __forceinline__ size_t cell(int i, int j, int k, int N) {
  return ((size_t)i * N + j) * N + k;
}

// The two z cells k0, k1 of one (x, y) column of the cloud.  When they lie
// in one 16-byte-aligned group of four floats they take a single float4
// atomic (zeros in the other two lanes leave those cells unchanged); else
// (k0 = 3 mod 4, or k1 wrapped to 0) two scalar atomics.  `col` is the
// cell (i, j, 0): a multiple of 4 floats since N is.
__device__ __forceinline__ void add_z_pair(float* __restrict__ d, size_t col, int k0, int k1,
                                           float w0, float w1) {
  const int q = k0 & 3;
  if (k1 == k0 + 1 && q != 3) {
    float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (q == 0) { v.x = w0; v.y = w1; }
    else if (q == 1) { v.y = w0; v.z = w1; }
    else { v.z = w0; v.w = w1; }
    atomicAdd(reinterpret_cast<float4*>(d + col + (k0 - q)), v);
  } else {
    atomicAdd(d + col + k0, w0);
    atomicAdd(d + col + k1, w1);
  }
}

__device__ __forceinline__ void deposit_one(float* __restrict__ d, const Cic& c, int N,
                                            float wpar) {
  const float T2W = __fmul_rn(c.t2, wpar);
  const float D2W = __fmul_rn(c.d2, wpar);
  if (0 <= c.i0 && c.i0 < N) {
    add_z_pair(d, cell(c.i0, c.j0, 0, N), c.k0, c.k1, __fmul_rn(__fmul_rn(c.t3, c.t1), T2W),
               __fmul_rn(__fmul_rn(c.d3, c.t1), T2W));
    add_z_pair(d, cell(c.i0, c.j1, 0, N), c.k0, c.k1, __fmul_rn(__fmul_rn(c.t3, c.t1), D2W),
               __fmul_rn(__fmul_rn(c.d3, c.t1), D2W));
  }
  if (0 <= c.i1 && c.i1 < N) {
    add_z_pair(d, cell(c.i1, c.j0, 0, N), c.k0, c.k1, __fmul_rn(__fmul_rn(c.t3, c.d1), T2W),
               __fmul_rn(__fmul_rn(c.d3, c.d1), T2W));
    add_z_pair(d, cell(c.i1, c.j1, 0, N), c.k0, c.k1, __fmul_rn(__fmul_rn(c.t3, c.d1), D2W),
               __fmul_rn(__fmul_rn(c.d3, c.d1), D2W));
  }
}

// PtoMesh (pm.c:229-276) incl. the buffer copy of send_buffer_positions
// (pm.c:437-445, 477-481).  The mesh holds -1 on entry (pm.c:221-224).
__global__ void __launch_bounds__(T) k_deposit(const float* __restrict__ x0,
                                               const float* __restrict__ x1,
                                               const float* __restrict__ x2, long long n,
                                               float* __restrict__ dens, int N, float scale,
                                               float wpar, float x_right, float shiftx,
                                               unsigned* __restrict__ err) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    const float px = x0[i], py = x1[i], pz = x2[i];
    Cic c = cic_index(px, py, pz, N, scale);
    if (!c.ok) {
      atomicOr(err, isfinite(px) && isfinite(py) && isfinite(pz) ? CG_ERR_BAD_CELL
                                                                  : CG_ERR_NONFINITE);
      continue;
    }
    deposit_one(dens, c, N, wpar);
    if (px > x_right) {
      Cic g = cic_index(__fadd_rn(px, shiftx), py, pz, N, scale);
      if (g.ok) deposit_one(dens, g, N, wpar);
    }
  }
}

// The same deposit for a chunk of CHUNK consecutive particles per CTA,
// accumulated first in a shared-memory copy of the chunk's bounding box of
// cells when that box is small.  In cell order (reorder.cu) the particles
// of a halo sit next to each other, so a warp's eight CIC corners hit the
// same few cells: global float atomics on one address serialise in L2,
// shared-memory ones are cheap, and the box is then added to the mesh with
// one atomic per touched cell.  The weights are deposit_one's products, so
// only the order of the float additions changes.  Particles whose cloud
// wraps in y or z, leaves the mesh in x, or has a buffer copy (x > x_right)
// take the global path, as does every particle of a CTA whose box is large.
// Shapes of the box deposit (particles per CTA, box cells of shared memory),
// a schedule parameter per mesh size chosen by cg_sim_tune_deposit on the
// particles of a run (variant 0 by default); chunk 0: every cloud takes the
// global atomics (k_deposit).
struct DepCfg { int chunk, vmax; };
constexpr DepCfg kDepCfg[PM_NUM_DEP_VARIANTS] = {
    {512, 3072}, {256, 3072}, {1024, 6144}, {2048, 12288}, {512, 6144}, {0, 0}};

__device__ __forceinline__ void deposit_one_box(float* __restrict__ box, const Cic& c, int bx,
                                                int by, int bz, int ny, int nz, float wpar) {
  const float T2W = __fmul_rn(c.t2, wpar);
  const float D2W = __fmul_rn(c.d2, wpar);
  const int i0 = c.i0 - bx, j0 = c.j0 - by, k0 = c.k0 - bz;
  float* r00 = box + ((i0 * ny) + j0) * nz + k0;          // (i0, j0)
  float* r01 = r00 + nz;                                   // (i0, j1)
  float* r10 = r00 + ny * nz;                              // (i1, j0)
  float* r11 = r10 + nz;                                   // (i1, j1)
  atomicAdd(r00, __fmul_rn(__fmul_rn(c.t3, c.t1), T2W));
  atomicAdd(r00 + 1, __fmul_rn(__fmul_rn(c.d3, c.t1), T2W));
  atomicAdd(r01, __fmul_rn(__fmul_rn(c.t3, c.t1), D2W));
  atomicAdd(r01 + 1, __fmul_rn(__fmul_rn(c.d3, c.t1), D2W));
  atomicAdd(r10, __fmul_rn(__fmul_rn(c.t3, c.d1), T2W));
  atomicAdd(r10 + 1, __fmul_rn(__fmul_rn(c.d3, c.d1), T2W));
  atomicAdd(r11, __fmul_rn(__fmul_rn(c.t3, c.d1), D2W));
  atomicAdd(r11 + 1, __fmul_rn(__fmul_rn(c.d3, c.d1), D2W));
}

__device__ __forceinline__ bool box_eligible(const Cic& c, float px, float x_right, int N) {
  return c.ok && !(px > x_right) && c.i0 >= 0 && c.i1 < N && c.j1 == c.j0 + 1 &&
         c.k1 == c.k0 + 1;
}

template <int CHUNK, int VMAX>
__global__ void __launch_bounds__(T) k_deposit_box(const float* __restrict__ x0,
                                                   const float* __restrict__ x1,
                                                   const float* __restrict__ x2, long long n,
                                                   float* __restrict__ dens, int N, float scale,
                                                   float wpar, float x_right, float shiftx,
                                                   unsigned* __restrict__ err) {
  extern __shared__ float box[];                  // VMAX cells
  __shared__ int red[6][T / 32];
  const long long base = (long long)blockIdx.x * CHUNK;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // bounding box of the eligible clouds' lower corners
  int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff};
  int hi[3] = {-1, -1, -1};
  for (int q = 0; q < CHUNK / T; q++) {
    const long long i = base + q * T + tid;
    if (i >= n) break;
    const float px = x0[i];
    const Cic c = cic_index(px, x1[i], x2[i], N, scale);
    if (!box_eligible(c, px, x_right, N)) continue;
    lo[0] = min(lo[0], c.i0); hi[0] = max(hi[0], c.i0);
    lo[1] = min(lo[1], c.j0); hi[1] = max(hi[1], c.j0);
    lo[2] = min(lo[2], c.k0); hi[2] = max(hi[2], c.k0);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
    if (lane == 0) {
      red[a][warp] = lo[a];
      red[3 + a][warp] = hi[a];
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 3; a++) {
    lo[a] = red[a][0];
    hi[a] = red[3 + a][0];
    for (int w = 1; w < T / 32; w++) {
      lo[a] = min(lo[a], red[a][w]);
      hi[a] = max(hi[a], red[3 + a][w]);
    }
  }
  // cells lo .. hi + 1 per axis
  const long long nx = (long long)hi[0] - lo[0] + 2, ny = (long long)hi[1] - lo[1] + 2,
                  nz = (long long)hi[2] - lo[2] + 2;
  const bool use_box = hi[0] >= 0 && nx * ny * nz <= VMAX;
  const int vol = use_box ? (int)(nx * ny * nz) : 0;
  for (int v = tid; v < vol; v += T) box[v] = 0.0f;
  __syncthreads();
  for (int q = 0; q < CHUNK / T; q++) {
    const long long i = base + q * T + tid;
    if (i >= n) break;
    const float px = x0[i], py = x1[i], pz = x2[i];
    const Cic c = cic_index(px, py, pz, N, scale);
    if (!c.ok) {
      atomicOr(err, isfinite(px) && isfinite(py) && isfinite(pz) ? CG_ERR_BAD_CELL
                                                                  : CG_ERR_NONFINITE);
      continue;
    }
    if (use_box && box_eligible(c, px, x_right, N)) {
      deposit_one_box(box, c, lo[0], lo[1], lo[2], (int)ny, (int)nz, wpar);
      continue;
    }
    deposit_one(dens, c, N, wpar);
    if (px > x_right) {
      Cic g = cic_index(__fadd_rn(px, shiftx), py, pz, N, scale);
      if (g.ok) deposit_one(dens, g, N, wpar);
    }
  }
  __syncthreads();
  if (!use_box) return;
  // flush: one 16-byte atomic per touched group of four z cells, aligned in
  // the mesh (N is a multiple of 4, and every box cell lies inside the mesh:
  // eligible clouds neither wrap nor leave it)
  const int q0 = lo[2] >> 2;
  const int nq = ((lo[2] + (int)nz - 1) >> 2) - q0 + 1;
  const int nvec = (int)(nx * ny) * nq;
  for (int v = tid; v < nvec; v += T) {
    const int q = v % nq, jj = (v / nq) % (int)ny, ii = v / (nq * (int)ny);
    const int k0 = 4 * (q0 + q) - lo[2];          // box z index of the group's first cell
    const float* row = box + (ii * (int)ny + jj) * (int)nz;
    float4 w;
    w.x = (k0 >= 0 && k0 < nz) ? row[k0] : 0.0f;
    w.y = (k0 + 1 >= 0 && k0 + 1 < nz) ? row[k0 + 1] : 0.0f;
    w.z = (k0 + 2 >= 0 && k0 + 2 < nz) ? row[k0 + 2] : 0.0f;
    w.w = (k0 + 3 >= 0 && k0 + 3 < nz) ? row[k0 + 3] : 0.0f;
    if (w.x == 0.0f && w.y == 0.0f && w.z == 0.0f && w.w == 0.0f) continue;
    atomicAdd(reinterpret_cast<float4*>(dens + cell(lo[0] + ii, lo[1] + jj, 4 * (q0 + q), N)), w);
  }
}

// force_at_particle_locations (pm.c:370-411) for all three axes, plus the
// buffer copy's force added back as in add_buffer_forces (pm.c:526-531).
__device__ __forceinline__ float gather4(const float* __restrict__ m, int i, const Cic& c,
                                         int N, float wi) {
  // ((m*T3)*Ti)*T2 + ((m*D3)*Ti)*T2 + ((m*T3)*Ti)*D2 + ((m*D3)*Ti)*D2
  float a = __fmul_rn(__fmul_rn(__fmul_rn(__ldg(m + cell(i, c.j0, c.k0, N)), c.t3), wi), c.t2);
  float b = __fmul_rn(__fmul_rn(__fmul_rn(__ldg(m + cell(i, c.j0, c.k1, N)), c.d3), wi), c.t2);
  float d = __fmul_rn(__fmul_rn(__fmul_rn(__ldg(m + cell(i, c.j1, c.k0, N)), c.t3), wi), c.d2);
  float e = __fmul_rn(__fmul_rn(__fmul_rn(__ldg(m + cell(i, c.j1, c.k1, N)), c.d3), wi), c.d2);
  return __fadd_rn(__fadd_rn(__fadd_rn(a, b), d), e);
}

// Planes lo <= i < hi take part (the whole mesh: 0, N; a slab of a
// decomposed mesh: its own planes, pm.c:379-405's local_nx test).
__device__ __forceinline__ float interp_one(const float* __restrict__ m, const Cic& c, int N,
                                            int lo, int hi) {
  float f = 0.0f;
  if (lo <= c.i0 && c.i0 < hi) f = __fadd_rn(f, gather4(m, c.i0, c, N, c.t1));
  if (lo <= c.i1 && c.i1 < hi) f = __fadd_rn(f, gather4(m, c.i1, c, N, c.d1));
  return f;
}

// Grid of the interpolation: 5 CTAs per SM of grid-stride threads, so that
// the particles in flight at any time are a window of about 190k (about 3
// particle planes of a 256^3 lattice order).  The mesh planes they gather
// from, for the three force meshes, then stay in L2 (768^3: about 70 MB
// against 126 MB): 0.92-0.95 ms per step against 1.15 ms with 16 CTAs per
// SM, whose 600k-particle window reached about 200 MB of planes.  3 CTAs per
// SM leave too few warps in flight (1.12 ms).
constexpr int kInterpCtasPerSm = 5;

__global__ void __launch_bounds__(T) k_interp(const float* __restrict__ x0,
                                              const float* __restrict__ x1,
                                              const float* __restrict__ x2, long long n,
                                              const float* __restrict__ m0,
                                              const float* __restrict__ m1,
                                              const float* __restrict__ m2,
                                              float* __restrict__ f0, float* __restrict__ f1,
                                              float* __restrict__ f2, int N, float scale,
                                              float x_right, float shiftx, int xlo, int xhi) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    const float px = x0[i], py = x1[i], pz = x2[i];
    Cic c = cic_index(px, py, pz, N, scale);
    float a = 0.0f, b = 0.0f, d = 0.0f;
    if (c.ok) {
      a = interp_one(m0, c, N, xlo, xhi);
      b = interp_one(m1, c, N, xlo, xhi);
      d = interp_one(m2, c, N, xlo, xhi);
      if (px > x_right) {
        Cic g = cic_index(__fadd_rn(px, shiftx), py, pz, N, scale);
        if (g.ok) {
          a = __fadd_rn(a, interp_one(m0, g, N, xlo, xhi));
          b = __fadd_rn(b, interp_one(m1, g, N, xlo, xhi));
          d = __fadd_rn(d, interp_one(m2, g, N, xlo, xhi));
        }
      }
    }
    f0[i] = a;
    f1[i] = b;
    f2[i] = d;
  }
}

// ------------------------------------------------------------ FFT passes
// Every pass: a CTA owns a tile of complete lines; the first radix stage
// loads its legs straight from HBM, the last stage stores straight to HBM,
// and only the exchanges between stages use the padded shared tile
// (fft_core.cuh).
using cgfft::Gmem;
using cgfft::SmemCol;
using cgfft::SmemLine;

// Schedules of the strided x pass and the fused y Green pass.  Variant 0
// is the default; the others are compiled for meshes from MIN_TUNED_N up
// and chosen per mesh size by the autotuner (pm_autotune) or set
// explicitly.  x pass: ky columns per CTA and maximum radix (0: radix 8
// from 768 up, else 16; -1: the other of the two).  Green pass: lines per
// CTA, maximum radix and the resident CTAs per SM the kernel is
// register-limited to.  The Green default is the fastest shape measured at
// 384 and 768; for the x pass the tuner picks 16 columns (variant 2) there,
// ahead of the 8-column default.
constexpr int MIN_TUNED_N = 256;
// Variants compiled at size N.  The 8-line Green variants stop at 768: at
// 1024 they would spill registers.
__host__ __device__ constexpr int n_fx_variants(int N) {
  return N >= MIN_TUNED_N ? PM_NUM_FX_VARIANTS : 1;
}
__host__ __device__ constexpr int n_green_variants(int N) {
  return N >= MIN_TUNED_N && N <= 768 ? PM_NUM_GREEN_VARIANTS : 1;
}
struct FxCfg { int tk, rm; };
struct GreenCfg { int byg, rm, minb, thr; };
constexpr FxCfg kFxCfg[PM_NUM_FX_VARIANTS] = {{8, 0}, {8, -1}, {16, 16}};
// (lines per CTA, maximum radix, CTAs per SM, threads): at 768 a radix-16
// stage has 48 butterflies per line, so 8 lines fill 384 threads, 4 lines
// 192 and 2 lines 96 once each; 2 lines on 128 threads split the radix-3
// stage's 512 butterflies evenly.  The default, 2 lines on 128 threads at 7
// CTAs per SM, keeps a barrier to 4 warps (768^3: 1.39 ms; 4 lines on 256
// threads, the earlier default: 1.64 ms; 2 lines on 96 threads: 1.62 ms; 2
// on 128 at 8 or 6 CTAs per SM: 1.41 and 1.42 ms).
constexpr GreenCfg kGreenCfg[PM_NUM_GREEN_VARIANTS] = {
    {2, 16, 7, 128}, {8, 8, 2, 256}, {8, 16, 2, 384}, {4, 16, 4, 192}, {2, 16, 8, 96},
    {2, 16, 8, 128}, {4, 16, 3, 256}};
__host__ __device__ constexpr int rm_x_default(int N) { return N >= 768 ? 8 : 16; }
__host__ __device__ constexpr int fx_rm(int N, int v) {
  return kFxCfg[v].rm == 0 ? rm_x_default(N)
                           : (kFxCfg[v].rm < 0 ? 24 - rm_x_default(N) : kFxCfg[v].rm);
}

// FZ: r2c along z of R (TY z-lines (x, y0..y0+TY-1) per CTA) through a
// complex FFT of length H = N/2 on (x_2m + i x_2m+1):
//   X_k = E_k + W_N^k O_k,  E_k = (Z_k + conj Z_{H-k})/2,
//   O_k = -i (Z_k - conj Z_{H-k})/2,            k = 0..H
// stored transposed into S[kz][x][y].  The sum of the mesh
// (check_total_density, pm.c:535-562) is the sum over lines of
// Re Z_0 + Im Z_0, accumulated in double.
// RESET: once its lines are in shared memory, the CTA writes them back as
// -1, the value the next deposit starts from, so that no fill pass is needed.
// The RESET form writes the mesh it reads, so its pointer is neither const
// nor __restrict__ there.
template <bool RESET> using DensPtr = typename std::conditional<RESET, float*, const float*>::type;

// The split of k_fz (after the H-point transform of the TY lines in `mid`):
// X_k for k = 0..H stored transposed into S[kz][x][y0 + b], and the lines'
// sum Re Z_0 + Im Z_0 added to *dsum in double.
template <int N>
__device__ __forceinline__ void fz_split_store(const SmemLine<cgfft::line_pitch<N / 2>()>& mid,
                                               int x, int y0, float2* __restrict__ spec,
                                               const float2* __restrict__ twN,
                                               double* __restrict__ dsum) {
  constexpr int H = N / 2;
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < (H + 1) * TY; idx += T) {
    const int b = idx % TY, k = idx / TY;
    const cplx zk = mid.ld(b, k == H ? 0 : k);
    const cplx zc0 = mid.ld(b, k == 0 ? 0 : H - k);
    const cplx zc = {zc0.x, -zc0.y};
    const cplx e = {0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y)};
    const cplx dlt = {zk.x - zc.x, zk.y - zc.y};
    const cplx o = {0.5f * dlt.y, -0.5f * dlt.x};
    const float2 w = __ldg(twN + k);
    const cplx X = {e.x + (w.x * o.x - w.y * o.y), e.y + (w.x * o.y + w.y * o.x)};
    if (k == 0) acc += (double)zk.x + (double)zk.y;
    spec[((size_t)k * N + x) * N + y0 + b] = make_float2(X.x, X.y);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(dsum, acc);
}

template <int N, bool RESET>
__global__ void __launch_bounds__(T) k_fz(DensPtr<RESET> dens,
                                          float2* __restrict__ spec,
                                          const float2* __restrict__ twH,
                                          const float2* __restrict__ twN,
                                          double* __restrict__ dsum) {
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  const SmemLine<cgfft::line_pitch<H>()> mid{reinterpret_cast<cplx*>(smraw)};
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * TY;
  const cgfft::GmemC<H, 1> gin{reinterpret_cast<float2*>(const_cast<float*>(dens)) +
                              ((size_t)x * N + y0) * H};
  cgfft::fft_io<H, TY, T, true, -1>(gin, mid, mid, twH);
  if constexpr (RESET) {
    __syncthreads();    // every thread's loads of the lines are done
    float4* line = reinterpret_cast<float4*>(dens + ((size_t)x * N + y0) * N);
    for (int i = threadIdx.x; i < TY * N / 4; i += T) line[i] = make_float4(-1.f, -1.f, -1.f, -1.f);
  }
  fz_split_store<N>(mid, x, y0, spec, twN, dsum);
}

// ------------------------------------------------- column-binned deposit
// The force step's deposit and r2c along z in one pass (k_dfz): a CTA of
// the z transform builds its own TY density lines (x, y0 .. y0+TY-1) in
// shared memory from the particles whose clouds reach them, transforms them
// and stores the spectrum, so the density mesh is never written to or read
// from HBM.  For that the clouds are binned by their lower-corner column
// (i0, j0) every force step (k_col_count, a prefix sum, k_col_scatter):
//   key = (i0 + 1) N + j0,   i0 in [-1, N-1] (the buffer copy of a particle
//                            with x > x_right has i0 = -1), j0 in [0, N-1]
// and each cloud becomes one 16-byte entry (x, y, z, particle index) at
// start[key] + its rank among the key's arrivals (x is the buffer copy's
// x - L for the copy, flagged by bit 31 of the index).  A cloud with i0
// outside [-1, N-1] deposits nothing (as in k_deposit) and gets no entry.
constexpr unsigned COL_NONE = 0xffffffffu;
constexpr unsigned COL_COPY = 0x80000000u;

__device__ __forceinline__ unsigned col_key(const Cic& c, int N) {
  return c.ok && c.i0 >= -1 && c.i0 <= N - 1 ? (unsigned)((c.i0 + 1) * N + c.j0) : COL_NONE;
}

// Rank of this lane's key among the warp's lanes with the same key, after
// the ranks the key already holds: one atomic per distinct key of the warp
// (warp-aggregated).  Every lane of the warp calls it; COL_NONE takes no rank.
__device__ __forceinline__ unsigned warp_rank(unsigned* __restrict__ cnt, unsigned key,
                                              int lane) {
  const unsigned m = __match_any_sync(0xffffffffu, key);
  const int leader = __ffs(m) - 1;
  unsigned b = 0;
  if (lane == leader && key != COL_NONE) b = atomicAdd(cnt + key, (unsigned)__popc(m));
  b = __shfl_sync(0xffffffffu, b, leader);
  return b + (unsigned)__popc(m & ((1u << lane) - 1u));
}

// Counts per key; rank[i] (primary cloud) and rank[cap + i] (buffer copy).
__global__ void __launch_bounds__(T) k_col_count(const float* __restrict__ x0,
                                                 const float* __restrict__ x1,
                                                 const float* __restrict__ x2, long long n,
                                                 int N, float scale, float x_right, float shiftx,
                                                 unsigned* __restrict__ cnt,
                                                 unsigned* __restrict__ rank, long long cap,
                                                 unsigned* __restrict__ err,
                                                 float* __restrict__ f0, float* __restrict__ f1,
                                                 float* __restrict__ f2) {
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * T;
  // warp-uniform trip count: every lane takes part in the warp's match
  for (long long base = (long long)blockIdx.x * T + (threadIdx.x & ~31); base < n;
       base += stride) {
    const long long i = base + lane;
    unsigned k0 = COL_NONE, k1 = COL_NONE;
    if (i < n) {
      const float px = x0[i], py = x1[i], pz = x2[i];
      const Cic c = cic_index(px, py, pz, N, scale);
      if (!c.ok) {
        atomicOr(err, isfinite(px) && isfinite(py) && isfinite(pz) ? CG_ERR_BAD_CELL
                                                                    : CG_ERR_NONFINITE);
      } else {
        k0 = col_key(c, N);
        if (px > x_right) k1 = col_key(cic_index(__fadd_rn(px, shiftx), py, pz, N, scale), N);
      }
    }
    const unsigned r0 = warp_rank(cnt, k0, lane);
    if (k0 != COL_NONE) rank[i] = r0;
    // the interpolation from the bins writes the forces of the primary
    // clouds only; a particle without one (its cell index not finite or x
    // rounded to L) has the force 0 of interp_one, plus its buffer copy's
    if (f0 && k0 == COL_NONE && i < n) f0[i] = f1[i] = f2[i] = 0.0f;
    if (__any_sync(0xffffffffu, k1 != COL_NONE)) {
      const unsigned r1 = warp_rank(cnt, k1, lane);
      if (k1 != COL_NONE) {
        rank[cap + i] = r1;
        // a copy outside key row 0 (x = L exactly after the wrap, or a
        // position never wrapped): counted past the keys, so that the
        // interpolation's copy pass looks at every entry
        if (k1 >= (unsigned)N) atomicAdd(cnt + (size_t)(N + 1) * N + 1, 1u);
      }
    }
  }
}

// Entries at start[key] + rank (cnt now holds the exclusive prefix sums).
__global__ void __launch_bounds__(T) k_col_scatter(const float* __restrict__ x0,
                                                   const float* __restrict__ x1,
                                                   const float* __restrict__ x2, long long n,
                                                   int N, float scale, float x_right,
                                                   float shiftx,
                                                   const unsigned* __restrict__ start,
                                                   const unsigned* __restrict__ rank,
                                                   long long cap, float4* __restrict__ ent) {
  long long i = (long long)blockIdx.x * T + threadIdx.x;
  const long long stride = (long long)gridDim.x * T;
  for (; i < n; i += stride) {
    const float px = x0[i], py = x1[i], pz = x2[i];
    const Cic c = cic_index(px, py, pz, N, scale);
    if (!c.ok) continue;
    const unsigned k0 = col_key(c, N);
    if (k0 != COL_NONE)
      ent[start[k0] + rank[i]] = make_float4(px, py, pz, __uint_as_float((unsigned)i));
    if (px > x_right) {
      const float qx = __fadd_rn(px, shiftx);
      const unsigned k1 = col_key(cic_index(qx, py, pz, N, scale), N);
      if (k1 != COL_NONE)
        ent[start[k1] + rank[cap + i]] =
            make_float4(qx, py, pz, __uint_as_float((unsigned)i | COL_COPY));
    }
  }
}

// The entry ranges of the clouds that reach the lines (x, y0 .. y0+TY-1):
// key rows x (i0 = x - 1) and x + 1 (i0 = x), columns y0 - 1 (mod N) ..
// y0 + TY - 1.  For y0 > 0 (or TY = N) the columns of one row are one run
// of keys; for y0 = 0 the wrapped column N - 1 is a second run.  Four
// (lo, hi) key pairs (an empty run is (0, 0)); range q holds entries
// start[lo_q] .. start[hi_q] - 1.
__device__ __forceinline__ void col_range_keys(int N, int x, int y0, int ty, unsigned (&k)[8]) {
  const unsigned r0 = (unsigned)x * N, r1 = r0 + N;
  if (y0 > 0 || ty == N) {
    const unsigned lo = y0 > 0 ? y0 - 1 : 0, hi = y0 + ty;
    k[0] = r0 + lo; k[1] = r0 + hi; k[2] = r1 + lo; k[3] = r1 + hi;
    k[4] = k[5] = k[6] = k[7] = 0;
  } else {
    k[0] = r0; k[1] = r0 + ty; k[2] = r0 + N - 1; k[3] = r0 + N;
    k[4] = r1; k[5] = r1 + ty; k[6] = r1 + N - 1; k[7] = r1 + N;
  }
}

// One cloud's contributions to the plane x lines of the tile.
template <int PH>
__device__ __forceinline__ void dfz_add(float* __restrict__ tf, const float4& w, int N, int x,
                                        int y0, float scale, float wpar) {
  const Cic c = cic_index(w.x, w.y, w.z, N, scale);
  const float wx = c.i0 == x ? c.t1 : c.d1;
  const float T2W = __fmul_rn(c.t2, wpar);
  const float D2W = __fmul_rn(c.d2, wpar);
  const int f0 = 2 * ((c.k0 >> 1) + (c.k0 >> 5)) + (c.k0 & 1);
  const int f1 = 2 * ((c.k1 >> 1) + (c.k1 >> 5)) + (c.k1 & 1);
  const unsigned b0 = (unsigned)(c.j0 - y0), b1 = (unsigned)(c.j1 - y0);
  if (b0 < (unsigned)TY) {
    float* row = tf + 2 * PH * (int)b0;
    atomicAdd(row + f0, __fmul_rn(__fmul_rn(c.t3, wx), T2W));
    atomicAdd(row + f1, __fmul_rn(__fmul_rn(c.d3, wx), T2W));
  }
  if (b1 < (unsigned)TY) {
    float* row = tf + 2 * PH * (int)b1;
    atomicAdd(row + f0, __fmul_rn(__fmul_rn(c.t3, wx), D2W));
    atomicAdd(row + f1, __fmul_rn(__fmul_rn(c.d3, wx), D2W));
  }
}

// Entries per thread loaded before any is deposited (loads in flight).
constexpr int DFZ_U = 4;

// DFZ: PtoMesh (pm.c:229-276, the buffer copy of pm.c:437-445 included)
// restricted to the TY z-lines (x, y0 .. y0+TY-1), accumulated in shared
// memory on -1 (pm.c:221-224) with deposit_one's weight products, then
// k_fz's r2c along z from the shared tile.  Only the order of the float
// additions differs from the global deposit.  Cell z of line b sits in
// complex element z / 2 (real part for even z) of the transform's tile.
template <int N, int MINB>
__global__ void __launch_bounds__(T, MINB) k_dfz(const float4* __restrict__ ent,
                                                 const unsigned* __restrict__ start,
                                                 float2* __restrict__ spec,
                                                 const float2* __restrict__ twH,
                                                 const float2* __restrict__ twN,
                                                 double* __restrict__ dsum, float scale,
                                                 float wpar) {
  constexpr int H = N / 2;
  constexpr int PH = cgfft::line_pitch<H>();
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ unsigned beg[4], pre[5];
  const SmemLine<PH> mid{reinterpret_cast<cplx*>(smraw)};
  float* tf = reinterpret_cast<float*>(smraw);
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * TY;
  if (threadIdx.x == 0) {
    unsigned k[8], sv[8];
    col_range_keys(N, x, y0, TY, k);
#pragma unroll
    for (int q = 0; q < 8; q++) sv[q] = start[k[q]];
    pre[0] = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      beg[q] = sv[2 * q];
      pre[q + 1] = pre[q] + (sv[2 * q + 1] - sv[2 * q]);
    }
  }
  __syncthreads();
  const unsigned total = pre[4];
  // the first entries' loads are in flight while the tile is set to -1
  float4 w[DFZ_U];
  unsigned e0 = threadIdx.x;
#pragma unroll
  for (int u = 0; u < DFZ_U; u++) {
    const unsigned e = e0 + u * T;
    if (e < total) {
      const int q = e < pre[1] ? 0 : e < pre[2] ? 1 : e < pre[3] ? 2 : 3;
      w[u] = __ldg(ent + beg[q] + (e - pre[q]));
    }
  }
  for (int idx = threadIdx.x; idx < TY * H; idx += T) mid.st(idx / H, idx % H, cplx{-1.0f, -1.0f});
  __syncthreads();
  for (;;) {
#pragma unroll
    for (int u = 0; u < DFZ_U; u++)
      if (e0 + u * T < total) dfz_add<PH>(tf, w[u], N, x, y0, scale, wpar);
    e0 += DFZ_U * T;
    if (e0 >= total) break;
#pragma unroll
    for (int u = 0; u < DFZ_U; u++) {
      const unsigned e = e0 + u * T;
      if (e < total) {
        const int q = e < pre[1] ? 0 : e < pre[2] ? 1 : e < pre[3] ? 2 : 3;
        w[u] = __ldg(ent + beg[q] + (e - pre[q]));
      }
    }
  }
  __syncthreads();
  cgfft::fft_io<H, TY, T, true, -1>(mid, mid, mid, twH);
  fz_split_store<N>(mid, x, y0, spec, twN, dsum);
}

// FY: c2c along ky, BY contiguous lines per CTA, in place.
template <int N, int DIR>
__global__ void __launch_bounds__(T) k_fy(float2* __restrict__ spec,
                                          const float2* __restrict__ twN) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const SmemLine<cgfft::line_pitch<N>()> mid{reinterpret_cast<cplx*>(smraw)};
  const cgfft::GmemC<N, 1> g{spec + (size_t)blockIdx.x * BY * N};
  cgfft::fft_io<N, BY, T, true, DIR>(g, mid, g, twN);
}

// Load of a kx column scaled by the force component's wavenumber index:
// SCALE 1 by n_x = I0 (signed, Nyquist at +N/2; the position n along the
// column), SCALE 2 by n_z = kz (the plane, constant over the CTA).  With a
// gradient table g (finite-difference gradient), g[n] replaces n_x.
template <int SCALE>
struct GmemScaled {
  const float2* p;
  size_t es;
  int N;
  float fz;
  const float* g;
  __device__ __forceinline__ cplx ld(int b, int n) const {
    const float2 v = __ldg(p + b + (size_t)n * es);
    const float f = SCALE == 1 ? (g ? __ldg(g + n) : (float)(n <= N / 2 ? n : n - N)) : fz;
    // rounded products (never fused into the transform's first additions),
    // so that every gather of the pass gives the same bits
    return cplx{__fmul_rn(v.x, f), __fmul_rn(v.y, f)};
  }
  static constexpr bool kShared = false;
};

// FX: c2c along kx (stride N), TKV ky columns per CTA, from `in` to `out`
// (the same array for an in-place pass).  SCALE 0: plain; 1 / 2: the input
// is first multiplied by n_x / n_z (GmemScaled; gtab: the gradient table or
// NULL, unused by SCALE 0).
template <int N, int DIR, int SCALE, int TKV, int RMX>
__global__ void __launch_bounds__(T) k_fx(const float2* in, float2* out,
                                          const float2* __restrict__ twN,
                                          const float* __restrict__ gtab) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const SmemCol<TKV> mid{reinterpret_cast<cplx*>(smraw)};
  const size_t off = (size_t)blockIdx.y * N * N + blockIdx.x * TKV;
  const cgfft::GmemC<1, N> go{out + off};
  if constexpr (SCALE == 0) {
    const cgfft::GmemC<1, N> gi{const_cast<float2*>(in) + off};
    cgfft::fft_io<N, TKV, T, false, DIR, RMX>(gi, mid, go, twN);
  } else {
    const float fz = SCALE == 2 && gtab ? __ldg(gtab + blockIdx.y) : (float)blockIdx.y;
    const GmemScaled<SCALE> gi{in + off, (size_t)N, N, fz, gtab};
    cgfft::fft_io<N, TKV, T, false, DIR, RMX>(gi, mid, go, twN);
  }
}

// FX with the strided column gather done by TMA: the CTA's TKV ky columns
// of one kz plane (N rows of TKV complex, 64 or 128 bytes) land densely in
// the transform's own tile by tiled tensor loads with the 64- or 128-byte
// swizzle (cgfft::SmemSw8 / SmemSw16 undo it), in NB boxes of KR rows; the
// first stage then reads the tile, scaled by n_x or n_z as k_fx's loads
// scale them.  Same arithmetic as k_fx; bounded wait, CG_ERR_TMA_WAIT on a
// timeout.  The tensor map views the spectrum as floats (2N, N, N/2+1).
template <int N> __host__ __device__ constexpr int fx_nbox() { return (N + 255) / 256; }
template <int N> __host__ __device__ constexpr int fx_krows() { return N / fx_nbox<N>(); }
// Meshes up to 768^3 keep the twiddle entries of the x pass in shared memory
// (a few KB, copied while the tensor loads land).  A shared-memory load
// takes a 32-bit address where a table load took a 64-bit one: the
// 16-column radix-16 form fell from 186 to 128 registers, fits 2 CTAs per
// SM instead of 1, and takes 0.57 instead of 0.90 ms per launch at 768^3.
// Larger meshes read the table (their copies would cost a resident CTA per
// SM).  The z c2r measured slower with its copy (2.36 against 2.24-2.29 ms
// per step at 768^3) and reads the table.
template <int N> __host__ __device__ constexpr bool tw_in_smem() { return N <= 768; }

template <int N, int TKV, int RMX> __host__ __device__ constexpr size_t fx_sw_smem() {
  return sizeof(float2) * (size_t)N * TKV + 1024 + 16 +
         (tw_in_smem<N>() ? (size_t)cgfft::TwPack<N, RMX, false, false>::bytes : 0);
}
template <int TKV> struct SwTile;
template <> struct SwTile<8> { using type = cgfft::SmemSw8; };
template <> struct SwTile<16> { using type = cgfft::SmemSw16; };

// Shared tile element scaled on load like GmemScaled (SCALE 1: n_x or the
// gradient table at n; 2: the plane's n_z).
template <class S, int SCALE>
struct SmemScaled {
  S t;
  int N;
  float fz;
  const float* g;
  __device__ __forceinline__ cplx ld(int b, int n) const {
    const cplx v = t.ld(b, n);
    const float f = SCALE == 1 ? (g ? __ldg(g + n) : (float)(n <= N / 2 ? n : n - N)) : fz;
    return cplx{__fmul_rn(v.x, f), __fmul_rn(v.y, f)};
  }
  __device__ __forceinline__ void st(int b, int n, cplx v) const { t.st(b, n, v); }
  static constexpr bool kShared = true;
};

template <int N, int DIR, int SCALE, int TKV, int RMX>
__global__ void __launch_bounds__(T) k_fx_sw(const __grid_constant__ CUtensorMap tm,
                                             float2* out, const float2* __restrict__ twN,
                                             const float* __restrict__ gtab,
                                             unsigned* __restrict__ err) {
  static_assert(N % fx_nbox<N>() == 0 && fx_krows<N>() % 8 == 0, "box rows");
  constexpr int KR = fx_krows<N>(), NB = fx_nbox<N>();
  constexpr unsigned kBytes = (unsigned)(sizeof(float2) * N * TKV);
  extern __shared__ __align__(16) unsigned char smraw[];
  unsigned char* base =
      smraw + ((1024u - ((unsigned)__cvta_generic_to_shared(smraw) & 1023u)) & 1023u);
  using Tile = typename SwTile<TKV>::type;
  const Tile t{reinterpret_cast<cplx*>(base)};
  const unsigned bar = (unsigned)__cvta_generic_to_shared(base + kBytes);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                 "r"(kBytes) : "memory");
    const unsigned dst0 = (unsigned)__cvta_generic_to_shared(base);
#pragma unroll
    for (int h = 0; h < NB; h++) {
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst0 + (unsigned)(sizeof(float2) * TKV * KR * h)),
          "l"(reinterpret_cast<unsigned long long>(&tm)), "r"((int)(2 * TKV * blockIdx.x)),
          "r"(h * KR), "r"((int)blockIdx.y), "r"(bar)
          : "memory");
    }
  }
  // the stages' twiddles into shared memory while the tensor loads land
  using TP = cgfft::TwPack<N, RMX, false, false>;
  float2* tws = reinterpret_cast<float2*>(base + kBytes + 16);
  if constexpr (tw_in_smem<N>()) {
    TP::template copy<T>(tws, twN);
    __syncthreads();
  }
  const auto tw = [&] {
    if constexpr (tw_in_smem<N>()) return TP{tws};
    else return twN;
  }();
  unsigned done = 0;
  for (int it = 0; it < (1 << 22) && !done; it++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(bar) : "memory");
  }
  if (!done) {
    if (threadIdx.x == 0) atomicOr(err, (unsigned)CG_ERR_TMA_WAIT);
    return;
  }
  const size_t off = (size_t)blockIdx.y * N * N + blockIdx.x * TKV;
  const cgfft::GmemC<1, N> go{out + off};
  if constexpr (SCALE == 0) {
    cgfft::fft_io<N, TKV, T, false, DIR, RMX>(t, t, go, tw);
  } else {
    const float fz = SCALE == 2 && gtab ? __ldg(gtab + blockIdx.y) : (float)blockIdx.y;
    const SmemScaled<Tile, SCALE> ts{t, N, fz, gtab};
    cgfft::fft_io<N, TKV, T, false, DIR, RMX>(ts, t, go, tw);
  }
}

// Options of the Green step beyond the reference's kernel (all off: the
// reference's exact spectral force).
//  * t: an isotropic transfer function of the force T(|n|) (|n| in units of
//    the fundamental), sampled at knots |n| = j / inv_dn, j < n, linear in
//    between (the last knot beyond the table): the Fourier-space form of
//    the learned force correction.  NULL: none.
//  * tab: NULL, or three tables of N floats indexed like the spectrum's
//    axes (signed index s = i <= N/2 ? i : i - N): the gradient factor that
//    replaces s (a finite-difference gradient), the per-axis term of the
//    Laplacian that replaces s^2 in |n|^2 (the discrete Laplacian), and
//    the per-axis factor that divides out the CIC window.
struct GreenMods {
  const float* t;
  int n;
  float inv_dn;
  const float* tab;
  int kz0;          // kz of the first plane the launch sees (a kz slab; 0: the whole spectrum)
  __device__ __forceinline__ float at(int den) const {
    const float r = __fmul_rn(sqrtf((float)den), inv_dn);
    const int i = (int)r;
    if (i >= n - 1) return t[n - 1];
    const float a = t[i], b = t[i + 1];
    return __fadd_rn(a, __fmul_rn(__fsub_rn(r, (float)i), __fsub_rn(b, a)));
  }
};

// compute_force_mesh (pm.c:304-346) on lines (kz, kx) that are already
// transformed along z and x:  F_a = i f2 delta_k,
//   f2 = f1 / (K^2 + I0^2 + J0^2) * n_a,  f1 = -1/(N^3 2 pi/L),
//   I0, J0 signed with the Nyquist index kept at +N/2, F(0,0,0) = 0.
// GreenLoad applies the factor while the first inverse stage loads the
// forward-transformed tile: MODE 0 the y component (n_y = J0, the position
// along the line), MODE 1 the factor without n_a, MODE 2 the y component
// while it writes the MODE 1 value back in place.
template <int P, int MODE, bool MODS>
struct GreenLoad {
  cplx* s;
  int kz, kx0, N;
  float f1;
  GreenMods gm;
  __device__ __forceinline__ cplx ld(int b, int n) const {
    const cplx p = s[b * P + n + (n >> 4)];
    const int kx = kx0 + b;
    const int I0 = kx <= N / 2 ? kx : kx - N;
    const int J0 = n <= N / 2 ? n : n - N;
    const int den = kz * kz + I0 * I0 + J0 * J0;
    if (den == 0) {
      if (MODE == 2) s[b * P + n + (n >> 4)] = cplx{0.0f, 0.0f};
      return cplx{0.0f, 0.0f};
    }
    // MODS false: the reference's kernel, with none of the options' code
    const float* tab = MODS ? gm.tab : nullptr;
    float f2;
    if (tab) {
      const float* lap = tab + N;
      const float* win = tab + 2 * N;
      f2 = __fdiv_rn(f1, __fadd_rn(__fadd_rn(__ldg(lap + kx), __ldg(lap + n)), __ldg(lap + kz)));
      if (gm.t) f2 = __fmul_rn(f2, gm.at(den));
      f2 = __fmul_rn(f2, __fmul_rn(__fmul_rn(__ldg(win + kx), __ldg(win + n)), __ldg(win + kz)));
    } else {
      f2 = __fdiv_rn(f1, (float)den);
      if (MODS && gm.t) f2 = __fmul_rn(f2, gm.at(den));
    }
    if (MODE == 2) {
      // the shared x/z value replaces the loaded one in place (this thread
      // is the element's only reader in this stage), so the second inverse
      // transform reads it plainly instead of dividing again
      s[b * P + n + (n >> 4)] = cplx{-__fmul_rn(f2, p.y), __fmul_rn(f2, p.x)};
    }
    if (MODE != 1) f2 = __fmul_rn(f2, tab ? __ldg(tab + n) : (float)J0);
    return cplx{-__fmul_rn(f2, p.y), __fmul_rn(f2, p.x)};
  }
  static constexpr bool kShared = true;
  // never the output tile of the stage that reads it (k_green's first
  // inverse stage reads D and writes W), so that stage needs no barrier
  // between its loads and its stores; unreferenced where the transform has
  // one stage
#pragma nv_diag_suppress 177
  static constexpr bool kDistinct = true;
#pragma nv_diag_default 177
};

// The three transforms of the fused pass as separate (not inlined) calls:
// each keeps its own register live range, so the kernel fits MINB CTAs per
// SM without spilling.
template <int N, int BG, int RMG, int TG, int DIR, class First, class Mid, class Last>
__device__ __noinline__ void fft_tile_y(const First f, const Mid m, const Last l,
                                        const float2* __restrict__ tw) {
  cgfft::fft_io<N, BG, TG, true, DIR, RMG>(f, m, l, tw);
}

// GREEN: forward c2c along ky, Green/gradient, inverse c2c along ky:
//   g1 = IFFT_y(i f1 n_y/|n|^2 delta)       the y component
//   g2 = IFFT_y(i f1/|n|^2 delta)           the x and z components before
// their factor n_x / n_z, which is constant along a y line and is applied
// by the inverse x pass as it loads g2 (k_fx, SCALE 1 and 2): one inverse
// transform serves both components.  BG lines (kz, kx0 .. kx0+BG-1) per
// CTA of TG threads; N is a multiple of BG so the lines of a CTA share kz.
template <int N, int BG, int RMG, int MINB, int TG, bool MODS>
__global__ void __launch_bounds__(TG, MINB) k_green(const float2* __restrict__ spec,
                                                         float2* __restrict__ g1,
                                                         float2* __restrict__ g2,
                                                         const float2* __restrict__ twN,
                                                         float f1, GreenMods gm) {
  constexpr int P = cgfft::line_pitch<N>();
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx* D = reinterpret_cast<cplx*>(smraw);
  cplx* W = D + BG * P;
  const size_t l0 = (size_t)blockIdx.x * BG;
  const int kz = (int)(l0 / N) + gm.kz0;
  const int kx0 = (int)(l0 % N);
  const size_t off = l0 * N;
  const cgfft::GmemC<N, 1> gin{const_cast<float2*>(spec) + off};
  const SmemLine<P> d{D}, w{W};
  fft_tile_y<N, BG, RMG, TG, -1>(gin, d, d, twN);
  // the y component's load also leaves the shared x/z value in D
  const GreenLoad<P, 2, MODS> gy{D, kz, kx0, N, f1, gm};
  const cgfft::GmemC<N, 1> oy{g1 + off};
  fft_tile_y<N, BG, RMG, TG, 1>(gy, w, oy, twN);
  __syncthreads();
  const cgfft::GmemC<N, 1> os{g2 + off};
  fft_tile_y<N, BG, RMG, TG, 1>(d, d, os, twN);
}

// ZI: c2r along z of S (lines (x, y0..y0+TY-1) per CTA) into R.  The
// transposed tile is gathered with cp.async (8-byte copies, no register
// staging).  Half-complex convention (the FFTW c2r the reference relies
// on): Im X_0 and Im X_{N/2} are ignored.
//   Z_k = (X_k + conj X_{H-k}) + i W_N^{-k} (X_k - conj X_{H-k}),  k < H
//   z = IDFT_H(Z),  x_2m = Re z_m,  x_2m+1 = Im z_m   (unnormalised)
template <int N>
__global__ void __launch_bounds__(T) k_zi(const float2* __restrict__ gsp,
                                          float* __restrict__ out,
                                          const float2* __restrict__ twH,
                                          const float2* __restrict__ twN) {
  constexpr int H = N / 2;
  constexpr int PZ = cgfft::line_pitch<H + 1>();
  extern __shared__ __align__(16) unsigned char smraw[];
  const SmemLine<PZ> mid{reinterpret_cast<cplx*>(smraw)};
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * TY;
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smraw);
  for (int idx = threadIdx.x; idx < (H + 1) * TY; idx += T) {
    const int b = idx % TY, k = idx / TY;
    const float2* src = gsp + ((size_t)k * N + x) * N + y0 + b;
    const unsigned dst = sbase + 8u * (unsigned)(b * PZ + k + (k >> 4));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  for (int idx = threadIdx.x; idx < (H / 2 + 1) * TY; idx += T) {
    const int b = idx % TY, k = idx / TY;
    if (k == 0) {
      const float x0 = mid.ld(b, 0).x, xh = mid.ld(b, H).x;
      mid.st(b, 0, cplx{x0 + xh, x0 - xh});
    } else {
      const int k2 = H - k;
      const cplx a = mid.ld(b, k), c = mid.ld(b, k2);
      const float2 wa = __ldg(twN + k), wc = __ldg(twN + k2);
      // i * conj(w) * d  with conj(w) = (w.x, -w.y)
      const cplx sa = {a.x + c.x, a.y - c.y}, da = {a.x - c.x, a.y + c.y};
      const cplx ra = {da.x * wa.x + da.y * wa.y, da.y * wa.x - da.x * wa.y};
      const cplx za = {sa.x - ra.y, sa.y + ra.x};
      const cplx sc = {c.x + a.x, c.y - a.y}, dc = {c.x - a.x, c.y + a.y};
      const cplx rc = {dc.x * wc.x + dc.y * wc.y, dc.y * wc.x - dc.x * wc.y};
      const cplx zc = {sc.x - rc.y, sc.y + rc.x};
      mid.st(b, k, za);
      if (k2 != k) mid.st(b, k2, zc);
    }
  }
  __syncthreads();
  const cgfft::GmemC<H, 1> gout{reinterpret_cast<float2*>(out) + ((size_t)x * N + y0) * H};
  cgfft::fft_io<H, TY, T, true, 1>(mid, mid, gout, twH);
}

// ZI with the transposed gather done by TMA: the (N/2+1) kz rows of TY
// complex (128 B each) for one (x, y0) land densely in shared memory from
// ZI_NB tiled tensor loads of ZI_KROWS rows (a box dimension is at most 256),
// completing on one mbarrier; the half-complex combination then copies them
// into the padded line tile that the transform reads.  Bit for bit the same
// arithmetic as k_zi.  The wait is bounded: on a timeout the CTA sets
// CG_ERR_TMA_WAIT and returns.  The tensor map views the spectrum as floats
// (2N, N, N/2+1) with box (2 TY, 1, ZI_KROWS); the x coordinate 2 y0 is a
// multiple of 32 floats (128 B).
template <int N> __host__ __device__ constexpr int zi_nbox() { return (N / 2 + 1 + 255) / 256; }
template <int N> __host__ __device__ constexpr int zi_krows() {
  return (N / 2 + 1 + zi_nbox<N>() - 1) / zi_nbox<N>();
}
template <int N> __host__ __device__ constexpr size_t zi_tma_smem() {
  return sizeof(float2) * zi_nbox<N>() * zi_krows<N>() * TY +
         sizeof(cplx) * TY * cgfft::line_pitch<N / 2 + 1>() + 16 + 128;   // + alignment slack
}

template <int N>
__global__ void __launch_bounds__(T, 2) k_zi_tma(const __grid_constant__ CUtensorMap tm,
                                                 float* __restrict__ out,
                                                 const float2* __restrict__ twH,
                                                 const float2* __restrict__ twN,
                                                 unsigned* __restrict__ err) {
  constexpr int H = N / 2;
  constexpr int PZ = cgfft::line_pitch<H + 1>();
  constexpr int KR = zi_krows<N>(), NB = zi_nbox<N>();
  constexpr unsigned kBytes = (unsigned)(sizeof(float2) * NB * KR * TY);
  extern __shared__ __align__(16) unsigned char smraw[];
  // the landing area starts on a 128-byte boundary of the shared window
  unsigned char* base =
      smraw + ((128u - ((unsigned)__cvta_generic_to_shared(smraw) & 127u)) & 127u);
  const float2* land = reinterpret_cast<const float2*>(base);
  const SmemLine<PZ> mid{reinterpret_cast<cplx*>(base + kBytes)};
  const unsigned bar = (unsigned)__cvta_generic_to_shared(base + kBytes + sizeof(cplx) * TY * PZ);
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * TY;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                 "r"(kBytes) : "memory");
    const unsigned dst0 = (unsigned)__cvta_generic_to_shared(base);
    for (int h = 0; h < NB; h++) {
      const unsigned dst = dst0 + (unsigned)(sizeof(float2) * h * KR * TY);
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
          "l"(reinterpret_cast<unsigned long long>(&tm)), "r"(2 * y0), "r"(x), "r"(h * KR),
          "r"(bar)
          : "memory");
    }
  }
  unsigned done = 0;
  for (int it = 0; it < (1 << 22) && !done; it++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(bar) : "memory");
  }
  if (!done) {
    if (threadIdx.x == 0) atomicOr(err, (unsigned)CG_ERR_TMA_WAIT);
    return;
  }
  for (int idx = threadIdx.x; idx < (H / 2 + 1) * TY; idx += T) {
    const int b = idx % TY, k = idx / TY;
    if (k == 0) {
      const float x0 = land[b].x, xh = land[H * TY + b].x;
      mid.st(b, 0, cplx{x0 + xh, x0 - xh});
    } else {
      const int k2 = H - k;
      const float2 a2 = land[k * TY + b], c2 = land[k2 * TY + b];
      const cplx a = {a2.x, a2.y}, c = {c2.x, c2.y};
      const float2 wa = __ldg(twN + k), wc = __ldg(twN + k2);
      const cplx sa = {a.x + c.x, a.y - c.y}, da = {a.x - c.x, a.y + c.y};
      const cplx ra = {da.x * wa.x + da.y * wa.y, da.y * wa.x - da.x * wa.y};
      const cplx za = {sa.x - ra.y, sa.y + ra.x};
      const cplx sc = {c.x + a.x, c.y - a.y}, dc = {c.x - a.x, c.y + a.y};
      const cplx rc = {dc.x * wc.x + dc.y * wc.y, dc.y * wc.x - dc.x * wc.y};
      const cplx zc = {sc.x - rc.y, sc.y + rc.x};
      mid.st(b, k, za);
      if (k2 != k) mid.st(b, k2, zc);
    }
  }
  __syncthreads();
  const cgfft::GmemC<H, 1> gout{reinterpret_cast<float2*>(out) + ((size_t)x * N + y0) * H};
  cgfft::fft_io<H, TY, T, true, 1>(mid, mid, gout, twH);
}

// ZI with the transposed gather landing straight in the transform's tile:
// the tile is dense, n-major ([kz][b], 128-byte rows of TY = 16 complex),
// written by tiled tensor loads with the 128-byte swizzle (cgfft::SmemSw16
// undoes it), so no padded copy is needed and the CTA holds one tile only
// ((N/2+1) x 128 B rounded up to whole boxes: 51 KB at 768^3, four CTAs per
// SM).  ZSW_NB boxes of ZSW_KR rows (a multiple of 8, so every box starts on
// a 1024-byte boundary of the tile; rows past N/2 are filled with zeros and
// never read).  The half-complex combination runs in place on the tile, the
// inner stages map consecutive threads to consecutive lines (conflict-free
// on the swizzled rows) and the last stage to consecutive butterflies of a
// line (coalesced stores).  Same arithmetic as k_zi; bounded wait, error
// word CG_ERR_TMA_WAIT on a timeout.
template <int N> __host__ __device__ constexpr int zsw_nbox() { return (N / 2 + 1 + 255) / 256; }
template <int N> __host__ __device__ constexpr int zsw_krows() {
  return ((N / 2 + 1 + zsw_nbox<N>() - 1) / zsw_nbox<N>() + 7) / 8 * 8;
}
template <int N> __host__ __device__ constexpr size_t zsw_smem() {
  return (size_t)128 * zsw_nbox<N>() * zsw_krows<N>() + 1024 + 16;   // + alignment, mbarrier
}
// The z c2r's stage twiddles (its N/2-point transform: column-mapped stages,
// a line-major last stage), packed in shared memory after the tile from
// 1024^3 on.  There the 32-bit shared addresses take the kernel from 188 to 4
// bytes of spill at 3 CTAs per SM (1024^3: 5.72 against 6.76 ms per step).
// At 384^3 and 768^3 the copy made the pass slower (768^3: 2.34-2.35
// against 2.25-2.30 ms per step), and it reads the table.
template <int N> using ZswPack = cgfft::TwPack<N / 2, 16, false, true>;
template <int N> __host__ __device__ constexpr bool zsw_pack() { return N >= 1024; }

// The swizzled tile's gather: thread 0 issues the NB tensor loads of the
// (N/2+1) kz rows of the lines (x, y0 .. y0+15) of the spectrum behind `tm`
// (mbarrier `bar`, already initialised, phase `parity`); every thread then
// waits, bounded.  False (for every thread) when the loads did not complete.
// `during` runs on every thread after the loads are issued, before the wait.
template <int N, class F>
__device__ __forceinline__ bool zsw_gather(const CUtensorMap& tm, unsigned char* base,
                                           unsigned bar, unsigned parity, int x, int y0,
                                           F during) {
  constexpr int KR = zsw_krows<N>(), NB = zsw_nbox<N>();
  constexpr unsigned kBytes = 128u * NB * KR;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                 "r"(kBytes) : "memory");
    const unsigned dst0 = (unsigned)__cvta_generic_to_shared(base);
#pragma unroll
    for (int h = 0; h < NB; h++) {
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst0 + 128u * KR * h),
          "l"(reinterpret_cast<unsigned long long>(&tm)), "r"(2 * y0), "r"(x), "r"(h * KR),
          "r"(bar)
          : "memory");
    }
  }
  during();
  unsigned done = 0;
  for (int it = 0; it < (1 << 22) && !done; it++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(bar), "r"(parity) : "memory");
  }
  return !__syncthreads_or(!done);
}

// Half-complex combination of k_zi (rows k and H - k of every line), in
// place on the swizzled tile.
template <int N>
__device__ __forceinline__ void zsw_halfcomplex(const cgfft::SmemSw16& t,
                                                const float2* __restrict__ twN) {
  constexpr int H = N / 2;
  for (int idx = threadIdx.x; idx < (H / 2 + 1) * TY; idx += T) {
    const int b = idx % TY, k = idx / TY;
    if (k == 0) {
      const float x0 = t.ld(b, 0).x, xh = t.ld(b, H).x;
      t.st(b, 0, cplx{x0 + xh, x0 - xh});
    } else {
      const int k2 = H - k;
      const cplx a = t.ld(b, k), c = t.ld(b, k2);
      const float2 wa = __ldg(twN + k), wc = __ldg(twN + k2);
      const cplx sa = {a.x + c.x, a.y - c.y}, da = {a.x - c.x, a.y + c.y};
      const cplx ra = {da.x * wa.x + da.y * wa.y, da.y * wa.x - da.x * wa.y};
      const cplx za = {sa.x - ra.y, sa.y + ra.x};
      const cplx sc = {c.x + a.x, c.y - a.y}, dc = {c.x - a.x, c.y + a.y};
      const cplx rc = {dc.x * wc.x + dc.y * wc.y, dc.y * wc.x - dc.x * wc.y};
      const cplx zc = {sc.x - rc.y, sc.y + rc.x};
      t.st(b, k, za);
      if (k2 != k) t.st(b, k2, zc);
    }
  }
}

template <int N>
__global__ void __launch_bounds__(T, N >= 768 ? 3 : 4) k_zi_sw(const __grid_constant__ CUtensorMap tm,
                                             float* __restrict__ out,
                                             const float2* __restrict__ twH,
                                             const float2* __restrict__ twN,
                                             unsigned* __restrict__ err) {
  static_assert(TY == 16, "the swizzled tile holds 16 lines per 128-byte row");
  constexpr int H = N / 2;
  constexpr int KR = zsw_krows<N>(), NB = zsw_nbox<N>();
  constexpr unsigned kBytes = 128u * NB * KR;
  extern __shared__ __align__(16) unsigned char smraw[];
  unsigned char* base =
      smraw + ((1024u - ((unsigned)__cvta_generic_to_shared(smraw) & 1023u)) & 1023u);
  const cgfft::SmemSw16 t{reinterpret_cast<cplx*>(base)};
  const unsigned bar = (unsigned)__cvta_generic_to_shared(base + kBytes);
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * TY;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  // from 1024^3 on, the transform's stage twiddles (4 KB) into shared
  // memory while the tensor loads land
  using TP = ZswPack<N>;
  float2* tws = reinterpret_cast<float2*>(base + kBytes + 16);
  if (!zsw_gather<N>(tm, base, bar, 0, x, y0, [&] {
        if constexpr (zsw_pack<N>()) TP::template copy<T>(tws, twH);
      })) {
    if (threadIdx.x == 0) atomicOr(err, (unsigned)CG_ERR_TMA_WAIT);
    return;
  }
  zsw_halfcomplex<N>(t, twN);
  __syncthreads();
  const cgfft::GmemC<H, 1> gout{reinterpret_cast<float2*>(out) + ((size_t)x * N + y0) * H};
  if constexpr (zsw_pack<N>())
    cgfft::fft_io<H, TY, T, false, 1, 16, true>(t, t, gout, TP{tws});
  else
    cgfft::fft_io<H, TY, T, false, 1, 16, true>(t, t, gout, twH);
}

// ------------------------------------------ z c2r fused with interpolation
// ZIP: the z c2r of one force component with the CIC interpolation of its
// plane (force_at_particle_locations, pm.c:370-411) done from the
// transformed lines in shared memory, so the force mesh is never written to
// or read from HBM.  A CTA computes the 16 lines (x, y0 .. y0+15), y0 = 14 t
// (tiles overlap by two lines: a cloud with lower corner column j0 needs
// lines j0 and j0 + 1), and interpolates the clouds of the column bins
// (k_col_count) with i0 = x (plane x is the cloud's i0) or i0 = x - 1 (its
// i1) and j0 in y0 .. y0+13.  Tiles that reach past line N - 1 hold the
// lines (y0 + b) mod N, gathered by plain loads (line 0 follows line N - 1);
// the others take k_zi_sw's tensor loads (y0 = 14 t keeps the box's x
// coordinate 2 y0 floats on a 16-byte boundary).  Each cloud's gather4
// partial goes to its slot: p0[e] (plane i0) or p1[e] (plane i1).  The
// lines are bit for bit k_zi's, and the partials are gather4 of
// interp_one, so k_interp_sum reproduces k_interp's forces exactly.
constexpr int ZIP_S = 14;
__host__ __device__ constexpr int zip_tiles(int N) { return (N + ZIP_S - 1) / ZIP_S; }

__device__ __forceinline__ float zsw_real(const cgfft::SmemSw16& t, int b, int k) {
  const cplx z = t.ld(b, k >> 1);
  return (k & 1) ? z.y : z.x;
}

template <int N>
__global__ void __launch_bounds__(T, N >= 1024 ? 3 : 4) k_zi_interp(
    const __grid_constant__ CUtensorMap tm, const float2* __restrict__ gsp,
    const float4* __restrict__ ent, const unsigned* __restrict__ start,
    float* __restrict__ p0, float* __restrict__ p1, const float2* __restrict__ twH,
    const float2* __restrict__ twN, float scale, unsigned* __restrict__ err) {
  static_assert(TY == 16, "the swizzled tile holds 16 lines per 128-byte row");
  constexpr int H = N / 2;
  constexpr int KR = zsw_krows<N>(), NB = zsw_nbox<N>();
  constexpr unsigned kBytes = 128u * NB * KR;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ unsigned beg[2], pre[3];
  unsigned char* base =
      smraw + ((1024u - ((unsigned)__cvta_generic_to_shared(smraw) & 1023u)) & 1023u);
  const cgfft::SmemSw16 t{reinterpret_cast<cplx*>(base)};
  const unsigned bar = (unsigned)__cvta_generic_to_shared(base + kBytes);
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * ZIP_S;
  const bool wrap = y0 + TY > N;
  if (!wrap) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
  }
  // the tensor loads go out first; the entry ranges are read while they land
  // (key rows x (i0 = x - 1) and x + 1 (i0 = x), columns y0 .. min(y0+14, N) - 1)
  const auto ranges = [&] {
    if (threadIdx.x == 0) {
      const unsigned c0 = (unsigned)y0, c1 = (unsigned)min(y0 + ZIP_S, N);
      const unsigned k0 = (unsigned)x * N, k1 = k0 + N;
      const unsigned s00 = start[k0 + c0], s01 = start[k0 + c1];
      const unsigned s10 = start[k1 + c0], s11 = start[k1 + c1];
      beg[0] = s00;
      beg[1] = s10;
      pre[0] = 0;
      pre[1] = s01 - s00;
      pre[2] = pre[1] + (s11 - s10);
    }
  };
  if (!wrap) {
    if (!zsw_gather<N>(tm, base, bar, 0, x, y0, ranges)) {
      if (threadIdx.x == 0) atomicOr(err, (unsigned)CG_ERR_TMA_WAIT);
      return;
    }
  } else {
    ranges();
    for (int idx = threadIdx.x; idx < (H + 1) * TY; idx += T) {
      const int b = idx % TY, k = idx / TY;
      const int y = y0 + b < N ? y0 + b : y0 + b - N;
      const float2 v = __ldg(gsp + ((size_t)k * N + x) * N + y);
      t.st(b, k, cplx{v.x, v.y});
    }
    __syncthreads();
  }
  zsw_halfcomplex<N>(t, twN);
  __syncthreads();
  cgfft::fft_io<H, TY, T, false, 1>(t, t, t, twH);
  const unsigned total = pre[2];
  for (unsigned e = threadIdx.x; e < total; e += T) {
    const int q = e < pre[1] ? 0 : 1;
    const unsigned ei = beg[q] + (e - pre[q]);
    const float4 w = __ldg(ent + ei);
    const Cic c = cic_index(w.x, w.y, w.z, N, scale);
    const bool at_i0 = c.i0 == x;
    const float wi = at_i0 ? c.t1 : c.d1;
    const int b0 = c.j0 - y0;            // line j1 = j0 + 1 (mod N) sits at b0 + 1
    // gather4: ((m*T3)*Ti)*T2 + ((m*D3)*Ti)*T2 + ((m*T3)*Ti)*D2 + ((m*D3)*Ti)*D2
    const float a = __fmul_rn(__fmul_rn(__fmul_rn(zsw_real(t, b0, c.k0), c.t3), wi), c.t2);
    const float b = __fmul_rn(__fmul_rn(__fmul_rn(zsw_real(t, b0, c.k1), c.d3), wi), c.t2);
    const float d = __fmul_rn(__fmul_rn(__fmul_rn(zsw_real(t, b0 + 1, c.k0), c.t3), wi), c.d2);
    const float g = __fmul_rn(__fmul_rn(__fmul_rn(zsw_real(t, b0 + 1, c.k1), c.d3), wi), c.d2);
    (at_i0 ? p0 : p1)[ei] = __fadd_rn(__fadd_rn(__fadd_rn(a, b), d), g);
  }
}

// The forces of the primary clouds, in interp_one's order:
// f = (0 + gather4(i0)) + gather4(i1), each term for a plane inside the mesh.
// part holds the slots p0, p1 of the x, y and z components, stride cap2.
__global__ void __launch_bounds__(T) k_interp_sum(const float4* __restrict__ ent,
                                                  const unsigned* __restrict__ start, int N,
                                                  float scale, const float* __restrict__ part,
                                                  long long cap2, float* __restrict__ f0,
                                                  float* __restrict__ f1, float* __restrict__ f2) {
  const unsigned hi = start[(size_t)(N + 1) * N];
  float* const f[3] = {f0, f1, f2};
  for (unsigned e = blockIdx.x * T + threadIdx.x; e < hi; e += gridDim.x * T) {
    const float4 w = __ldg(ent + e);
    const unsigned i = __float_as_uint(w.w);
    if (i & COL_COPY) continue;
    const Cic c = cic_index(w.x, w.y, w.z, N, scale);
    const bool in0 = 0 <= c.i0 && c.i0 < N, in1 = 0 <= c.i1 && c.i1 < N;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      float s = 0.0f;
      if (in0) s = __fadd_rn(s, __ldg(part + (2 * a) * cap2 + e));
      if (in1) s = __fadd_rn(s, __ldg(part + (2 * a + 1) * cap2 + e));
      f[a][i] = s;
    }
  }
}

// The buffer copies' forces added to their particles' (add_buffer_forces,
// pm.c:526-531, of interp_one for the copy).  After the wrap every copy
// sits in key row 0 (i0 = -1, i1 = 0), the entries before start[N]; when
// k_col_count counted copies elsewhere, every entry is looked at.
__global__ void __launch_bounds__(T) k_interp_copies(const float4* __restrict__ ent,
                                                     const unsigned* __restrict__ start, int N,
                                                     float scale, const float* __restrict__ part,
                                                     long long cap2, float* __restrict__ f0,
                                                     float* __restrict__ f1,
                                                     float* __restrict__ f2) {
  const size_t keys = (size_t)(N + 1) * N;
  const unsigned hi = start[keys + 1] ? start[keys] : start[N];
  float* const f[3] = {f0, f1, f2};
  for (unsigned e = blockIdx.x * T + threadIdx.x; e < hi; e += gridDim.x * T) {
    const float4 w = __ldg(ent + e);
    const unsigned i = __float_as_uint(w.w);
    if (!(i & COL_COPY)) continue;
    const Cic c = cic_index(w.x, w.y, w.z, N, scale);
    const bool in0 = 0 <= c.i0 && c.i0 < N, in1 = 0 <= c.i1 && c.i1 < N;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      float s = 0.0f;
      if (in0) s = __fadd_rn(s, __ldg(part + (2 * a) * cap2 + e));
      if (in1) s = __fadd_rn(s, __ldg(part + (2 * a + 1) * cap2 + e));
      f[a][i & ~COL_COPY] = __fadd_rn(f[a][i & ~COL_COPY], s);
    }
  }
}

// Gather of the z c2r by mesh size (the plans created afterwards):
//   0  cp.async (k_zi)
//   1  TMA into a landing area, copied into the padded tile (k_zi_tma)
//   2  TMA into the swizzled dense tile itself (k_zi_sw)
// All three give bit-identical output.  Default: 2, the fastest at 384^3
// (0.104 ms per launch against 0.115 and 0.124 for 1 and 0) and at 768^3
// (0.81 ms against 1.15 and 0.97), per launch inside the 10-step runs;
// cg_set_z_gather, or COLAGPU_ZI=0/1/2, selects one.
std::atomic<int> g_zmode{-1};

// Gather of the strided x pass in the force step (plans created afterwards):
// 0 direct loads (k_fx), 1 TMA into the swizzled tile (k_fx_sw).
// cg_set_x_gather, or COLAGPU_FXG=0/1, selects one; both give bit-identical
// output.
std::atomic<int> g_xmode{-1};

// Deposit of the force step: 0 the mesh deposit + k_fz (the default), 1
// column bins + k_dfz.  pm_set_force_deposit / cg_set_force_deposit, or
// COLAGPU_FUSED_DEPOSIT=0/1, selects one.  The default stays the mesh
// deposit: the column bins' ranks come from atomics whose order varies from
// run to run, so the binned deposit adds the clouds in a different order
// every time and its results are not bit-reproducible, and it measured only
// 0.15 ms per step faster at 768^3 (0.31 ms binning + 1.24 ms k_dfz against
// 0.75 ms deposit + 0.98 ms k_fz).
std::atomic<int> g_fdep{-1};

bool fused_deposit() {
  static const int forced = [] {
    const char* e = getenv("COLAGPU_FUSED_DEPOSIT");
    return e ? atoi(e) : -1;
  }();
  const int m = forced >= 0 ? forced : g_fdep.load();
  return m == 1;
}

int x_gather_mode(int N, bool* explicit_choice) {
  static const int forced = [] {
    const char* e = getenv("COLAGPU_FXG");
    return e ? atoi(e) : -1;
  }();
  const int m = forced >= 0 ? forced : g_xmode.load();
  *explicit_choice = m == 0 || m == 1;
  if (*explicit_choice) return m;
  (void)N;
  return 1;
}

int z_gather_mode(int N, bool* explicit_choice) {
  static const int forced = [] {
    const char* e = getenv("COLAGPU_ZI");
    return e ? atoi(e) : -1;
  }();
  const int m = forced >= 0 ? forced : g_zmode.load();
  *explicit_choice = m >= 0 && m <= 2;
  if (*explicit_choice) return m;
  (void)N;
  return 2;
}

// ---------------------------------------------------- power spectrum bins
// Shell average of |delta_k|^2 over the half spectrum S[kz][kx][ky]: bin b
// holds modes with |n| in [b + 1/2, b + 3/2) (|n| in units of the
// fundamental), weight 2 for 0 < kz < N/2 (each stands for itself and its
// conjugate), 1 on the kz = 0 and kz = N/2 planes.  Optional division by the
// CIC window prod_i sinc^2(pi n_i / N) squared.  acc = [sum w, sum w |n|,
// sum w |S|^2] per bin, accumulated in double.
__global__ void __launch_bounds__(T) k_pk_bin(const float2* __restrict__ spec, int N, int nbins,
                                              int deconv, double* __restrict__ acc) {
  extern __shared__ double sb[];
  for (int i = threadIdx.x; i < 3 * nbins; i += T) sb[i] = 0.0;
  __syncthreads();
  const size_t total = (size_t)(N / 2 + 1) * N * N;
  for (size_t t = (size_t)blockIdx.x * T + threadIdx.x; t < total; t += (size_t)gridDim.x * T) {
    const int kz = (int)(t / ((size_t)N * N));
    const int i = (int)((t / N) % N);
    const int j = (int)(t % N);
    const int si = i <= N / 2 ? i : i - N;
    const int sj = j <= N / 2 ? j : j - N;
    const double n2 = (double)si * si + (double)sj * sj + (double)kz * kz;
    const double nm = sqrt(n2);
    const int b = (int)floor(nm + 0.5) - 1;
    if (b < 0 || b >= nbins) continue;
    const double w = (kz == 0 || kz == N / 2) ? 1.0 : 2.0;
    const float2 s = spec[t];
    double p = (double)s.x * s.x + (double)s.y * s.y;
    if (deconv) {
      double win = 1.0;
      const int ns[3] = {si, sj, kz};
      for (int a = 0; a < 3; a++) {
        if (ns[a] != 0) {
          const double x = M_PI * ns[a] / N;
          const double sc = sin(x) / x;
          win *= sc * sc;
        }
      }
      p /= win * win;
    }
    atomicAdd(&sb[b], w);
    atomicAdd(&sb[nbins + b], w * nm);
    atomicAdd(&sb[2 * nbins + b], w * p);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * nbins; i += T)
    if (sb[i] != 0.0) atomicAdd(&acc[i], sb[i]);
}

// ------------------------------------------------------- dispatch table
struct MeshKernels {
  void (*fz)(const float*, float2*, const float2*, const float2*, double*);
  void (*fz_reset)(float*, float2*, const float2*, const float2*, double*);
  void (*dfz)(const float4*, const unsigned*, float2*, const float2*, const float2*, double*,
              float, float);
  void (*fyf)(float2*, const float2*);
  void (*fyi)(float2*, const float2*);
  void (*fxf)(const float2*, float2*, const float2*, const float*);
  void (*fxi)(const float2*, float2*, const float2*, const float*);
  void (*fxi_x)(const float2*, float2*, const float2*, const float*);   // input times n_x
  void (*fxi_z)(const float2*, float2*, const float2*, const float*);   // input times n_z
  // the same four with the TMA gather (k_fx_sw)
  void (*fxf_sw)(CUtensorMap, float2*, const float2*, const float*, unsigned*);
  void (*fxi_sw)(CUtensorMap, float2*, const float2*, const float*, unsigned*);
  void (*fxi_x_sw)(CUtensorMap, float2*, const float2*, const float*, unsigned*);
  void (*fxi_z_sw)(CUtensorMap, float2*, const float2*, const float*, unsigned*);
  size_t sm_fx_sw;
  void (*green)(const float2*, float2*, float2*, const float2*, float, GreenMods);
  void (*green_mods)(const float2*, float2*, float2*, const float2*, float, GreenMods);
  void (*zi)(const float2*, float*, const float2*, const float2*);
  void (*zi_tma)(CUtensorMap, float*, const float2*, const float2*, unsigned*);
  void (*zi_sw)(CUtensorMap, float*, const float2*, const float2*, unsigned*);
  void (*zip)(CUtensorMap, const float2*, const float4*, const unsigned*, float*, float*,
              const float2*, const float2*, float, unsigned*);
  size_t sm_fz, sm_fy, sm_fx, sm_green, sm_zi, sm_zi_tma, sm_zi_sw;
  int tk;    // ky columns per CTA of the x pass
  int byg;   // lines per CTA of the Green pass
  int tg;    // threads per CTA of the Green pass
};

template <int N, int V>
void set_fx(MeshKernels* k) {
  constexpr int TKV = kFxCfg[V].tk, RMX = fx_rm(N, V);
  k->fxf = k_fx<N, -1, 0, TKV, RMX>;
  k->fxi = k_fx<N, 1, 0, TKV, RMX>;
  k->fxi_x = k_fx<N, 1, 1, TKV, RMX>;
  k->fxi_z = k_fx<N, 1, 2, TKV, RMX>;
  k->fxf_sw = k_fx_sw<N, -1, 0, TKV, RMX>;
  k->fxi_sw = k_fx_sw<N, 1, 0, TKV, RMX>;
  k->fxi_x_sw = k_fx_sw<N, 1, 1, TKV, RMX>;
  k->fxi_z_sw = k_fx_sw<N, 1, 2, TKV, RMX>;
  k->sm_fx_sw = fx_sw_smem<N, TKV, RMX>();
  k->sm_fx = sizeof(cplx) * cgfft::col_tile_elems<N, TKV>();
  k->tk = TKV;
}

template <int N, int V>
void set_green(MeshKernels* k) {
  constexpr GreenCfg c = kGreenCfg[V];
  k->green = k_green<N, c.byg, c.rm, c.minb, c.thr, false>;
  k->green_mods = k_green<N, c.byg, c.rm, c.minb, c.thr, true>;
  k->tg = c.thr;
  k->sm_green = sizeof(cplx) * 2 * c.byg * cgfft::line_pitch<N>();
  k->byg = c.byg;
}

template <int N>
MeshKernels make_kernels(MeshSched s) {
  MeshKernels k;
  k.fz = k_fz<N, false>;
  k.fz_reset = k_fz<N, true>;
  k.dfz = k_dfz<N, 4>;
  k.fyf = k_fy<N, -1>;
  k.fyi = k_fy<N, 1>;
  k.zi = k_zi<N>;
  k.zi_tma = k_zi_tma<N>;
  k.sm_zi_tma = zi_tma_smem<N>();
  k.zi_sw = k_zi_sw<N>;
  k.sm_zi_sw = zsw_smem<N>() + (zsw_pack<N>() ? ZswPack<N>::bytes : 0);
  k.zip = k_zi_interp<N>;
  k.sm_fz = sizeof(cplx) * TY * cgfft::line_pitch<N / 2>();
  k.sm_fy = sizeof(cplx) * BY * cgfft::line_pitch<N>();
  k.sm_zi = sizeof(cplx) * TY * cgfft::line_pitch<N / 2 + 1>();
  if constexpr (n_fx_variants(N) > 1) {
    switch (s.fx) {
      case 1: set_fx<N, 1>(&k); break;
      case 2: set_fx<N, 2>(&k); break;
      default: set_fx<N, 0>(&k);
    }
  } else {
    set_fx<N, 0>(&k);
  }
  if constexpr (n_green_variants(N) > 1) {
    switch (s.green) {
      case 1: set_green<N, 1>(&k); break;
      case 2: set_green<N, 2>(&k); break;
      case 3: set_green<N, 3>(&k); break;
      case 4: set_green<N, 4>(&k); break;
      case 5: set_green<N, 5>(&k); break;
      case 6: set_green<N, 6>(&k); break;
      default: set_green<N, 0>(&k);
    }
  } else {
    set_green<N, 0>(&k);
  }
  return k;
}

#define CG_MESH_SIZES(X) X(16) X(32) X(48) X(64) X(96) X(128) X(144) X(192) X(256) X(384) X(512) X(768) X(1024)

bool kernels_with(int N, MeshSched s, MeshKernels* out) {
  switch (N) {
#define CG_CASE(n) case n: *out = make_kernels<n>(s); return true;
    CG_MESH_SIZES(CG_CASE)
#undef CG_CASE
    default: return false;
  }
}

// The schedule in use per mesh size (variant 0 unless tuned or set).
std::mutex g_sched_mu;
std::map<int, MeshSched> g_sched;

MeshSched sched_for(int N) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  auto it = g_sched.find(N);
  return it == g_sched.end() ? MeshSched{} : it->second;
}

bool get_kernels(int N, MeshKernels* out) { return kernels_with(N, sched_for(N), out); }

cudaError_t set_smem(const void* fn, size_t bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Dynamic shared-memory limits of the pass kernels of one mesh size, for
// every schedule variant (a schedule may change after a plan exists).
cudaError_t set_all_smem(int N) {
  cudaError_t e = cudaSuccess;
  const int nv = n_fx_variants(N);
  const int ng = n_green_variants(N);
  for (int v = 0; v < (nv > ng ? nv : ng) && e == cudaSuccess; v++) {
    MeshKernels k;
    if (!kernels_with(N, MeshSched{v < ng ? v : 0, v < nv ? v : 0}, &k))
      return cudaErrorInvalidValue;
    if (e == cudaSuccess) e = set_smem((const void*)k.fz, k.sm_fz);
    if (e == cudaSuccess) e = set_smem((const void*)k.fz_reset, k.sm_fz);
    if (e == cudaSuccess) e = set_smem((const void*)k.dfz, k.sm_fz);
    if (e == cudaSuccess) e = set_smem((const void*)k.fyf, k.sm_fy);
    if (e == cudaSuccess) e = set_smem((const void*)k.fyi, k.sm_fy);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxf, k.sm_fx);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxi, k.sm_fx);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxi_x, k.sm_fx);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxi_z, k.sm_fx);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxf_sw, k.sm_fx_sw);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxi_sw, k.sm_fx_sw);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxi_x_sw, k.sm_fx_sw);
    if (e == cudaSuccess) e = set_smem((const void*)k.fxi_z_sw, k.sm_fx_sw);
    if (e == cudaSuccess) e = set_smem((const void*)k.green, k.sm_green);
    if (e == cudaSuccess) e = set_smem((const void*)k.green_mods, k.sm_green);
    if (e == cudaSuccess) e = set_smem((const void*)k.zi, k.sm_zi);
    if (e == cudaSuccess) e = set_smem((const void*)k.zi_tma, k.sm_zi_tma);
    if (e == cudaSuccess) e = set_smem((const void*)k.zi_sw, k.sm_zi_sw);
    if (e == cudaSuccess) e = set_smem((const void*)k.zip, k.sm_zi_sw);
  }
  return e;
}

// The twiddle table of length L (W_L^k rounded once from double), the
// per-stage rows after it (cgfft::stage_tw_offset) and the same stages'
// transposed runs (cgfft::stage_twt_offset), which copy its entries.
size_t twiddle_table_len(int L) { return (size_t)cgfft::twiddle_table_len(L); }

void twiddle_table(float2* h, int L) {
  for (int k = 0; k < L; k++) {
    const double a = -2.0 * 3.14159265358979323846264338327950288 * (double)k / (double)L;
    h[k] = make_float2((float)cos(a), (float)sin(a));
  }
  for (int pass = 0; pass < 2; pass++) {
    const int rm = pass == 0 ? 16 : 8;
    if (!cgfft::supported_length(L, rm)) continue;
    for (int st = 1; st < cgfft::num_stages(L, rm); st++) {
      const int ns = cgfft::ns_before(L, st, rm), r = cgfft::radix_at(L, st, rm);
      const int off = cgfft::stage_tw_offset(L, ns, r);
      const int rp = cgfft::stage_rp(r), step = L / (ns * r);
      for (int jm = 0; jm < ns; jm++)
        for (int i = 0; i < rp; i++)
          h[off + jm * rp + i] = i + 1 < r ? h[jm * (i + 1) * step] : make_float2(0.0f, 0.0f);
      const int offt = cgfft::stage_twt_offset(L, ns, r);
      for (int i = 1; i < r; i++)
        for (int jm = 0; jm < ns; jm++) h[offt + (i - 1) * ns + jm] = h[jm * i * step];
    }
  }
}

}  // namespace

int pm_set_z_gather(int mode) {
  if (mode < -1 || mode > 2) return -1;
  g_zmode.store(mode);
  return 0;
}

int pm_set_x_gather(int mode) {
  if (mode < -1 || mode > 1) return -1;
  g_xmode.store(mode);
  return 0;
}

bool pm_force_deposit_binned() { return fused_deposit(); }

// Interpolation of the force step: 0 from the force meshes (the default), 1
// from the z c2r's shared tiles.  COLAGPU_FUSED_INTERP=0/1 overrides.  The
// default stays the force meshes: at 768^3 the fused form measured 1.04 ms
// per component (the tiles overlap by two lines, 14 % more transform work,
// and the gathers from shared memory add issue slots) plus 0.35 ms of
// binning and 0.42 ms of sums, against 0.81 ms per k_zi_sw and 1.05 ms for
// k_interp: 10.76 against 10.50 ms per step.
std::atomic<int> g_fint{-1};

bool pm_force_interp_binned() {
  static const int forced = [] {
    const char* e = getenv("COLAGPU_FUSED_INTERP");
    return e ? atoi(e) : -1;
  }();
  const int m = forced >= 0 ? forced : g_fint.load();
  return m == 1;
}

int pm_set_force_interp(int mode) {
  if (mode < -1 || mode > 1) return -1;
  g_fint.store(mode);
  return 0;
}

int pm_set_force_deposit(int mode) {
  if (mode < -1 || mode > 1) return -1;
  g_fdep.store(mode);
  return 0;
}

cudaError_t pm_colbins_reserve(PmPlan* p, long long n) {
  const long long keys = (long long)(p->N + 1) * p->N + 1;
  cudaError_t e = cudaSuccess;
  if (keys > p->cb_keys) {
    cudaFree(p->cb_cnt);
    cudaFree(p->cb_bsum);
    p->cb_cnt = nullptr;
    p->cb_bsum = nullptr;
    p->cb_keys = 0;
    e = cudaMalloc(&p->cb_cnt, sizeof(unsigned) * (keys + 1));
    if (e == cudaSuccess)
      e = cudaMalloc(&p->cb_bsum, sizeof(unsigned) * (cgscan::scratch_entries(keys) + 1));
    if (e != cudaSuccess) return e;
    p->cb_keys = keys;
  }
  if (n > p->cb_cap) {
    cudaFree(p->cb_rank);
    cudaFree(p->cb_ent);
    p->cb_rank = nullptr;
    p->cb_ent = nullptr;
    p->cb_cap = 0;
    cudaFree(p->cb_part);
    p->cb_part = nullptr;
    e = cudaMalloc(&p->cb_rank, sizeof(unsigned) * 2 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&p->cb_ent, sizeof(float4) * 2 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&p->cb_part, sizeof(float) * 12 * (size_t)n);
    if (e != cudaSuccess) return e;
    p->cb_cap = n;
  }
  return e;
}

template <int V>
void deposit_variant(PmPlan* p, const float* const x[3], long long n, cudaStream_t st) {
  constexpr DepCfg c = kDepCfg[V];
  prof_mark(st, CG_ST_DEPOSIT);
  if constexpr (c.chunk == 0) {
    k_deposit<<<grid_for(n), T, 0, st>>>(x[0], x[1], x[2], n, p->dens, p->N, p->scale, p->wpar,
                                         p->x_right, p->shiftx, p->err);
  } else {
    k_deposit_box<c.chunk, c.vmax><<<(unsigned)((n + c.chunk - 1) / c.chunk), T,
                                     sizeof(float) * c.vmax, st>>>(
        x[0], x[1], x[2], n, p->dens, p->N, p->scale, p->wpar, p->x_right, p->shiftx, p->err);
  }
}

template <int V>
cudaError_t deposit_smem_attr() {
  constexpr DepCfg c = kDepCfg[V];
  if constexpr (c.chunk == 0) return cudaSuccess;
  else return set_smem((const void*)k_deposit_box<c.chunk, c.vmax>, sizeof(float) * c.vmax);
}

// The CIC scatter into the mesh (which holds -1) with deposit variant v.
void launch_deposit(PmPlan* p, const float* const x[3], long long n, int v, cudaStream_t st) {
  static const cudaError_t attr = [] {
    cudaError_t e = deposit_smem_attr<0>();
    if (e == cudaSuccess) e = deposit_smem_attr<1>();
    if (e == cudaSuccess) e = deposit_smem_attr<2>();
    if (e == cudaSuccess) e = deposit_smem_attr<3>();
    if (e == cudaSuccess) e = deposit_smem_attr<4>();
    return e;
  }();
  (void)attr;
  switch (v) {
    case 1: deposit_variant<1>(p, x, n, st); break;
    case 2: deposit_variant<2>(p, x, n, st); break;
    case 3: deposit_variant<3>(p, x, n, st); break;
    case 4: deposit_variant<4>(p, x, n, st); break;
    case 5: deposit_variant<5>(p, x, n, st); break;
    default: deposit_variant<0>(p, x, n, st);
  }
}

bool pm_supported_mesh(int N) {
  MeshKernels k;
  return get_kernels(N, &k);
}

int pm_num_variants(int N, int* n_green, int* n_fx) {
  MeshKernels k;
  if (!get_kernels(N, &k)) return 0;
  if (n_green) *n_green = n_green_variants(N);
  if (n_fx) *n_fx = n_fx_variants(N);
  return 1;
}

MeshSched pm_get_schedule(int N) { return sched_for(N); }

void pm_set_schedule(int N, MeshSched s) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  g_sched[N] = s;
}

// Best time of each of nvar variants over `rounds` rounds that time every
// variant once in turn (after one untimed round), so that a clock or power
// state that changes during the tuning does not favour a late variant.
template <class F>
static cudaError_t interleaved_best(cudaStream_t st, int nvar, int rounds, F launch, float* ms) {
  cudaEvent_t a, b;
  cudaError_t e = cudaEventCreate(&a);
  if (e != cudaSuccess) return e;
  if ((e = cudaEventCreate(&b)) != cudaSuccess) {
    cudaEventDestroy(a);
    return e;
  }
  for (int v = 0; v < nvar; v++) {
    ms[v] = 1e30f;
    launch(v);
  }
  for (int r = 0; r < rounds && e == cudaSuccess; r++) {
    for (int v = 0; v < nvar && e == cudaSuccess; v++) {
      cudaEventRecord(a, st);
      launch(v);
      cudaEventRecord(b, st);
      e = cudaEventSynchronize(b);
      float t = 0.0f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
      if (e == cudaSuccess && t < ms[v]) ms[v] = t;
    }
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return e;
}

cudaError_t pm_autotune(PmPlan* p, cudaStream_t st, MeshSched* best, float* ms_green,
                        float* ms_fx) {
  const int N = p->N;
  int ng = 0, nf = 0;
  if (!pm_num_variants(N, &ng, &nf)) return cudaErrorInvalidValue;
  cudaError_t e = set_all_smem(N);
  // defined, non-zero contents for the timed passes (the values do not
  // change the work); every spectrum is larger than L2 from 512 up
  const size_t s4 = p->spec_bytes / 16;
  if (e == cudaSuccess) {
    prof_mark(st, CG_ST_OTHER);
    k_fill<<<grid_for((long long)s4), T, 0, st>>>(reinterpret_cast<float4*>(p->spec), s4, 0.5f);
    for (int a = 0; a < 3; a++) {
      prof_mark(st, CG_ST_OTHER);
      k_fill<<<grid_for((long long)s4), T, 0, st>>>(reinterpret_cast<float4*>(p->gsp[a]), s4,
                                                    0.25f);
    }
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return e;
  constexpr int kRounds = 5;
  MeshSched out;
  float tg[PM_NUM_GREEN_VARIANTS], tx[PM_NUM_FX_VARIANTS];
  MeshKernels kg[PM_NUM_GREEN_VARIANTS], kx[PM_NUM_FX_VARIANTS];
  for (int v = 0; v < ng; v++) kernels_with(N, MeshSched{v, 0}, &kg[v]);
  for (int v = 0; v < nf; v++) kernels_with(N, MeshSched{0, v}, &kx[v]);
  e = interleaved_best(st, ng, kRounds, [&](int v) {
    const MeshKernels& k = kg[v];
    prof_mark(st, CG_ST_OTHER);
    k.green<<<(N / 2 + 1) * N / k.byg, k.tg, k.sm_green, st>>>(p->spec, p->gsp[1], p->gsp[2],
                                                             p->twN, p->f1, GreenMods{});
  }, tg);
  // time the gather the plan uses (its TMA maps, kernel parameters, are
  // encoded on the host for each variant's columns per CTA)
  if (e == cudaSuccess)
    e = interleaved_best(st, nf, kRounds, [&](int v) {
      const MeshKernels& k = kx[v];
      const bool sw = x_maps_for(p, k.tk);
      prof_mark(st, CG_ST_OTHER);
      if (sw)
        k.fxi_x_sw<<<dim3(N / k.tk, N / 2 + 1), T, k.sm_fx_sw, st>>>(p->xtm[2], p->gsp[0],
                                                                     p->twN, nullptr, p->err);
      else
        k.fxi_x<<<dim3(N / k.tk, N / 2 + 1), T, k.sm_fx, st>>>(p->gsp[2], p->gsp[0], p->twN,
                                                               nullptr);
    }, tx);
  if (e != cudaSuccess) return e;
  float tbest = 1e30f;
  for (int v = 0; v < ng; v++) {
    if (ms_green) ms_green[v] = tg[v];
    if (tg[v] < tbest) { tbest = tg[v]; out.green = v; }
  }
  tbest = 1e30f;
  for (int v = 0; v < nf; v++) {
    if (ms_fx) ms_fx[v] = tx[v];
    if (tx[v] < tbest) { tbest = tx[v]; out.fx = v; }
  }
  *best = out;
  return e;
}

bool encode_zi_maps(PmPlan* p, bool swizzled);
bool encode_x_maps(PmPlan* p, int tk);

cudaError_t pm_plan_alloc(PmPlan* p, int N, int factor, float L) {
  memset(p, 0, sizeof(*p));
  p->kfilt_cur = -1;
  MeshKernels k;
  if (!get_kernels(N, &k)) return cudaErrorInvalidValue;
  p->N = N;
  p->factor = factor;
  p->L = L;
  // float constants exactly as the reference forms them
  p->scale = (float)N / L;                                        // pm.c:215
  p->wpar = (float)pow((double)factor, 3.0);                      // pm.c:216
  {
    const float sc = (float)(2.0 * 3.1415926535897932384626433832795 / (double)L);  // pm.c:315
    p->f1 = (float)(-1.0 / pow((double)N, 3.0) / (double)sc);                        // pm.c:317
  }
  {
    const float eps = L / (float)N;                               // pm.c:422
    p->x_right = L / (float)N * (float)N - eps;                   // pm.c:423
    p->shiftx = -L;                                               // pm.c:434
  }
  const size_t nh = (size_t)(N / 2 + 1);
  p->mesh_bytes = sizeof(float) * (size_t)N * N * N;
  p->spec_bytes = sizeof(float2) * nh * N * N;
  cudaError_t e;
#define CG_TRY(x) do { e = (x); if (e != cudaSuccess) { pm_plan_free(p); return e; } } while (0)
  CG_TRY(cudaMalloc(&p->dens, p->mesh_bytes));
  CG_TRY(cudaMalloc(&p->spec, p->spec_bytes));
  for (int a = 0; a < 3; a++) {
    CG_TRY(cudaMalloc(&p->gsp[a], p->spec_bytes));
    CG_TRY(cudaMalloc(&p->fmesh[a], p->mesh_bytes));
  }
  const size_t lenN = twiddle_table_len(N), lenH = twiddle_table_len(N / 2);
  CG_TRY(cudaMalloc(&p->twN, sizeof(float2) * lenN));
  CG_TRY(cudaMalloc(&p->twH, sizeof(float2) * lenH));
  CG_TRY(cudaMalloc(&p->dsum, sizeof(double)));
  CG_TRY(cudaMalloc(&p->pk_acc, sizeof(double) * 3 * N));
  CG_TRY(cudaMalloc(&p->err, sizeof(unsigned)));
  {
    float2* h = (float2*)malloc(sizeof(float2) * (lenN > lenH ? lenN : lenH));
    twiddle_table(h, N);
    CG_TRY(cudaMemcpy(p->twN, h, sizeof(float2) * lenN, cudaMemcpyHostToDevice));
    twiddle_table(h, N / 2);
    CG_TRY(cudaMemcpy(p->twH, h, sizeof(float2) * lenH, cudaMemcpyHostToDevice));
    free(h);
  }
  CG_TRY(cudaMemset(p->dsum, 0, sizeof(double)));
  CG_TRY(cudaMemset(p->err, 0, sizeof(unsigned)));
  CG_TRY(set_all_smem(N));
  bool zexplicit = false;
  const int zmode = z_gather_mode(N, &zexplicit);
  p->zsw_ok = zmode == 2 && encode_zi_maps(p, true);
  p->ztm_ok = zmode == 1 && encode_zi_maps(p, false);
  // a TMA gather that was asked for explicitly and cannot be set up is an
  // error; by default the plan falls back to the cp.async gather
  if (zexplicit && zmode > 0 && !p->zsw_ok && !p->ztm_ok) {
    pm_plan_free(p);
    return cudaErrorNotSupported;
  }
  bool xexplicit = false;
  p->xsw_ok = x_gather_mode(N, &xexplicit) == 1 && encode_x_maps(p, k.tk);
  if (xexplicit && x_gather_mode(N, &xexplicit) == 1 && !p->xsw_ok) {
    pm_plan_free(p);
    return cudaErrorNotSupported;
  }
#undef CG_TRY
  return cudaSuccess;
}

cudaError_t mesh_fft_alloc(MeshFFT* f, int N) {
  memset(f, 0, sizeof(*f));
  MeshKernels k;
  if (!get_kernels(N, &k)) return cudaErrorInvalidValue;
  f->N = N;
  const size_t lenN = twiddle_table_len(N), lenH = twiddle_table_len(N / 2);
  cudaError_t e = cudaMalloc(&f->twN, sizeof(float2) * lenN);
  if (e == cudaSuccess) e = cudaMalloc(&f->twH, sizeof(float2) * lenH);
  if (e == cudaSuccess) e = cudaMalloc(&f->dsum, sizeof(double));
  if (e == cudaSuccess) {
    float2* h = (float2*)malloc(sizeof(float2) * (lenN > lenH ? lenN : lenH));
    twiddle_table(h, N);
    e = cudaMemcpy(f->twN, h, sizeof(float2) * lenN, cudaMemcpyHostToDevice);
    twiddle_table(h, N / 2);
    if (e == cudaSuccess) e = cudaMemcpy(f->twH, h, sizeof(float2) * lenH, cudaMemcpyHostToDevice);
    free(h);
  }
  if (e == cudaSuccess) e = set_all_smem(N);
  if (e != cudaSuccess) mesh_fft_free(f);
  return e;
}

void mesh_fft_free(MeshFFT* f) {
  cudaFree(f->twN);
  cudaFree(f->twH);
  cudaFree(f->dsum);
  memset(f, 0, sizeof(*f));
}

cudaError_t mesh_r2c(const MeshFFT* f, const float* real, float2* spec, cudaStream_t st) {
  MeshKernels k;
  if (!get_kernels(f->N, &k)) return cudaErrorInvalidValue;
  const int N = f->N;
  prof_mark(st, CG_ST_FZ);
  k.fz<<<dim3(N / TY, N), T, k.sm_fz, st>>>(real, spec, f->twH, f->twN, f->dsum);
  prof_mark(st, CG_ST_OTHER);
  k.fyf<<<(N / 2 + 1) * N / BY, T, k.sm_fy, st>>>(spec, f->twN);
  prof_mark(st, CG_ST_FX_FWD);
  k.fxf<<<dim3(N / k.tk, N / 2 + 1), T, k.sm_fx, st>>>(spec, spec, f->twN, nullptr);
  return cudaGetLastError();
}

cudaError_t mesh_c2r(const MeshFFT* f, float2* spec, float* real, cudaStream_t st) {
  MeshKernels k;
  if (!get_kernels(f->N, &k)) return cudaErrorInvalidValue;
  const int N = f->N;
  prof_mark(st, CG_ST_FX_INV);
  k.fxi<<<dim3(N / k.tk, N / 2 + 1), T, k.sm_fx, st>>>(spec, spec, f->twN, nullptr);
  prof_mark(st, CG_ST_OTHER);
  k.fyi<<<(N / 2 + 1) * N / BY, T, k.sm_fy, st>>>(spec, f->twN);
  prof_mark(st, CG_ST_ZI);
  k.zi<<<dim3(N / TY, N), T, k.sm_zi, st>>>(spec, real, f->twH, f->twN);
  return cudaGetLastError();
}

cudaError_t pm_set_filters(PmPlan* p, const float* knots, int n, int nsets) {
  p->kfilt_cur = -1;
  if (n <= 1 || nsets <= 0 || !knots) {
    p->kfilt_n = p->kfilt_sets = 0;
    return cudaSuccess;
  }
  const size_t need = (size_t)n * nsets;
  if (need > p->kfilt_cap) {
    cudaFree(p->kfilt);
    p->kfilt = nullptr;
    p->kfilt_cap = 0;
    cudaError_t e = cudaMalloc(&p->kfilt, sizeof(float) * need);
    if (e != cudaSuccess) return e;
    p->kfilt_cap = need;
  }
  // a plain (synchronous) copy: done once, before the run that uses it
  cudaError_t e = cudaMemcpy(p->kfilt, knots, sizeof(float) * need, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  p->kfilt_n = n;
  p->kfilt_sets = nsets;
  p->kfilt_cur = 0;
  p->kfilt_inv_dn = (float)((n - 1) / (sqrt(3.0) * p->N / 2.0));
  return cudaSuccess;
}

cudaError_t pm_set_force_kernel(PmPlan* p, int gradient, int laplacian, int deconvolve) {
  if (gradient == 0 && laplacian == 0 && deconvolve == 0) {
    cudaFree(p->ktab);
    p->ktab = nullptr;
    return cudaSuccess;
  }
  const int N = p->N;
  std::vector<float> t(3 * (size_t)N);
  for (int i = 0; i < N; i++) {
    const double s = i <= N / 2 ? i : i - N;
    const double w = M_PI * s / N;               // half the mesh phase k h / 2
    // gradient: the transfer function of the difference operator, in units
    // of the fundamental (h = L / N, k = 2 pi s / L, k h = 2 w)
    double g = s;
    if (gradient == 2) g = N / (2 * M_PI) * sin(2 * w);
    if (gradient == 4) g = N / (2 * M_PI) * (8 * sin(2 * w) - sin(4 * w)) / 6;
    // Laplacian: s^2, or the 3-point second difference's (N / pi sin w)^2
    const double l = laplacian ? (N / M_PI * sin(w)) * (N / M_PI * sin(w)) : s * s;
    // CIC window per axis sinc^2(w); divided out `deconvolve` times
    const double sinc = i == 0 ? 1.0 : sin(w) / w;
    const double c = pow(sinc * sinc, -(double)deconvolve);
    t[i] = (float)g;
    t[N + i] = (float)l;
    t[2 * N + i] = (float)c;
  }
  if (!p->ktab) {
    cudaError_t e = cudaMalloc(&p->ktab, sizeof(float) * t.size());
    if (e != cudaSuccess) return e;
  }
  return cudaMemcpy(p->ktab, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice);
}

bool pm_use_filter(PmPlan* p, int set) {
  if (set >= p->kfilt_sets) return false;
  p->kfilt_cur = set < 0 ? -1 : set;
  return true;
}

void pm_plan_free(PmPlan* p) {
  cudaFree(p->kfilt);
  cudaFree(p->ktab);
  cudaFree(p->dens);
  cudaFree(p->spec);
  for (int a = 0; a < 3; a++) {
    cudaFree(p->gsp[a]);
    cudaFree(p->fmesh[a]);
  }
  cudaFree(p->twN);
  cudaFree(p->twH);
  cudaFree(p->dsum);
  cudaFree(p->pk_acc);
  cudaFree(p->err);
  cudaFree(p->cb_cnt);
  cudaFree(p->cb_bsum);
  cudaFree(p->cb_rank);
  cudaFree(p->cb_ent);
  cudaFree(p->cb_part);
  memset(p, 0, sizeof(*p));
}

cudaError_t pm_deposit(PmPlan* p, const float* const x[3], long long n, cudaStream_t st) {
  // scatter with global float atomics into a mesh filled with -1
  const size_t n4 = (size_t)p->N * p->N * p->N / 4;
  if (!p->dens_reset) {   // else the last z r2c left the mesh at -1 already
    prof_mark(st, CG_ST_FILL);
    k_fill<<<grid_for((long long)n4), T, 0, st>>>(reinterpret_cast<float4*>(p->dens), n4, -1.0f);
  }
  p->dens_reset = false;
  p->dens_stale = false;
  if (n > 0) {
    static const bool plain = getenv("COLAGPU_DEPOSIT") && getenv("COLAGPU_DEPOSIT")[0] == 'p';
    launch_deposit(p, x, n, plain ? PM_NUM_DEP_VARIANTS - 1 : sched_for(p->N).dep, st);
  }
  return cudaGetLastError();
}

// Forward x pass of the spectrum (in place).
void launch_fx_fwd(PmPlan* p, const MeshKernels& k, cudaStream_t st) {
  const int N = p->N;
  prof_mark(st, CG_ST_FX_FWD);
  if (x_maps_for(p, k.tk))
    k.fxf_sw<<<dim3(N / k.tk, N / 2 + 1), T, k.sm_fx_sw, st>>>(p->xtm[0], p->spec, p->twN,
                                                               nullptr, p->err);
  else
    k.fxf<<<dim3(N / k.tk, N / 2 + 1), T, k.sm_fx, st>>>(p->spec, p->spec, p->twN, nullptr);
}

cudaError_t pm_r2c(PmPlan* p, cudaStream_t st) {
  MeshKernels k;
  get_kernels(p->N, &k);
  const int N = p->N;
  cudaMemsetAsync(p->dsum, 0, sizeof(double), st);
  prof_mark(st, CG_ST_FZ);
  if (p->keep_dens)
    k.fz<<<dim3(N / TY, N), T, k.sm_fz, st>>>(p->dens, p->spec, p->twH, p->twN, p->dsum);
  else
    k.fz_reset<<<dim3(N / TY, N), T, k.sm_fz, st>>>(p->dens, p->spec, p->twH, p->twN, p->dsum);
  p->dens_reset = !p->keep_dens;
  launch_fx_fwd(p, k, st);
  return cudaGetLastError();
}

void launch_zi(const PmPlan* p, const MeshKernels& k, int a, cudaStream_t st);

// The column bins of the particles' clouds for this force step: counts with
// warp-aggregated ranks, their prefix sum, the entries.  With f, the
// forces of particles without a primary cloud are set to 0 (the
// interpolation from the bins writes the others).
cudaError_t pm_build_bins(PmPlan* p, const float* const x[3], long long n, float* const* f,
                          cudaStream_t st) {
  const int N = p->N;
  const long long keys = (long long)(N + 1) * N + 1;
  if (n > p->cb_cap || keys > p->cb_keys) return cudaErrorInvalidValue;
  // the counts, and past them the count of buffer copies outside key row 0
  cudaMemsetAsync(p->cb_cnt, 0, sizeof(unsigned) * (keys + 1), st);
  if (n > 0) {
    prof_mark(st, CG_ST_DEPOSIT);
    k_col_count<<<grid_for(n), T, 0, st>>>(x[0], x[1], x[2], n, N, p->scale, p->x_right,
                                           p->shiftx, p->cb_cnt, p->cb_rank, p->cb_cap, p->err,
                                           f ? f[0] : nullptr, f ? f[1] : nullptr,
                                           f ? f[2] : nullptr);
  }
  cgscan::exclusive(p->cb_cnt, p->cb_cnt, keys, p->cb_bsum, nullptr, CG_ST_DEPOSIT, st);
  if (n > 0) {
    prof_mark(st, CG_ST_DEPOSIT);
    k_col_scatter<<<grid_for(n), T, 0, st>>>(x[0], x[1], x[2], n, N, p->scale, p->x_right,
                                             p->shiftx, p->cb_cnt, p->cb_rank, p->cb_cap,
                                             p->cb_ent);
  }
  return cudaGetLastError();
}

// The force step's deposit and r2c through the column bins (built): k_dfz
// (deposit in shared memory + r2c along z) and the forward x pass.  The
// density mesh is left untouched (dens_stale).
cudaError_t pm_binned_r2c(PmPlan* p, cudaStream_t st) {
  MeshKernels k;
  get_kernels(p->N, &k);
  const int N = p->N;
  cudaMemsetAsync(p->dsum, 0, sizeof(double), st);
  prof_mark(st, CG_ST_FZ);
  k.dfz<<<dim3(N / TY, N), T, k.sm_fz, st>>>(p->cb_ent, p->cb_cnt, p->spec, p->twH, p->twN,
                                             p->dsum, p->scale, p->wpar);
  p->dens_reset = false;
  p->dens_stale = true;
  launch_fx_fwd(p, k, st);
  return cudaGetLastError();
}

// The z c2r of the three components fused with the interpolation (bins
// built, spectra gsp[0..2] inverse-transformed along x), then the sums.
cudaError_t pm_zi_interp(PmPlan* p, long long n, float* const f[3], cudaStream_t st) {
  MeshKernels k;
  get_kernels(p->N, &k);
  const int N = p->N;
  const long long cap2 = 2 * p->cb_cap;
  for (int a = 0; a < 3; a++) {
    prof_mark(st, CG_ST_ZI);
    k.zip<<<dim3(zip_tiles(N), N), T, k.sm_zi_sw, st>>>(
        p->ztm[a], p->gsp[a], p->cb_ent, p->cb_cnt, p->cb_part + 2 * a * cap2,
        p->cb_part + (2 * a + 1) * cap2, p->twH, p->twN, p->scale, p->err);
  }
  if (n > 0) {
    prof_mark(st, CG_ST_INTERP);
    k_interp_sum<<<grid_for(n), T, 0, st>>>(p->cb_ent, p->cb_cnt, N, p->scale, p->cb_part, cap2,
                                            f[0], f[1], f[2]);
    prof_mark(st, CG_ST_INTERP);
    k_interp_copies<<<cg_grid((long long)N * N, 4), T, 0, st>>>(p->cb_ent, p->cb_cnt, N,
                                                                p->scale, p->cb_part, cap2,
                                                                f[0], f[1], f[2]);
  }
  p->fmesh_stale = true;
  return cudaGetLastError();
}

cudaError_t pm_force_mesh(PmPlan* p, int a, cudaStream_t st) {
  if (!p->fmesh_stale) return cudaSuccess;
  MeshKernels k;
  get_kernels(p->N, &k);
  prof_mark(st, CG_ST_ZI);
  launch_zi(p, k, a, st);
  return cudaGetLastError();
}

// z c2r of component a: gsp[a] -> fmesh[a], by the TMA gather where the
// plan holds its tensor maps
void launch_zi(const PmPlan* p, const MeshKernels& k, int a, cudaStream_t st) {
  const int N = p->N;
  const dim3 gz(N / TY, N);
  if (p->zsw_ok)
    k.zi_sw<<<gz, T, k.sm_zi_sw, st>>>(p->ztm[a], p->fmesh[a], p->twH, p->twN, p->err);
  else if (p->ztm_ok)
    k.zi_tma<<<gz, T, k.sm_zi_tma, st>>>(p->ztm[a], p->fmesh[a], p->twH, p->twN, p->err);
  else
    k.zi<<<gz, T, k.sm_zi, st>>>(p->gsp[a], p->fmesh[a], p->twH, p->twN);
}

// Tensor maps of the three spectra for k_zi_tma or (swizzled) k_zi_sw (see
// there); false when the driver's encoder is unavailable or refuses the
// layout.
bool encode_zi_maps(PmPlan* p, bool swizzled) {
  static PFN_cuTensorMapEncodeTiled_v12000 enc = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  if (!enc) return false;
  const int N = p->N;
  const int nb = (N / 2 + 1 + 255) / 256;
  // rows per box: the landing form splits the kz rows evenly; the swizzled
  // form rounds up to a multiple of 8 rows (every box 1024-byte aligned)
  int kr = (N / 2 + 1 + nb - 1) / nb;
  if (swizzled) kr = (kr + 7) / 8 * 8;
  if (kr > 256) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)2 * N, (cuuint64_t)N, (cuuint64_t)(N / 2 + 1)};
  const cuuint64_t strides[2] = {(cuuint64_t)N * 8, (cuuint64_t)N * N * 8};
  const cuuint32_t box[3] = {2 * TY, 1, (cuuint32_t)kr};   // 2 TY floats = 128 bytes
  const cuuint32_t es[3] = {1, 1, 1};
  for (int a = 0; a < 3; a++) {
    if (enc(&p->ztm[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)p->gsp[a], dims, strides, box,
            es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            swizzled ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

// Tensor maps of the x pass's inputs (spec, gsp[1], gsp[2]) for k_fx_sw
// with tk columns per CTA: floats (2N, N, N/2+1), box (2 tk, N / nbox, 1),
// swizzled like the tile.
bool encode_x_maps(PmPlan* p, int tk) {
  static PFN_cuTensorMapEncodeTiled_v12000 enc = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  if (!enc) return false;
  const int N = p->N;
  const int nb = (N + 255) / 256;
  if (N % nb || (N / nb) % 8 || (tk != 8 && tk != 16)) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)2 * N, (cuuint64_t)N, (cuuint64_t)(N / 2 + 1)};
  const cuuint64_t strides[2] = {(cuuint64_t)N * 8, (cuuint64_t)N * N * 8};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * tk), (cuuint32_t)(N / nb), 1};
  const cuuint32_t es[3] = {1, 1, 1};
  float2* const src[3] = {p->spec, p->gsp[1], p->gsp[2]};
  for (int a = 0; a < 3; a++) {
    if (enc(&p->xtm[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)src[a], dims, strides, box,
            es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            tk == 8 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  p->xtm_tk = tk;
  return true;
}

// The x pass's TMA maps for the columns per CTA of the schedule in use (a
// schedule may change after the plan exists); false: load directly.
bool x_maps_for(PmPlan* p, int tk) {
  if (!p->xsw_ok) return false;
  if (p->xtm_tk != tk && !encode_x_maps(p, tk)) {
    p->xsw_ok = false;
    return false;
  }
  return true;
}

// The Green pass and the inverse x passes; with zi, each component's z c2r
// into its force mesh after its x pass.
static cudaError_t green_x_zi(PmPlan* p, cudaStream_t st, bool zi) {
  MeshKernels k;
  get_kernels(p->N, &k);
  const int N = p->N;
  // gsp[1] <- y component, gsp[2] <- the shared x/z spectrum
  prof_mark(st, CG_ST_GREEN);
  const GreenMods gm{p->kfilt_cur >= 0 ? p->kfilt + (size_t)p->kfilt_cur * p->kfilt_n : nullptr,
                     p->kfilt_n, p->kfilt_inv_dn, p->ktab};
  (gm.t || gm.tab ? k.green_mods : k.green)<<<(N / 2 + 1) * N / k.byg, k.tg, k.sm_green, st>>>(
      p->spec, p->gsp[1], p->gsp[2], p->twN, p->f1, gm);
  const dim3 gx(N / k.tk, N / 2 + 1);
  const bool xsw = x_maps_for(p, k.tk);
  // x: n_x * gsp[2] -> gsp[0] (gsp[2] is still needed for z)
  prof_mark(st, CG_ST_FX_INV);
  if (xsw)
    k.fxi_x_sw<<<gx, T, k.sm_fx_sw, st>>>(p->xtm[2], p->gsp[0], p->twN, p->ktab, p->err);
  else
    k.fxi_x<<<gx, T, k.sm_fx, st>>>(p->gsp[2], p->gsp[0], p->twN, p->ktab);
  if (zi) {
    prof_mark(st, CG_ST_ZI);
    launch_zi(p, k, 0, st);
  }
  // y: in place
  prof_mark(st, CG_ST_FX_INV);
  if (xsw)
    k.fxi_sw<<<gx, T, k.sm_fx_sw, st>>>(p->xtm[1], p->gsp[1], p->twN, nullptr, p->err);
  else
    k.fxi<<<gx, T, k.sm_fx, st>>>(p->gsp[1], p->gsp[1], p->twN, nullptr);
  if (zi) {
    prof_mark(st, CG_ST_ZI);
    launch_zi(p, k, 1, st);
  }
  // z: n_z * gsp[2], in place
  prof_mark(st, CG_ST_FX_INV);
  if (xsw)
    k.fxi_z_sw<<<gx, T, k.sm_fx_sw, st>>>(p->xtm[2], p->gsp[2], p->twN, p->ktab, p->err);
  else
    k.fxi_z<<<gx, T, k.sm_fx, st>>>(p->gsp[2], p->gsp[2], p->twN, p->ktab);
  if (zi) {
    prof_mark(st, CG_ST_ZI);
    launch_zi(p, k, 2, st);
  }
  return cudaGetLastError();
}

cudaError_t pm_green_c2r(PmPlan* p, cudaStream_t st) {
  p->fmesh_stale = false;
  return green_x_zi(p, st, true);
}

cudaError_t pm_interp(PmPlan* p, const float* const x[3], long long n, float* const f[3],
                      cudaStream_t st) {
  if (n > 0) {
    prof_mark(st, CG_ST_INTERP);
    k_interp<<<cg_grid(n, kInterpCtasPerSm), T, 0, st>>>(x[0], x[1], x[2], n, p->fmesh[0], p->fmesh[1],
                                        p->fmesh[2], f[0], f[1], f[2], p->N, p->scale,
                                        p->x_right, p->shiftx, 0, p->N);
  }
  return cudaGetLastError();
}

// ------------------------------------------------ slab decomposition
// One realization's PM force split over ranks by x slabs of mesh planes,
// the reference's MPI decomposition (comm.c:35-111, pm.c:416-532) with the
// exchanges left to the caller.  Every rank holds full-size meshes; rank r
// works on planes [x0, x0 + nx) in real space and on kz planes
// [kz0, kz0 + nkz) of the spectra.  Particles within one cell of a slab's
// upper edge act on the next slab through buffer copies, as in
// send_buffer_positions / add_buffer_forces: the owner sends their
// positions (shifted by -L across the periodic face), the next rank deposits
// them and interpolates their forces, and the owner adds those forces to its
// particles'.  The copies inside the kernels are switched off
// (x_right = +inf) and each rank reads only its own planes.

// Signed wavenumber index table (n <= N/2 ? n : n - N), the n_z factor of
// the z component's inverse x pass from an offset kz.
static cudaError_t sgn_table(PmPlan* p, const float** out) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, float*> tabs;   // (device, N)
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = tabs.find({dev, p->N});
  if (it == tabs.end()) {
    std::vector<float> h(p->N);
    for (int i = 0; i < p->N; i++) h[i] = (float)(i <= p->N / 2 ? i : i - p->N);
    float* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(float) * p->N);
    if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), sizeof(float) * p->N, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    it = tabs.emplace(std::make_pair(dev, p->N), d).first;
  }
  *out = it->second;
  return cudaSuccess;
}

cudaError_t pm_slab_density(PmPlan* p, int x0, int nx, const float* const x[3], long long n,
                            const float* const bx[3], long long nb, cudaStream_t st) {
  MeshKernels k;
  if (!get_kernels(p->N, &k)) return cudaErrorInvalidValue;
  const int N = p->N;
  if (x0 < 0 || nx < 1 || x0 + nx > N) return cudaErrorInvalidValue;
  const size_t plane = (size_t)N * N;
  const size_t n4 = plane * nx / 4;
  prof_mark(st, CG_ST_FILL);
  k_fill<<<grid_for((long long)n4), T, 0, st>>>(reinterpret_cast<float4*>(p->dens + x0 * plane),
                                               n4, -1.0f);
  PmPlan q = *p;
  q.x_right = INFINITY;      // the buffer copies are deposited by the next rank
  if (n > 0) launch_deposit(&q, x, n, sched_for(N).dep, st);
  if (nb > 0) {
    prof_mark(st, CG_ST_DEPOSIT);
    k_deposit<<<grid_for(nb), T, 0, st>>>(bx[0], bx[1], bx[2], nb, p->dens, N, p->scale,
                                          p->wpar, INFINITY, 0.0f, p->err);
  }
  cudaMemsetAsync(p->dsum, 0, sizeof(double), st);
  prof_mark(st, CG_ST_FZ);
  k.fz<<<dim3(N / TY, nx), T, k.sm_fz, st>>>(p->dens + x0 * plane, p->spec + (size_t)x0 * N,
                                             p->twH, p->twN, p->dsum);
  p->dens_reset = false;
  p->dens_stale = true;       // only this slab's planes hold the density
  p->fmesh_stale = false;
  return cudaGetLastError();
}

cudaError_t pm_slab_kspace(PmPlan* p, int kz0, int nkz, cudaStream_t st) {
  MeshKernels k;
  if (!get_kernels(p->N, &k)) return cudaErrorInvalidValue;
  const int N = p->N;
  if (kz0 < 0 || nkz < 1 || kz0 + nkz > N / 2 + 1) return cudaErrorInvalidValue;
  const float* sgn = nullptr;
  cudaError_t e = sgn_table(p, &sgn);
  if (e != cudaSuccess) return e;
  const size_t off = (size_t)kz0 * N * N;
  const dim3 gx(N / k.tk, nkz);
  prof_mark(st, CG_ST_FX_FWD);
  k.fxf<<<gx, T, k.sm_fx, st>>>(p->spec + off, p->spec + off, p->twN, nullptr);
  prof_mark(st, CG_ST_GREEN);
  GreenMods gm{p->kfilt_cur >= 0 ? p->kfilt + (size_t)p->kfilt_cur * p->kfilt_n : nullptr,
               p->kfilt_n, p->kfilt_inv_dn, p->ktab, kz0};
  (gm.t || gm.tab ? k.green_mods : k.green)<<<nkz * N / k.byg, k.tg, k.sm_green, st>>>(
      p->spec + off, p->gsp[1] + off, p->gsp[2] + off, p->twN, p->f1, gm);
  prof_mark(st, CG_ST_FX_INV);
  k.fxi_x<<<gx, T, k.sm_fx, st>>>(p->gsp[2] + off, p->gsp[0] + off, p->twN, p->ktab);
  prof_mark(st, CG_ST_FX_INV);
  k.fxi<<<gx, T, k.sm_fx, st>>>(p->gsp[1] + off, p->gsp[1] + off, p->twN, nullptr);
  prof_mark(st, CG_ST_FX_INV);
  k.fxi_z<<<gx, T, k.sm_fx, st>>>(p->gsp[2] + off, p->gsp[2] + off, p->twN,
                                  (p->ktab ? p->ktab : sgn) + kz0);
  return cudaGetLastError();
}

cudaError_t pm_slab_c2r(PmPlan* p, int x0, int nx, cudaStream_t st) {
  MeshKernels k;
  if (!get_kernels(p->N, &k)) return cudaErrorInvalidValue;
  const int N = p->N;
  if (x0 < 0 || nx < 1 || x0 + nx > N) return cudaErrorInvalidValue;
  for (int a = 0; a < 3; a++) {
    prof_mark(st, CG_ST_ZI);
    k.zi<<<dim3(N / TY, nx), T, k.sm_zi, st>>>(p->gsp[a] + (size_t)x0 * N,
                                               p->fmesh[a] + (size_t)x0 * N * N, p->twH,
                                               p->twN);
  }
  return cudaGetLastError();
}

cudaError_t pm_slab_interp(PmPlan* p, int x0, int nx, const float* const x[3], long long n,
                           float* const f[3], const float* const bx[3], long long nb,
                           float* const bf[3], cudaStream_t st) {
  const int N = p->N;
  if (x0 < 0 || nx < 1 || x0 + nx > N) return cudaErrorInvalidValue;
  if (n > 0) {
    prof_mark(st, CG_ST_INTERP);
    k_interp<<<cg_grid(n, kInterpCtasPerSm), T, 0, st>>>(x[0], x[1], x[2], n, p->fmesh[0], p->fmesh[1],
                                        p->fmesh[2], f[0], f[1], f[2], N, p->scale, INFINITY,
                                        0.0f, x0, x0 + nx);
  }
  if (nb > 0) {
    prof_mark(st, CG_ST_INTERP);
    k_interp<<<grid_for(nb), T, 0, st>>>(bx[0], bx[1], bx[2], nb, p->fmesh[0], p->fmesh[1],
                                         p->fmesh[2], bf[0], bf[1], bf[2], N, p->scale,
                                         INFINITY, 0.0f, x0, x0 + nx);
  }
  return cudaGetLastError();
}

cudaError_t pm_forces(PmPlan* p, const float* const x[3], long long n, float* const f[3],
                      cudaStream_t st) {
  cudaError_t e;
  // the column bins serve the binned deposit and the interpolation from the
  // z c2r's tiles (which needs the swizzled tiles' tensor maps)
  const bool bdep = !p->keep_dens && fused_deposit();
  const bool bint = pm_force_interp_binned() && p->zsw_ok;
  if (bdep || bint) {
    if ((e = pm_colbins_reserve(p, n)) != cudaSuccess) return e;
    if ((e = pm_build_bins(p, x, n, bint ? f : nullptr, st)) != cudaSuccess) return e;
  }
  if (bdep) {
    if ((e = pm_binned_r2c(p, st)) != cudaSuccess) return e;
  } else {
    if ((e = pm_deposit(p, x, n, st)) != cudaSuccess) return e;
    if ((e = pm_r2c(p, st)) != cudaSuccess) return e;
  }
  if (bint) {
    if ((e = green_x_zi(p, st, false)) != cudaSuccess) return e;
    return pm_zi_interp(p, n, f, st);
  }
  if ((e = pm_green_c2r(p, st)) != cudaSuccess) return e;
  return pm_interp(p, x, n, f, st);
}

cudaError_t pm_tune_deposit(PmPlan* p, const float* const x[3], long long n, cudaStream_t st,
                            int* best, float* ms) {
  if (n < 1) return cudaErrorInvalidValue;
  const size_t n4 = (size_t)p->N * p->N * p->N / 4;
  cudaEvent_t a, b;
  cudaError_t e = cudaEventCreate(&a);
  if (e != cudaSuccess) return e;
  if ((e = cudaEventCreate(&b)) != cudaSuccess) {
    cudaEventDestroy(a);
    return e;
  }
  float tbest = 1e30f;
  int vbest = 0;
  for (int v = 0; v < PM_NUM_DEP_VARIANTS && e == cudaSuccess; v++) {
    float t = 1e30f;
    for (int r = 0; r < 3 && e == cudaSuccess; r++) {
      prof_mark(st, CG_ST_FILL);
      k_fill<<<grid_for((long long)n4), T, 0, st>>>(reinterpret_cast<float4*>(p->dens), n4, -1.0f);
      cudaEventRecord(a, st);
      launch_deposit(p, x, n, v, st);
      cudaEventRecord(b, st);
      e = cudaEventSynchronize(b);
      float tr = 0.0f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&tr, a, b);
      if (e == cudaSuccess && tr < t) t = tr;
    }
    if (ms) ms[v] = t;
    if (e == cudaSuccess && t < tbest) {
      tbest = t;
      vbest = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e == cudaSuccess) e = cudaGetLastError();
  p->dens_reset = false;   // the mesh holds the last timed deposit
  p->dens_stale = false;
  *best = vbest;
  return e;
}

cudaError_t pm_power_spectrum(PmPlan* p, const float* const x[3], long long n, int nbins,
                              int deconv, double* acc, cudaStream_t st) {
  MeshKernels k;
  if (!get_kernels(p->N, &k)) return cudaErrorInvalidValue;
  if (nbins < 1 || nbins > p->N) return cudaErrorInvalidValue;
  const int N = p->N;
  cudaError_t e = pm_deposit(p, x, n, st);
  if (e != cudaSuccess) return e;
  cudaMemsetAsync(p->dsum, 0, sizeof(double), st);
  prof_mark(st, CG_ST_FZ);
  k.fz<<<dim3(N / TY, N), T, k.sm_fz, st>>>(p->dens, p->spec, p->twH, p->twN, p->dsum);
  prof_mark(st, CG_ST_FX_FWD);
  k.fxf<<<dim3(N / k.tk, N / 2 + 1), T, k.sm_fx, st>>>(p->spec, p->spec, p->twN, nullptr);
  prof_mark(st, CG_ST_OTHER);
  k.fyf<<<(N / 2 + 1) * N / BY, T, k.sm_fy, st>>>(p->spec, p->twN);
  cudaMemsetAsync(acc, 0, sizeof(double) * 3 * nbins, st);
  prof_mark(st, CG_ST_OTHER);
  k_pk_bin<<<grid_for((long long)(N / 2 + 1) * N * N), T, sizeof(double) * 3 * nbins, st>>>(
      p->spec, N, nbins, deconv, acc);
  return cudaGetLastError();
}
