// Coarse density grid of a snapshot (coarse_grid.c:17-121 on one process).
//
// CIC mass assignment of the snapshot particles onto an nc^3 grid with the
// reference's weights -- cell ix = floor(x nc/L), left weight
// w = 1 - (x nc/L - ix), periodic neighbours, products w0 w1 w2 formed left
// to right in float (coarse_grid.c:96-121) -- accumulated with float
// atomics, then delta = (ngrid / np_total) rho - 1 (coarse_grid.c:70-74).
// The reference adds in particle order; the atomics add in any order, so
// cells agree to float rounding.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../include/colagpu.h"
#include "../../include/colagpu_dropin.h"
#include "gadget.h"
#include "internal.h"

extern int cg_set_error_from_lpt(int code, const char* msg);
void cg_dropin_error(int code, const char* msg);

namespace {

constexpr int T = CG_THREADS;

// The eight cells and CIC weights of one particle, in the reference's
// corner order and arithmetic (coarse_grid.c:101-120).
__device__ __forceinline__ void cic_corners(const ParticleMinimum& q, float dx_inv, int nc,
                                            int idx[8], float val[8]) {
  int i0[3], i1[3];
  float w[3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const float s = __fmul_rn(q.x[j], dx_inv);
    const int ix = (int)floorf(s);
    w[j] = __fsub_rn(1.0f, __fsub_rn(s, (float)ix));
    // (ix + nc) % nc and (ix + 1 + nc) % nc for ix >= -nc, as the
    // reference; any other ix (a particle far outside the box, NaN)
    // still lands in the grid
    int m = ix % nc;
    if (m < 0) m += nc;
    i0[j] = m;
    i1[j] = m + 1 == nc ? 0 : m + 1;
  }
  const float u0 = __fsub_rn(1.0f, w[0]), u1 = __fsub_rn(1.0f, w[1]), u2 = __fsub_rn(1.0f, w[2]);
  const int a0 = i0[0] * nc, a1 = i1[0] * nc;
  idx[0] = (a0 + i0[1]) * nc + i0[2];  val[0] = __fmul_rn(__fmul_rn(w[0], w[1]), w[2]);
  idx[1] = (a0 + i1[1]) * nc + i0[2];  val[1] = __fmul_rn(__fmul_rn(w[0], u1), w[2]);
  idx[2] = (a0 + i0[1]) * nc + i1[2];  val[2] = __fmul_rn(__fmul_rn(w[0], w[1]), u2);
  idx[3] = (a0 + i1[1]) * nc + i1[2];  val[3] = __fmul_rn(__fmul_rn(w[0], u1), u2);
  idx[4] = (a1 + i0[1]) * nc + i0[2];  val[4] = __fmul_rn(__fmul_rn(u0, w[1]), w[2]);
  idx[5] = (a1 + i1[1]) * nc + i0[2];  val[5] = __fmul_rn(__fmul_rn(u0, u1), w[2]);
  idx[6] = (a1 + i0[1]) * nc + i1[2];  val[6] = __fmul_rn(__fmul_rn(u0, w[1]), u2);
  idx[7] = (a1 + i1[1]) * nc + i1[2];  val[7] = __fmul_rn(__fmul_rn(u0, u1), u2);
}

// Grids up to kSmemCells cells: each CTA accumulates its particles into a
// private copy of the grid in shared memory, then adds the copy to the
// global grid, so the global atomics are one per cell per CTA instead of
// eight per particle on a few thousand addresses.
constexpr int kSmemThreads = 512;
constexpr int kSmemCells = 16384;

__global__ void __launch_bounds__(kSmemThreads) k_coarse_cic_smem(
    const ParticleMinimum* __restrict__ p, long long n, float dx_inv, int nc,
    float* __restrict__ grid) {
  extern __shared__ float sg[];
  const int ng = nc * nc * nc;
  for (int i = threadIdx.x; i < ng; i += kSmemThreads) sg[i] = 0.0f;
  __syncthreads();
  for (long long i = (long long)blockIdx.x * kSmemThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kSmemThreads) {
    int idx[8];
    float val[8];
    cic_corners(p[i], dx_inv, nc, idx, val);
#pragma unroll
    for (int c = 0; c < 8; c++) atomicAdd(&sg[idx[c]], val[c]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < ng; i += kSmemThreads) {
    const float v = sg[i];
    if (v != 0.0f) atomicAdd(grid + i, v);
  }
}

// Larger grids: eight global atomics per particle, spread over many cells.
__global__ void k_coarse_cic(const ParticleMinimum* __restrict__ p, long long n, float dx_inv,
                             int nc, float* __restrict__ grid) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    int idx[8];
    float val[8];
    cic_corners(p[i], dx_inv, nc, idx, val);
#pragma unroll
    for (int c = 0; c < 8; c++) atomicAdd(grid + idx[c], val[c]);
  }
}

// delta = nbar_inv * rho - 1 in float (coarse_grid.c:73); the mass sum of
// the grid in double on the way (the reference's check sum).
__global__ void k_coarse_delta(float* __restrict__ grid, long long n, float nbar_inv,
                               double* __restrict__ sum) {
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    const float r = grid[i];
    acc += (double)r;
    grid[i] = __fsub_rn(__fmul_rn(nbar_inv, r), 1.0f);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(sum, acc);
}

}  // namespace

extern "C" int cg_coarse_grid(const void* pmin, long long np, long long np_total, float boxsize,
                              int nc, float* delta, double* mass_sum) {
  if ((np > 0 && !pmin) || np < 0 || np_total <= 0 || !(boxsize > 0.0f) || nc < 1 || nc > 1024 ||
      !delta)
    return cg_set_error_from_lpt(CG_EINVAL, "cg_coarse_grid: bad arguments");
  const long long ng = (long long)nc * nc * nc;
  cudaPointerAttributes attr;
  const bool on_device = np > 0 && cudaPointerGetAttributes(&attr, pmin) == cudaSuccess &&
                         (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  const ParticleMinimum* d_p = on_device ? (const ParticleMinimum*)pmin : nullptr;
  ParticleMinimum* d_own = nullptr;
  float* d_grid = nullptr;
  double* d_sum = nullptr;
  cudaStream_t st = 0;
  cudaError_t e = cudaSuccess;
  if (!on_device && np > 0) {
    e = cudaMalloc(&d_own, sizeof(ParticleMinimum) * np);
    if (e == cudaSuccess)
      e = cudaMemcpy(d_own, pmin, sizeof(ParticleMinimum) * np, cudaMemcpyHostToDevice);
    d_p = d_own;
  }
  if (e == cudaSuccess) e = cudaMalloc(&d_grid, sizeof(float) * ng);
  if (e == cudaSuccess) e = cudaMalloc(&d_sum, sizeof(double));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_grid, 0, sizeof(float) * ng, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_sum, 0, sizeof(double), st);
  if (e == cudaSuccess) {
    const float dx_inv = (float)nc / boxsize;                       // coarse_grid.c:100
    const float nbar_inv = (float)((double)ng / (double)np_total);  // coarse_grid.c:60
    if (np > 0 && ng <= kSmemCells) {
      const int smem = (int)(sizeof(float) * ng);
      int per_sm = 0, sms = 0, dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaFuncSetAttribute(k_coarse_cic_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(sizeof(float) * kSmemCells));
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coarse_cic_smem, kSmemThreads,
                                                    smem);
      long long blocks = (np + kSmemThreads - 1) / kSmemThreads;
      const long long cap = (long long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
      if (blocks > cap) blocks = cap;
      prof_mark(st, CG_ST_OTHER);
      k_coarse_cic_smem<<<(int)blocks, kSmemThreads, smem, st>>>(d_p, np, dx_inv, nc, d_grid);
    } else if (np > 0) {
      prof_mark(st, CG_ST_OTHER);
      k_coarse_cic<<<grid_for(np), T, 0, st>>>(d_p, np, dx_inv, nc, d_grid);
    }
    prof_mark(st, CG_ST_OTHER);
    k_coarse_delta<<<grid_for(ng), T, 0, st>>>(d_grid, ng, nbar_inv, d_sum);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(delta, d_grid, sizeof(float) * ng, cudaMemcpyDefault);
  double sum = 0.0;
  if (e == cudaSuccess) e = cudaMemcpy(&sum, d_sum, sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_own);
  cudaFree(d_grid);
  cudaFree(d_sum);
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof(msg), "cg_coarse_grid: %s", cudaGetErrorString(e));
    return cg_set_error_from_lpt(e == cudaErrorMemoryAllocation ? CG_ENOMEM : CG_ECUDA, msg);
  }
  if (mass_sum) *mass_sum = sum;
  return CG_OK;
}

// coarse_grid.h:6 (coarse_grid.c:17-93): the grid file is the box size
// (float), nc (int), the nc^3 delta values (float, x slowest) and nc again.
extern "C" void coarse_grid2(const char filename[], Snapshot const* const snapshot, const int nc,
                             void* const mem1, const size_t size1) {
  (void)mem1;
  (void)size1;
  if (!snapshot || nc < 1) {
    cg_dropin_error(10010, "coarse_grid2: bad arguments");
    return;
  }
  const long long ng = (long long)nc * nc * nc;
  float* delta = (float*)malloc(sizeof(float) * ng);
  if (!delta) {
    cg_dropin_error(10010, "Not enough space for coarse grid");
    return;
  }
  double sum = 0.0;
  // the device copy cola_set_snapshot left, when it still matches
  cudaStream_t st = 0;
  const ParticleMinimum* d = dropin_device_snapshot(snapshot, &st);
  if (d) cudaStreamSynchronize(st);
  if (cg_coarse_grid(d ? (const void*)d : (const void*)snapshot->p, snapshot->np_local,
                     snapshot->np_total, snapshot->boxsize, nc, delta, &sum) != CG_OK) {
    free(delta);
    cg_dropin_error(10010, "coarse_grid2: coarse grid failed");
    return;
  }
  FILE* fp = fopen(filename, "w");
  if (!fp) {
    free(delta);
    char msg[512];
    snprintf(msg, sizeof(msg), "Unable to write grid to file: %s", filename);
    cg_dropin_error(10021, msg);
    return;
  }
  bool ok = fwrite(&snapshot->boxsize, sizeof(float), 1, fp) == 1;
  ok = ok && fwrite(&nc, sizeof(int), 1, fp) == 1;
  ok = ok && fwrite(delta, sizeof(float), ng, fp) == (size_t)ng;
  ok = ok && fwrite(&nc, sizeof(int), 1, fp) == 1;
  ok = (fclose(fp) == 0) && ok;
  free(delta);
  if (!ok) {
    cg_dropin_error(10021, "coarse_grid2: write failed");
    return;
  }
  // the reference's check: the grid holds the particles' mass (coarse_grid.c:88)
  if (fabs(sum - (double)snapshot->np_total) >= 0.1 * sum)
    cg_dropin_error(10030, "coarse_grid2: grid mass differs from the particle count");
}
