// Exclusive prefix sum of unsigned counts on the device, shared by the
// counting sorts (friends-of-friends cell binning, particle cell order).
#pragma once
#include <cuda_runtime.h>

#include "internal.h"

namespace cgscan {
namespace {

constexpr int SCAN_B = 1024;   // elements per scan block

// per-block inclusive scan in shared memory, written out exclusive; the
// block's total into bsum
__global__ void __launch_bounds__(SCAN_B) k_scan_blocks(const unsigned* __restrict__ in,
                                                        unsigned* __restrict__ out, long long n,
                                                        unsigned* __restrict__ bsum) {
  __shared__ unsigned s[SCAN_B];
  const long long i = (long long)blockIdx.x * SCAN_B + threadIdx.x;
  const unsigned v = i < n ? in[i] : 0u;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < SCAN_B; o <<= 1) {
    const unsigned t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == SCAN_B - 1) bsum[blockIdx.x] = s[threadIdx.x];
}

// exclusive scan of the block totals by one CTA, chunk by chunk with a carry
__global__ void __launch_bounds__(SCAN_B) k_scan_sums(unsigned* __restrict__ bsum, long long nb,
                                                      unsigned* __restrict__ total) {
  __shared__ unsigned s[SCAN_B];
  unsigned carry = 0;
  for (long long base = 0; base < nb; base += SCAN_B) {
    const long long i = base + threadIdx.x;
    const unsigned v = i < nb ? bsum[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < SCAN_B; o <<= 1) {
      const unsigned t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) bsum[i] = carry + s[threadIdx.x] - v;
    const unsigned chunk = s[SCAN_B - 1];
    __syncthreads();
    carry += chunk;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_add(unsigned* __restrict__ out, long long n,
                           const unsigned* __restrict__ bsum) {
  for (long long i = (long long)blockIdx.x * CG_THREADS + threadIdx.x; i < n;
       i += (long long)gridDim.x * CG_THREADS)
    out[i] += bsum[i / SCAN_B];
}

}  // namespace

// Entries of block-sum scratch that exclusive() needs for n values.
inline long long scratch_entries(long long n) { return (n + SCAN_B - 1) / SCAN_B; }

// out[i] = in[0] + .. + in[i-1] (out may be in); bsum: scratch_entries(n)
// entries; *total (device, may be NULL) receives the sum.  Launches are
// counted under `stage`.
inline void exclusive(const unsigned* in, unsigned* out, long long n, unsigned* bsum,
                      unsigned* total, int stage, cudaStream_t st) {
  const long long nb = scratch_entries(n);
  if (nb == 0) {
    if (total) cudaMemsetAsync(total, 0, sizeof(unsigned), st);
    return;
  }
  const int add_blocks = cg_grid(n, 16);
  prof_mark(st, stage);
  k_scan_blocks<<<(unsigned)nb, SCAN_B, 0, st>>>(in, out, n, bsum);
  prof_mark(st, stage);
  k_scan_sums<<<1, SCAN_B, 0, st>>>(bsum, nb, total);
  prof_mark(st, stage);
  k_scan_add<<<(unsigned)add_blocks, CG_THREADS, 0, st>>>(out, n, bsum);
}

}  // namespace cgscan
