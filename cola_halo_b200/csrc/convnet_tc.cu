// 3x3x3 periodic convolution, 16 -> 16 channels, bf16 x bf16 -> fp32, on the
// fifth-generation tensor cores (tcgen05.mma, accumulator in tensor memory).
//
// Implicit GEMM per tile of 128 consecutive z voxels of one (x, y) line:
//   D[128 voxels][16 co] = sum over 27 taps of A_t[128][16 ci] . B_t[16 ci][16 co]
// The 27 taps read only 9 input lines -- the (x +- 1, y +- 1) neighbours --
// each over z0 - 1 .. z0 + 128.  A CTA copies those 9 lines (130 rows of
// 32 bytes) into shared memory once, in a row-contiguous K-major layout:
// per line, the 8-channel half h of row j sits at h * 2080 + j * 16 bytes.
// Read with core-matrix strides SBO = 128 B (8-row groups) and LBO = 2080 B
// (the two 8-channel halves), the operand of tap (dx, dy, dz) is the same
// buffer started dz rows further on: the z shift costs no copy.  B_t are the
// tap weights in the no-swizzle core-matrix layout (LBO 128 B, SBO 256 B).
//
// CTAs are persistent over tiles, 4 per SM with one line buffer each: one
// thread issues the tile's 27 MMAs (M=128, N=16, K=16), tcgen05.commit
// arrives on an mbarrier, the cp.async gather of the next tile starts, and
// the four warps read their 32 accumulator lanes with tcgen05.ld for bias +
// activation while it runs.  (A two-buffer form, 2 CTAs per SM, prefetches
// during the MMAs instead.)  Every mbarrier wait is bounded and reports through an error
// word; on a timeout the CTA drains its copies, frees its tensor memory and
// returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include "convnet.h"

namespace {

constexpr int C = CNET_C;
constexpr int TILE_M = 128;
constexpr int ROWS = TILE_M + 2;                 // z0 - 1 .. z0 + 128
constexpr int HALF_BYTES = ROWS * 16;            // 2080: one 8-channel half of a line
constexpr int LINE_BYTES = 2 * HALF_BYTES;       // 4160
constexpr int STAGE_BYTES = 9 * LINE_BYTES;      // 37440: the 9 neighbour lines
constexpr int B_BYTES = C * C * 2;               // 512: one tap's B operand
constexpr int THREADS = 128;
__host__ __device__ constexpr int smem_bytes(int stages) {
  return stages * STAGE_BYTES + 27 * B_BYTES + 64;
}
constexpr long long kWaitLimit = 1LL << 24;

__device__ unsigned g_tc_err = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: no swizzle, K-major, version 1.  LBO is
// the byte offset between the core matrices of the two K halves, SBO the
// offset between 8-row groups; the start address is 16-byte aligned.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)(lbo >> 4) << 16) |
         ((uint64_t)(sbo >> 4) << 32) | (1ULL << 46);
}

// Instruction descriptor, kind::f16: D f32, A bf16, B bf16, both K-major,
// N = 16, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) |
                            ((128u >> 4) << 24);

// offset of element (row, k) of a [rows][16] bf16 operand in core-matrix layout
__device__ __forceinline__ int cm_off(int row, int k) {
  return (((row >> 3) * 2 + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (long long i = 0; i < kWaitLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// cp.async of the 9 neighbour lines of tile `tile` into stage buffer `st`:
// element (line L, row j, half h) <- voxel (x + L/3 - 1, y + L%3 - 1,
// z0 - 1 + j), channels 8h .. 8h+7 (periodic).
__device__ __forceinline__ void gather(const __nv_bfloat16* __restrict__ in, int N, int tile,
                                       uint8_t* stage) {
  const int tiles_per_line = N / TILE_M;
  const int line = tile / tiles_per_line;
  const int z0 = (tile % tiles_per_line) * TILE_M;
  const int x = line / N, y = line % N;
  for (int i = threadIdx.x; i < 9 * ROWS * 2; i += THREADS) {
    const int h = i & 1, j = (i >> 1) % ROWS, L = (i >> 1) / ROWS;
    int xx = x + L / 3 - 1, yy = y + L % 3 - 1, zz = z0 - 1 + j;
    xx = xx < 0 ? xx + N : (xx >= N ? xx - N : xx);
    yy = yy < 0 ? yy + N : (yy >= N ? yy - N : yy);
    zz = zz < 0 ? zz + N : (zz >= N ? zz - N : zz);
    const __nv_bfloat16* src = in + (((size_t)xx * N + yy) * N + zz) * C + h * 8;
    const uint32_t dst = smem_u32(stage + L * LINE_BYTES + h * HALF_BYTES + j * 16);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
  }
}

// STAGES = 2: the next tile's gather runs during this tile's MMAs (2 CTAs
// per SM fit).  STAGES = 1: the next gather starts once this tile's MMAs
// are done and runs during its epilogue (4 CTAs per SM fit).
template <bool FLIP, int STAGES, int CPS>
__global__ void __launch_bounds__(THREADS, CPS)
    k_conv_tc(const __nv_bfloat16* __restrict__ in, int N, const __nv_bfloat16* __restrict__ w,
              const float* __restrict__ bias, int act, float* __restrict__ out_f,
              __nv_bfloat16* __restrict__ out_b, float4* __restrict__ out4) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* const stage0 = sm;
  uint8_t* const stage1 = sm + (STAGES - 1) * STAGE_BYTES;
  uint8_t* sB = sm + STAGES * STAGE_BYTES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + 27 * B_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(tslot)), "r"(32) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // B_t: element (n = output channel, k = input channel) of tap t
  for (int i = tid; i < 27 * C * C; i += THREADS) {
    const int t = i / (C * C), n = (i / C) % C, k = i % C;
    const __nv_bfloat16 v = FLIP ? w[((26 - t) * C + n) * C + k]   // W[26-t][ci=n][co=k]
                                 : w[(t * C + k) * C + n];         // W[t][ci=k][co=n]
    *reinterpret_cast<__nv_bfloat16*>(sB + t * B_BYTES + cm_off(n, k)) = v;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t bar = smem_u32(mbar);
  const int tiles_per_line = N / TILE_M;
  const int ntiles = N * N * tiles_per_line;
  uint32_t phase = 0;
  bool ok = true;

  int tile = blockIdx.x;
  if (tile < ntiles) gather(in, N, tile, stage0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int it = 0; tile < ntiles && ok; tile += gridDim.x, it++) {
    const int next = tile + gridDim.x;
    const uint8_t* s = (it & 1) ? stage1 : stage0;
    if (STAGES == 2) {
      // the next tile's lines load while this tile multiplies; that buffer's
      // previous MMAs completed before the last iteration's epilogue
      if (next < ntiles) gather(in, N, next, (it & 1) ? stage0 : stage1);
      asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      for (int t = 0; t < 27; t++) {
        // tap (dx, dy, dz): line t / 3, started dz = t % 3 rows on
        const uint64_t da =
            umma_desc(smem_u32(s + (t / 3) * LINE_BYTES + (t % 3) * 16), HALF_BYTES, 128);
        const uint64_t db = umma_desc(smem_u32(sB + t * B_BYTES), 128, 256);
        const uint32_t acc = t > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
            :: "r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(bar) : "memory");
    }
    // every thread waits (bounded); the CTA agrees on the outcome so that all
    // threads take the same path through the barriers below
    const bool got = mbar_wait(bar, phase);
    ok = __syncthreads_and(got ? 1 : 0) != 0;
    if (!ok && tid == 0) atomicOr(&g_tc_err, 1u);
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (STAGES == 1) {
      // the MMAs have read the buffer: the next tile's lines load during
      // this tile's epilogue
      if (ok && next < ntiles) gather(in, N, next, stage0);
      asm volatile("cp.async.commit_group;" ::: "memory");
    }
    if (ok) {
      const int line = tile / tiles_per_line;
      const int z0 = (tile % tiles_per_line) * TILE_M;
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
          "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
            "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
            "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const size_t v = (size_t)line * N + z0 + warp * 32 + lane;
      float o[C];
#pragma unroll
      for (int c = 0; c < C; c++) {
        float a = __uint_as_float(r[c]) + (bias ? bias[c] : 0.0f);
        if (act) a = a > 0.0f ? a : 0.1f * a;
        o[c] = a;
      }
      if (out_f) {
        float4* d = reinterpret_cast<float4*>(out_f + v * C);
#pragma unroll
        for (int q = 0; q < 4; q++)
          d[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
      }
      if (out_b) {
        __nv_bfloat16 hb[C];
#pragma unroll
        for (int c = 0; c < C; c++) hb[c] = __float2bfloat16_rn(o[c]);
        uint4* d = reinterpret_cast<uint4*>(out_b + v * C);
        d[0] = *reinterpret_cast<const uint4*>(&hb[0]);
        d[1] = *reinterpret_cast<const uint4*>(&hb[8]);
      }
      if (out4) out4[v] = make_float4(o[0], o[1], o[2], o[3]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  // copies still in flight (a prefetch after a timeout) finish before exit
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(32)
                 : "memory");
}

// The same convolution for a 128^3 mesh (one tile per line), with the input
// lines reused along y.  A CTA walks a contiguous run of lines (x, y),
// (x, y+1), ...: tile (x, y) reads the lines (x-1..x+1, y-1..y+1), so the
// next tile needs only the three lines of row y+2.  The rows sit in a ring
// of four slots of three lines (x-1, x, x+1); row j of the run goes to slot
// j mod 4 in its own cp.async group.  While tile i's epilogue runs, the
// slot that tile i's row y-1 used is refilled with row y+3, so a tile
// waits for one new row of 12 KB instead of gathering 37 KB.  The MMAs,
// their order and their operands are those of k_conv_tc: bit-identical
// output.  3 CTAs per SM (62 KB each).
constexpr int RING_BYTES = 12 * LINE_BYTES;      // 49920
__host__ __device__ constexpr int ring_smem_bytes() { return RING_BYTES + 27 * B_BYTES + 64; }

// cp.async of row y (periodic) of the lines x-1, x, x+1 into ring slot `slot`
// (line dx+1 of the slot; rows z = -1 .. 128, two 8-channel halves).
__device__ __forceinline__ void gather_row(const __nv_bfloat16* __restrict__ in, int N, int x,
                                           int y, uint8_t* slot) {
  y = y < 0 ? y + N : (y >= N ? y - N : y);
  for (int i = threadIdx.x; i < 3 * ROWS * 2; i += THREADS) {
    const int h = i & 1, j = (i >> 1) % ROWS, L = (i >> 1) / ROWS;
    int xx = x + L - 1, zz = j - 1;
    xx = xx < 0 ? xx + N : (xx >= N ? xx - N : xx);
    zz = zz < 0 ? zz + N : (zz >= N ? zz - N : zz);
    const __nv_bfloat16* src = in + (((size_t)xx * N + y) * N + zz) * C + h * 8;
    const uint32_t dst = smem_u32(slot + L * LINE_BYTES + h * HALF_BYTES + j * 16);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
  }
}

template <bool FLIP>
__global__ void __launch_bounds__(THREADS, 3)
    k_conv_ring(const __nv_bfloat16* __restrict__ in, int N, const __nv_bfloat16* __restrict__ w,
                const float* __restrict__ bias, int act, float* __restrict__ out_f,
                __nv_bfloat16* __restrict__ out_b, float4* __restrict__ out4) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* const ring = sm;
  uint8_t* sB = sm + RING_BYTES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + 27 * B_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(tslot)), "r"(32) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < 27 * C * C; i += THREADS) {
    const int t = i / (C * C), n = (i / C) % C, k = i % C;
    const __nv_bfloat16 v = FLIP ? w[((26 - t) * C + n) * C + k]
                                 : w[(t * C + k) * C + n];
    *reinterpret_cast<__nv_bfloat16*>(sB + t * B_BYTES + cm_off(n, k)) = v;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t bar = smem_u32(mbar);
  const int nlines = N * N;
  const int per = (nlines + (int)gridDim.x - 1) / (int)gridDim.x;
  const int l1 = min(nlines, (int)blockIdx.x * per + per);
  uint32_t phase = 0;
  bool ok = true;
  for (int l = (int)blockIdx.x * per; l < l1 && ok;) {
    const int x = l / N, y0 = l % N;
    const int run = min(l1 - l, N - y0);          // tiles of this x in the CTA's range
    // rows y0-1 .. y0+2 (loaded rows 0..3) into slots 0..3, one group each
    for (int j = 0; j < 4; j++) {
      if (j <= run + 1) gather_row(in, N, x, y0 - 1 + j, ring + j * 3 * LINE_BYTES);
      asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int i = 0; i < run && ok; i++) {
      // loaded rows i .. i+2 complete (row i+3 may still be in flight)
      asm volatile("cp.async.wait_group 1;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
        for (int t = 0; t < 27; t++) {
          // tap t: line L = t / 3 = (dx+1) * 3 + (dy+1), started dz = t % 3 rows on
          const int L = t / 3;
          const uint8_t* line = ring + (((i + L % 3) & 3) * 3 + L / 3) * LINE_BYTES;
          const uint64_t da = umma_desc(smem_u32(line + (t % 3) * 16), HALF_BYTES, 128);
          const uint64_t db = umma_desc(smem_u32(sB + t * B_BYTES), 128, 256);
          const uint32_t acc = t > 0 ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
              :: "r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
              : "memory");
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
            :: "r"(bar) : "memory");
      }
      const bool got = mbar_wait(bar, phase);
      ok = __syncthreads_and(got ? 1 : 0) != 0;
      if (!ok && tid == 0) atomicOr(&g_tc_err, 1u);
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // the MMAs have read loaded row i: its slot takes row i + 4
      if (ok && i + 4 <= run + 1) gather_row(in, N, x, y0 - 1 + i + 4, ring + (i & 3) * 3 * LINE_BYTES);
      asm volatile("cp.async.commit_group;" ::: "memory");
      if (ok) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const size_t v = (size_t)(l + i) * N + warp * 32 + lane;
        float o[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
          float a = __uint_as_float(r[c]) + (bias ? bias[c] : 0.0f);
          if (act) a = a > 0.0f ? a : 0.1f * a;
          o[c] = a;
        }
        if (out_f) {
          float4* d = reinterpret_cast<float4*>(out_f + v * C);
#pragma unroll
          for (int q = 0; q < 4; q++)
            d[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
        }
        if (out_b) {
          __nv_bfloat16 hb[C];
#pragma unroll
          for (int c = 0; c < C; c++) hb[c] = __float2bfloat16_rn(o[c]);
          uint4* d = reinterpret_cast<uint4*>(out_b + v * C);
          d[0] = *reinterpret_cast<const uint4*>(&hb[0]);
          d[1] = *reinterpret_cast<const uint4*>(&hb[8]);
        }
        if (out4) out4[v] = make_float4(o[0], o[1], o[2], o[3]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
    }
    // the run's prefetches land before the ring is refilled for the next x
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    l += run;
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(32)
                 : "memory");
}

template <bool FLIP>
cudaError_t launch_ring(const __nv_bfloat16* in, int N, const __nv_bfloat16* w,
                        const float* bias, int act, float* of, __nv_bfloat16* ob, float4* o4,
                        cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_ring<FLIP>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         ring_smem_bytes());
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int grid = 3 * cg_sm_count();
  prof_mark(st, CG_ST_OTHER);
  k_conv_ring<FLIP><<<grid, THREADS, ring_smem_bytes(), st>>>(in, N, w, bias, act, of, ob, o4);
  return cudaGetLastError();
}

template <bool FLIP, int STAGES, int CPS>
cudaError_t launch_v(const __nv_bfloat16* in, int N, const __nv_bfloat16* w, const float* bias,
                     int act, float* of, __nv_bfloat16* ob, float4* o4, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_tc<FLIP, STAGES, CPS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem_bytes(STAGES));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int ntiles = N * N * (N / TILE_M);
  const int sms = cg_sm_count();
  const int grid = ntiles < CPS * sms ? ntiles : CPS * sms;
  prof_mark(st, CG_ST_OTHER);
  k_conv_tc<FLIP, STAGES, CPS><<<grid, THREADS, smem_bytes(STAGES), st>>>(in, N, w, bias, act,
                                                                         of, ob, o4);
  return cudaGetLastError();
}

// pipeline variant: 2 (default at 128^3) = the line ring (k_conv_ring);
// 1 (default for larger meshes) = one stage, 4 CTAs/SM; 0 = two stages,
// 2 CTAs/SM.  Without the ring, at 128^3 the one-stage form is 1.2x faster
// than the two-stage one: the tile loop is latency-bound and more resident
// CTAs hide more of it than the prefetch does.  COLAGPU_CONV_VARIANT=0/1/2
// selects one (2 only at 128^3).
int g_conv_variant = -1;      // conv_tc_set_variant

int conv_variant(int N) {
  static const int forced = [] {
    const char* e = getenv("COLAGPU_CONV_VARIANT");
    return e ? atoi(e) : -1;
  }();
  const int v = forced >= 0 ? forced : g_conv_variant;
  if (v == 0 || v == 1 || (v == 2 && N == TILE_M)) return v;
  return N == TILE_M ? 2 : 1;
}

template <bool FLIP>
cudaError_t launch(const __nv_bfloat16* in, int N, const __nv_bfloat16* w, const float* bias,
                   int act, float* of, __nv_bfloat16* ob, float4* o4, cudaStream_t st) {
  if (N < TILE_M || N % TILE_M) return cudaErrorNotSupported;
  const int v = conv_variant(N);
  if (v == 2) return launch_ring<FLIP>(in, N, w, bias, act, of, ob, o4, st);
  if (v == 1) return launch_v<FLIP, 1, 4>(in, N, w, bias, act, of, ob, o4, st);
  return launch_v<FLIP, 2, 2>(in, N, w, bias, act, of, ob, o4, st);
}

}  // namespace

cudaError_t conv_tc_forward(const __nv_bfloat16* in, int N, const __nv_bfloat16* w,
                            const float* bias, int act, float* out_f, __nv_bfloat16* out_b,
                            float4* out4, cudaStream_t st) {
  return launch<false>(in, N, w, bias, act, out_f, out_b, out4, st);
}

cudaError_t conv_tc_backward_data(const __nv_bfloat16* g, int N, const __nv_bfloat16* w,
                                  float* out_f, cudaStream_t st) {
  return launch<true>(g, N, w, nullptr, 0, out_f, nullptr, nullptr, st);
}

int conv_tc_set_variant(int v) {
  return v >= -1 && v <= 2 ? (g_conv_variant = v, 0) : -1;
}

unsigned conv_tc_error_word() {
  unsigned v = 0;
  cudaMemcpyFromSymbol(&v, g_tc_err, sizeof(v));
  return v;
}
