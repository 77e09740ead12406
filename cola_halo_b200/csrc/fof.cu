// Friends-of-friends halos on the GPU (fof.c:427-1181 on one process).
//
// The reference builds a k-d tree and grows one group at a time from a
// FIFO; across the x faces it links through buffer particles shifted by
// -L.  On one process that is periodic friends-of-friends: particles whose
// squared distance (float32, as kdFoF forms it, fof.c:569-572) is below
// ll^2 are linked, and groups of at least 32 (fof.c:224) are halos, with
// centre = a member position + the mean minimum-image offset of all
// members, wrapped into [0, L) (fof.c:287-322, 1141-1150), and the mean
// velocity.  Here:
//   1. wrap positions (move_particles2_min, fof.c:1042) and bin them on a
//      grid of cells no smaller than ll (counting sort: count, scan, scatter)
//   2. each particle tests the particles of the 27 neighbouring cells that
//      come after it in cell order; a link joins the two sets of a
//      lock-free union-find over the original particle indices (hooking the
//      larger root under the smaller with atomicCAS, path halving)
//   3. flatten to roots, count members, number the roots with >= nfof_min
//      members in root order (a scan), accumulate the offsets from the root
//      particle and the velocities in double, and finish each halo.
// The root of a group is its smallest original index, so the catalogue is
// in a fixed order and each centre's reference member is fixed.  Every
// retry loop is bounded; running out of iterations sets an error word.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/colagpu.h"
#include "../../include/colagpu_dropin.h"
#include "gadget.h"
#include "internal.h"
#include "scan.cuh"

extern int cg_set_error_from_lpt(int code, const char* msg);

namespace {

constexpr int T = CG_THREADS;
constexpr int MAX_NCELL = 512;          // cells per dimension at most
constexpr int kRetryLimit = 1 << 22;    // union / find iterations per call

// Reference ParticleMinimum (particle.h:24-29): 32 bytes.
struct PMin {
  float x[3];
  float v[3];
  long long id;
};

__device__ __forceinline__ float wrap1(float x, float L) {
  // one-shot periodic wrap as move.c:34-41
  if (x < 0.0f) x += L;
  else if (x >= L) x -= L;
  return x;
}

__device__ __forceinline__ int cell_of(float x, float inv, int nc) {
  int c = (int)(x * inv);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_fof_bin(const PMin* __restrict__ p, long long n, float L, float inv, int nc,
                          float* __restrict__ xw, unsigned* __restrict__ key,
                          unsigned* __restrict__ count) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    const float x = wrap1(p[i].x[0], L), y = wrap1(p[i].x[1], L), z = wrap1(p[i].x[2], L);
    xw[3 * i] = x;
    xw[3 * i + 1] = y;
    xw[3 * i + 2] = z;
    const unsigned k =
        ((unsigned)cell_of(x, inv, nc) * nc + cell_of(y, inv, nc)) * nc + cell_of(z, inv, nc);
    key[i] = k;
    atomicAdd(count + k, 1u);
  }
}

__global__ void k_fof_scatter(const float* __restrict__ xw, const unsigned* __restrict__ key,
                              long long n, const unsigned* __restrict__ start,
                              unsigned* __restrict__ cursor, float4* __restrict__ pos) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    const unsigned k = key[i];
    const unsigned slot = start[k] + atomicAdd(cursor + k, 1u);
    pos[slot] = make_float4(xw[3 * i], xw[3 * i + 1], xw[3 * i + 2], __int_as_float((int)i));
  }
}

// ------------------------------------------------------------- union-find
// parent[] over original particle indices; a root is parent[r] == r.
__device__ __forceinline__ int find_root(int* parent, int x, unsigned* err) {
  for (int it = 0; it < kRetryLimit; it++) {
    const int p = __ldcg(parent + x);
    if (p == x) return x;
    const int gp = __ldcg(parent + p);
    if (gp != p) atomicCAS(parent + x, p, gp);   // path halving (benign race)
    x = gp;
  }
  atomicOr(err, 1u);
  return x;
}

__device__ __forceinline__ void unite(int* parent, int a, int b, unsigned* err) {
  for (int it = 0; it < kRetryLimit; it++) {
    a = find_root(parent, a, err);
    b = find_root(parent, b, err);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    // hang the larger root under the smaller one if it is still a root
    if (atomicCAS(parent + b, b, a) == b) return;
  }
  atomicOr(err, 2u);
}

__global__ void k_fof_init_parent(int* __restrict__ parent, long long n) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T)
    parent[i] = (int)i;
}

// Squared distance of two wrapped positions with the periodic image formed
// as the reference forms it: the coordinate of the particle on the far side
// is shifted by -L before the difference (fof.c:645-647, and the cell
// images of INTERSECT), float arithmetic without contraction.
__device__ __forceinline__ float dist2(float4 a, float4 b, float L, float half) {
  float d[3];
  const float pa[3] = {a.x, a.y, a.z}, pb[3] = {b.x, b.y, b.z};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    float t = __fsub_rn(pa[k], pb[k]);
    if (t > half) t = __fsub_rn(__fsub_rn(pa[k], L), pb[k]);
    else if (t < -half) t = __fsub_rn(__fsub_rn(pb[k], L), pa[k]);
    d[k] = t;
  }
  return __fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])),
                   __fmul_rn(d[2], d[2]));
}

// One thread per particle in cell order: links to the particles of the 27
// neighbouring cells that come later in cell order (each pair once).  With
// fewer than 3 cells per dimension every cell is a neighbour.
__global__ void k_fof_link(const float4* __restrict__ pos, long long n,
                           const unsigned* __restrict__ start, const unsigned* __restrict__ count,
                           int nc, float inv, float L, float ll2, int* __restrict__ parent,
                           unsigned* __restrict__ err) {
  const float half = 0.5f * L;
  for (long long s = (long long)blockIdx.x * T + threadIdx.x; s < n;
       s += (long long)gridDim.x * T) {
    const float4 a = pos[s];
    const int ia = __float_as_int(a.w);
    const int cx = cell_of(a.x, inv, nc), cy = cell_of(a.y, inv, nc), cz = cell_of(a.z, inv, nc);
    const int span = nc >= 3 ? 3 : nc;
    for (int ox = 0; ox < span; ox++) {
      const int gx = nc >= 3 ? (cx + ox - 1 + nc) % nc : ox;
      for (int oy = 0; oy < span; oy++) {
        const int gy = nc >= 3 ? (cy + oy - 1 + nc) % nc : oy;
        for (int oz = 0; oz < span; oz++) {
          const int gz = nc >= 3 ? (cz + oz - 1 + nc) % nc : oz;
          const unsigned k = ((unsigned)gx * nc + gy) * nc + gz;
          const unsigned b0 = start[k], b1 = b0 + count[k];
          for (unsigned t = b0 > (unsigned)s ? b0 : (unsigned)s + 1; t < b1; t++) {
            const float4 b = pos[t];
            if (dist2(a, b, L, half) < ll2) unite(parent, ia, __float_as_int(b.w), err);
          }
        }
      }
    }
  }
}

__global__ void k_fof_flatten(int* __restrict__ parent, long long n, unsigned* __restrict__ size,
                              unsigned* __restrict__ err) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    const int r = find_root(parent, (int)i, err);
    atomicAdd(size + r, 1u);
  }
}

// After flatten every particle's chain ends at its root; store it directly.
__global__ void k_fof_roots(int* __restrict__ parent, long long n, unsigned* __restrict__ err) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T)
    parent[i] = find_root(parent, (int)i, err);
}

__global__ void k_fof_flag(const int* __restrict__ root, const unsigned* __restrict__ size,
                           long long n, unsigned nmin, unsigned* __restrict__ flag) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T)
    flag[i] = (root[i] == (int)i && size[i] >= nmin) ? 1u : 0u;
}

// Per member: offset from the halo's root particle with the minimum-image
// wrap of halo_particle (fof.c:304-313, float), summed in double with the
// velocities.  acc[6 h + 0..2] = offsets, [3..5] = velocities.
__global__ void k_fof_accum(const PMin* __restrict__ p, const float* __restrict__ xw,
                            const int* __restrict__ root, const unsigned* __restrict__ hid,
                            const unsigned* __restrict__ flag, long long n, float L,
                            double* __restrict__ acc) {
  const float half = 0.5f * L;
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n;
       i += (long long)gridDim.x * T) {
    const int r = root[i];
    if (!flag[r]) continue;
    const unsigned h = hid[r];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float dx = __fsub_rn(xw[3 * i + k], xw[3 * (size_t)r + k]);
      if (dx > half) dx = __fsub_rn(dx, L);
      else if (dx < -half) dx = __fadd_rn(dx, L);
      atomicAdd(acc + 6 * (size_t)h + k, (double)dx);
      atomicAdd(acc + 6 * (size_t)h + 3 + k, (double)p[i].v[k]);
    }
  }
}

// Halo h: centre x0 + mean offset wrapped into [0, L) as fof.c:1141-1147,
// mean velocity (fof.c:1150).
__global__ void k_fof_finish(const float* __restrict__ xw, const unsigned* __restrict__ size,
                             const unsigned* __restrict__ hid, const unsigned* __restrict__ flag,
                             long long n, float L, const double* __restrict__ acc,
                             cg_halo* __restrict__ out, long long max_out) {
  for (long long r = (long long)blockIdx.x * T + threadIdx.x; r < n;
       r += (long long)gridDim.x * T) {
    if (!flag[r]) continue;
    const unsigned h = hid[r];
    if ((long long)h >= max_out) continue;
    const unsigned nf = size[r];
    cg_halo o;
    o.nfof = (int)nf;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float x = __fadd_rn(xw[3 * r + k], (float)(acc[6 * (size_t)h + k] / (double)nf));
      if (x < 0.0f) x += L;
      if (x >= L) x -= L;
      o.x[k] = x;
      o.v[k] = (float)(acc[6 * (size_t)h + 3 + k] / (double)nf);
    }
    out[h] = o;
  }
}

template <class TPtr>
void release(TPtr*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace

extern "C" int cg_fof(const void* pmin, long long np, float boxsize, float ll, int nfof_min,
                      cg_halo* halos, long long max_halos, long long* nhalo) {
  if (!nhalo || np < 0 || np >= (1LL << 31) - 1 || !(boxsize > 0.0f) || !(ll > 0.0f) ||
      nfof_min < 1 || (max_halos > 0 && !halos) || (np > 0 && !pmin))
    return cg_set_error_from_lpt(CG_EINVAL, "cg_fof: bad arguments");
  *nhalo = 0;
  if (np == 0) return CG_OK;
  // cells no smaller than ll (with a margin over the float rounding of the
  // cell index, so linked pairs are never two cells apart), at most
  // MAX_NCELL per side and about 8 per particle
  long long nc = (long long)floor((double)boxsize / (double)ll * 0.99999);
  const long long ncap = (long long)cbrt(8.0 * (double)np) + 1;
  if (nc > MAX_NCELL) nc = MAX_NCELL;
  if (nc > ncap) nc = ncap;
  if (nc < 1) nc = 1;
  const long long ncells = nc * nc * nc;
  const float inv = (float)nc / boxsize;
  const long long nblk = cgscan::scratch_entries(ncells > np ? ncells : np);

  cudaPointerAttributes attr;
  bool on_device = cudaPointerGetAttributes(&attr, pmin) == cudaSuccess &&
                   (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
  cudaGetLastError();   // a plain host pointer may leave an error behind
  PMin* d_p = on_device ? (PMin*)pmin : nullptr;
  float* xw = nullptr;
  unsigned *key = nullptr, *count = nullptr, *start = nullptr, *cursor = nullptr;
  unsigned *size = nullptr, *flag = nullptr, *hid = nullptr, *bsum = nullptr, *word = nullptr;
  int* parent = nullptr;
  float4* pos = nullptr;
  double* acc = nullptr;
  cg_halo* out = nullptr;
  cudaStream_t st = 0;
  cudaError_t e = cudaSuccess;
  if (!on_device) {
    e = cudaMalloc(&d_p, sizeof(PMin) * np);
    if (e == cudaSuccess) e = cudaMemcpy(d_p, pmin, sizeof(PMin) * np, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&xw, sizeof(float) * 3 * np);
  if (e == cudaSuccess) e = cudaMalloc(&key, sizeof(unsigned) * np);
  if (e == cudaSuccess) e = cudaMalloc(&count, sizeof(unsigned) * ncells);
  if (e == cudaSuccess) e = cudaMalloc(&start, sizeof(unsigned) * ncells);
  if (e == cudaSuccess) e = cudaMalloc(&cursor, sizeof(unsigned) * ncells);
  if (e == cudaSuccess) e = cudaMalloc(&pos, sizeof(float4) * np);
  if (e == cudaSuccess) e = cudaMalloc(&parent, sizeof(int) * np);
  if (e == cudaSuccess) e = cudaMalloc(&size, sizeof(unsigned) * np);
  if (e == cudaSuccess) e = cudaMalloc(&flag, sizeof(unsigned) * np);
  if (e == cudaSuccess) e = cudaMalloc(&hid, sizeof(unsigned) * np);
  if (e == cudaSuccess) e = cudaMalloc(&bsum, sizeof(unsigned) * (nblk + 1));
  if (e == cudaSuccess) e = cudaMalloc(&word, sizeof(unsigned) * 2);   // [0] total, [1] error
  if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, sizeof(unsigned) * ncells, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(cursor, 0, sizeof(unsigned) * ncells, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(size, 0, sizeof(unsigned) * np, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(word, 0, sizeof(unsigned) * 2, st);
  unsigned nh = 0, errw = 0;
  if (e == cudaSuccess) {
    const int g = grid_for(np);
    prof_mark(st, CG_ST_OTHER);
    k_fof_bin<<<g, T, 0, st>>>(d_p, np, boxsize, inv, (int)nc, xw, key, count);
    cgscan::exclusive(count, start, ncells, bsum, word, CG_ST_OTHER, st);
    prof_mark(st, CG_ST_OTHER);
    k_fof_scatter<<<g, T, 0, st>>>(xw, key, np, start, cursor, pos);
    prof_mark(st, CG_ST_OTHER);
    k_fof_init_parent<<<g, T, 0, st>>>(parent, np);
    prof_mark(st, CG_ST_OTHER);
    k_fof_link<<<g, T, 0, st>>>(pos, np, start, count, (int)nc, inv, boxsize, ll * ll, parent,
                                word + 1);
    prof_mark(st, CG_ST_OTHER);
    k_fof_flatten<<<g, T, 0, st>>>(parent, np, size, word + 1);
    prof_mark(st, CG_ST_OTHER);
    k_fof_roots<<<g, T, 0, st>>>(parent, np, word + 1);
    prof_mark(st, CG_ST_OTHER);
    k_fof_flag<<<g, T, 0, st>>>(parent, size, np, (unsigned)nfof_min, flag);
    cgscan::exclusive(flag, hid, np, bsum, word, CG_ST_OTHER, st);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&nh, word, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && nh > 0) {
      e = cudaMalloc(&acc, sizeof(double) * 6 * nh);
      if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(cg_halo) * nh);
      if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(double) * 6 * nh, st);
      if (e == cudaSuccess) {
        prof_mark(st, CG_ST_OTHER);
        k_fof_accum<<<g, T, 0, st>>>(d_p, xw, parent, hid, flag, np, boxsize, acc);
        prof_mark(st, CG_ST_OTHER);
        k_fof_finish<<<g, T, 0, st>>>(xw, size, hid, flag, np, boxsize, acc, out, nh);
        e = cudaGetLastError();
      }
      const long long ncopy = max_halos < (long long)nh ? max_halos : (long long)nh;
      if (e == cudaSuccess && ncopy > 0)
        e = cudaMemcpy(halos, out, sizeof(cg_halo) * ncopy, cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess) e = cudaMemcpy(&errw, word + 1, sizeof(unsigned), cudaMemcpyDeviceToHost);
  }
  if (!on_device) release(d_p);
  release(xw); release(key); release(count); release(start); release(cursor); release(pos);
  release(parent); release(size); release(flag); release(hid); release(bsum); release(word);
  release(acc); release(out);
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof(msg), "cg_fof: %s", cudaGetErrorString(e));
    return cg_set_error_from_lpt(e == cudaErrorMemoryAllocation ? CG_ENOMEM : CG_ECUDA, msg);
  }
  if (errw)
    return cg_set_error_from_lpt(CG_ECUDA, "cg_fof: union-find iteration limit reached");
  *nhalo = nh;
  return CG_OK;
}

// ---------------------------------------------------------------- drop-in
void cg_dropin_error(int code, const char* msg);

namespace {
cg_halo* g_halos = nullptr;
long long g_nhalo = 0;

// move_particles2_min's wrap of a snapshot (move.c:33-41, float add or
// subtract of L once per axis), in place on the device.  Particles it moves
// are listed -- index and new position, up to `cap` -- so that the host copy
// can be patched without downloading the whole snapshot.
__global__ void k_wrap_list(ParticleMinimum* __restrict__ p, long long n, float L,
                            unsigned long long* __restrict__ count, long long cap,
                            long long* __restrict__ idx, float* __restrict__ xs) {
  for (long long i = (long long)blockIdx.x * CG_THREADS + threadIdx.x; i < n;
       i += (long long)gridDim.x * CG_THREADS) {
    float x[3];
    bool moved = false;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      x[k] = p[i].x[k];
      if (x[k] < 0.0f) {
        x[k] = __fadd_rn(x[k], L);
        moved = true;
      } else if (x[k] >= L) {
        x[k] = __fsub_rn(x[k], L);
        moved = true;
      }
    }
    if (!moved) continue;
#pragma unroll
    for (int k = 0; k < 3; k++) p[i].x[k] = x[k];
    const unsigned long long slot = atomicAdd(count, 1ULL);
    if ((long long)slot < cap) {
      idx[slot] = i;
#pragma unroll
      for (int k = 0; k < 3; k++) xs[3 * slot + k] = x[k];
    }
  }
}

// Wrap the device snapshot d (n particles, after the work on st) and bring
// the host copy h to the same positions.
cudaError_t wrap_device_and_host(ParticleMinimum* d, ParticleMinimum* h, long long n, float L,
                                 cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const long long cap = n < (1LL << 20) ? n : (1LL << 20);
  unsigned long long* d_count = nullptr;
  long long* d_idx = nullptr;
  float* d_x = nullptr;
  cudaError_t e = cudaMalloc(&d_count, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&d_idx, sizeof(long long) * cap);
  if (e == cudaSuccess) e = cudaMalloc(&d_x, sizeof(float) * 3 * cap);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    prof_mark(st, CG_ST_WRAP);
    k_wrap_list<<<cg_grid(n, 16), CG_THREADS, 0, st>>>(d, n, L, d_count, cap, d_idx, d_x);
    e = cudaGetLastError();
  }
  unsigned long long moved = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&moved, d_count, sizeof(moved), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && moved > 0) {
    if ((long long)moved <= cap) {
      long long* idx = (long long*)malloc(sizeof(long long) * moved);
      float* xs = (float*)malloc(sizeof(float) * 3 * moved);
      if (!idx || !xs) e = cudaErrorMemoryAllocation;
      if (e == cudaSuccess)
        e = cudaMemcpy(idx, d_idx, sizeof(long long) * moved, cudaMemcpyDeviceToHost);
      if (e == cudaSuccess)
        e = cudaMemcpy(xs, d_x, sizeof(float) * 3 * moved, cudaMemcpyDeviceToHost);
      if (e == cudaSuccess)
        for (unsigned long long j = 0; j < moved; j++)
          memcpy(h[idx[j]].x, xs + 3 * j, sizeof(float) * 3);
      free(idx);
      free(xs);
    } else {
      e = cudaMemcpy(h, d, sizeof(ParticleMinimum) * n, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(d_count);
  cudaFree(d_idx);
  cudaFree(d_x);
  return e;
}
}  // namespace

extern "C" size_t fof_calc_memory(const int np_alloc, const int nc) {
  (void)np_alloc;
  (void)nc;
  return 0;   // the GPU finder needs none of the caller's arena
}

extern "C" void fof_init(const int np_alloc, const int nc, void* mem, size_t mem_size) {
  (void)np_alloc;
  (void)nc;
  (void)mem;
  (void)mem_size;
}

extern "C" void fof_find_halos(Snapshot* snapshot, const float ll) {
  if (!snapshot || !(snapshot->boxsize > 0.0f) || snapshot->np_local < 0 ||
      (snapshot->np_local > 0 && !snapshot->p)) {
    cg_dropin_error(7000, "fof_find_halos: bad snapshot");
    return;
  }
  const float L = snapshot->boxsize;
  const int n = snapshot->np_local;
  const long long cap = n / 32 + 1;   // halos hold at least 32 particles each
  cg_halo* h = (cg_halo*)realloc(g_halos, sizeof(cg_halo) * cap);
  if (!h) {
    cg_dropin_error(7050, "Not enough space for halo");
    return;
  }
  g_halos = h;
  g_nhalo = 0;
  // the snapshot on the device: the copy cola_set_snapshot left, or an upload
  cudaStream_t st = 0;
  ParticleMinimum* d = dropin_device_snapshot(snapshot, &st);
  ParticleMinimum* own = nullptr;
  cudaError_t e = cudaSuccess;
  if (!d && n > 0) {
    e = cudaMalloc(&own, sizeof(ParticleMinimum) * n);
    if (e == cudaSuccess)
      e = cudaMemcpy(own, snapshot->p, sizeof(ParticleMinimum) * n, cudaMemcpyHostToDevice);
    d = own;
    st = 0;
  }
  // move_particles2_min (fof.c:1042): one-shot wrap into the box, in place,
  // on both copies
  if (e == cudaSuccess) e = wrap_device_and_host(d, snapshot->p, n, L, st);
  long long nh = 0;
  const int rc = e == cudaSuccess ? cg_fof(d, n, L, ll, 32, g_halos, cap, &nh) : CG_ECUDA;
  cudaFree(own);
  if (rc != CG_OK) {
    cg_dropin_error(7050, "fof_find_halos failed");
    return;
  }
  g_nhalo = nh;
}

extern "C" void fof_write_halos(char filename[]) {
  FILE* fp = fopen(filename, "w");
  if (!fp) {
    char msg[512];
    snprintf(msg, sizeof(msg), "Error: Unable to write halo to file %s", filename);
    cg_dropin_error(8110, msg);
    return;
  }
  for (long long i = 0; i < g_nhalo; i++) {
    const cg_halo& h = g_halos[i];
    fprintf(fp, "%d %e %e %e %e %e %e\n", h.nfof, h.x[0], h.x[1], h.x[2], h.v[0], h.v[1],
            h.v[2]);
  }
  fclose(fp);
}
