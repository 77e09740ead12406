// GADGET-1 snapshot files (write.c:14-107 on one process), written from
// device memory with the download overlapped with the file writes.
//
// The file is four Fortran-style records, each framed by its byte length
// as an int: the 256-byte header, positions (3 floats per particle),
// velocities times 1/sqrt(a) (3 floats), and ids (unsigned int, or
// unsigned long long with use_long_id).  The particles are cut into chunks;
// for each chunk one kernel writes the three record slices from the
// ParticleMinimum array, one copy brings them into a pinned host buffer,
// and pwrite puts each slice at its offset in the file.  Two buffers
// alternate, so the GPU formats and downloads chunk k+1 while the host
// writes chunk k.
#include <cuda_runtime.h>
#include <errno.h>
#include <fcntl.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <mutex>

#include "../../include/colagpu.h"
#include "../../include/colagpu_dropin.h"
#include "gadget.h"
#include "internal.h"

extern int cg_set_error_from_lpt(int code, const char* msg);

namespace {

// The header record (gadget_file.h:4-24): the field order, widths and the
// 60 fill bytes are the file format, so they match the reference's struct.
struct GadgetHeader {
  int np[6];
  double mass[6];
  double time;
  double redshift;
  int flag_sfr;
  int flag_feedback;
  unsigned int np_total[6];
  int flag_cooling;
  int num_files;
  double boxsize;
  double omega0;
  double omega_lambda;
  double hubble_param;
  int flag_stellarage;
  int flag_metals;
  unsigned int np_total_highword[6];
  int flag_entropy_instead_u;
  char fill[60];
};
static_assert(sizeof(GadgetHeader) == 256, "GADGET header record is 256 bytes");

constexpr long long kChunk = 1LL << 20;       // particles per chunk
constexpr size_t kMaxSlice = 32;               // bytes per particle in one chunk's slices
constexpr int T = CG_THREADS;

// One chunk of the three record slices: pos[3c], vel[3c] = vfac * v in
// float (write.c:77-80), ids as 4- or 8-byte unsigned (write.c:86-101).
__global__ void k_gadget_slices(const ParticleMinimum* __restrict__ p, long long c, float vfac,
                                int long_id, float* __restrict__ pos, float* __restrict__ vel,
                                void* __restrict__ ids) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < c;
       i += (long long)gridDim.x * T) {
    const ParticleMinimum q = p[i];
    pos[3 * i + 0] = q.x[0];
    pos[3 * i + 1] = q.x[1];
    pos[3 * i + 2] = q.x[2];
    vel[3 * i + 0] = __fmul_rn(vfac, q.v[0]);
    vel[3 * i + 1] = __fmul_rn(vfac, q.v[1]);
    vel[3 * i + 2] = __fmul_rn(vfac, q.v[2]);
    if (long_id)
      ((unsigned long long*)ids)[i] = (unsigned long long)q.id;
    else
      ((unsigned int*)ids)[i] = (unsigned int)q.id;
  }
}

// Pinned host and device buffers of the pipeline, kept for the process
// (one set per device; the writer is serialised by the mutex).
struct Stage {
  int device = -1;
  char* host[2] = {nullptr, nullptr};
  char* dev[2] = {nullptr, nullptr};     // slices
  char* in[2] = {nullptr, nullptr};      // uploaded particles (host input)
  cudaEvent_t done[2] = {nullptr, nullptr};
  cudaStream_t st = nullptr;
};
std::mutex g_mu;
Stage g_stage;

cudaError_t stage_ready(Stage& s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (s.device == dev) return cudaSuccess;
  if (s.device >= 0) return cudaErrorInvalidDevice;   // one device per process
  const size_t bytes = kMaxSlice * kChunk;
  for (int b = 0; b < 2 && e == cudaSuccess; b++) {
    e = cudaHostAlloc(&s.host[b], bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&s.dev[b], bytes);
    if (e == cudaSuccess) e = cudaMalloc(&s.in[b], sizeof(ParticleMinimum) * kChunk);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done[b], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    for (int b = 0; b < 2; b++) {
      cudaFreeHost(s.host[b]);
      cudaFree(s.dev[b]);
      cudaFree(s.in[b]);
      if (s.done[b]) cudaEventDestroy(s.done[b]);
      s.host[b] = s.dev[b] = s.in[b] = nullptr;
      s.done[b] = nullptr;
    }
    if (s.st) cudaStreamDestroy(s.st);
    s.st = nullptr;
    return e;
  }
  s.device = dev;
  return cudaSuccess;
}

bool pwrite_all(int fd, const void* buf, size_t n, off_t off) {
  const char* c = (const char*)buf;
  while (n > 0) {
    const ssize_t w = pwrite(fd, c, n, off);
    if (w < 0) {
      if (errno == EINTR) continue;
      return false;
    }
    if (w == 0) return false;
    c += w;
    n -= (size_t)w;
    off += w;
  }
  return true;
}

int fail(int code, const char* what, const char* detail) {
  char msg[600];
  snprintf(msg, sizeof(msg), "%s: %s", what, detail);
  return cg_set_error_from_lpt(code, msg);
}

}  // namespace

int gadget_write(const char* filename, const void* pmin, bool on_device, long long np,
                 long long np_total, int num_files, float a, float boxsize, float omega_m,
                 float h, int use_long_id, cudaStream_t upstream) {
  if (!filename || (np > 0 && !pmin) || np < 0 || np > INT32_MAX || np_total < np ||
      !(a > 0.0f))
    return cg_set_error_from_lpt(CG_EINVAL, "gadget write: bad arguments");
  std::lock_guard<std::mutex> lock(g_mu);
  cudaError_t e = stage_ready(g_stage);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? CG_ENOMEM : CG_ECUDA, "gadget write buffers",
                cudaGetErrorString(e));
  Stage& S = g_stage;
  // the particles' producer runs on `upstream`: start after it
  if (on_device && np > 0) {
    cudaEvent_t ready;
    e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, upstream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(S.st, ready, 0);
    cudaEventDestroy(ready);
    if (e != cudaSuccess) return fail(CG_ECUDA, "gadget write", cudaGetErrorString(e));
  }

  const int fd = open(filename, O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) return fail(CG_EFILE, "Unable to write to file", filename);

  // header (write.c:42-64): every derived value in double, as the reference
  GadgetHeader hd;
  memset(&hd, 0, sizeof(hd));
  const double rho_crit = 27.7455;
  const double L = (double)boxsize, om = (double)omega_m;
  hd.np[1] = (int)np;
  hd.mass[1] = om * rho_crit * pow(L, 3.0) / (double)np_total;
  hd.time = (double)a;
  hd.redshift = 1.0 / hd.time - 1;
  hd.np_total[1] = (unsigned int)np_total;
  hd.np_total_highword[1] = (unsigned int)(np_total >> 32);
  hd.num_files = num_files;
  hd.boxsize = L;
  hd.omega0 = om;
  hd.omega_lambda = 1.0 - om;
  hd.hubble_param = (double)h;

  // record lengths are ints in the file (write.c:67,90,98): np * size
  // truncated to int as the reference's assignment does
  const size_t idb = use_long_id ? sizeof(unsigned long long) : sizeof(unsigned int);
  const int len_hdr = (int)sizeof(GadgetHeader);
  const int len_vec = (int)(uint32_t)((size_t)np * 12);
  const int len_id = (int)(uint32_t)((size_t)np * idb);
  const off_t o_pos = 4 + 256 + 4 + 4;                  // first position byte
  const off_t o_vel = o_pos + 12 * (off_t)np + 4 + 4;
  const off_t o_id = o_vel + 12 * (off_t)np + 4 + 4;
  bool ok = pwrite_all(fd, &len_hdr, 4, 0) && pwrite_all(fd, &hd, 256, 4) &&
            pwrite_all(fd, &len_hdr, 4, 260) && pwrite_all(fd, &len_vec, 4, o_pos - 4) &&
            pwrite_all(fd, &len_vec, 4, o_pos + 12 * (off_t)np) &&
            pwrite_all(fd, &len_vec, 4, o_vel - 4) &&
            pwrite_all(fd, &len_vec, 4, o_vel + 12 * (off_t)np) &&
            pwrite_all(fd, &len_id, 4, o_id - 4) &&
            pwrite_all(fd, &len_id, 4, o_id + (off_t)idb * np);

  const float vfac = (float)(1.0 / sqrt((double)a));    // write.c:74
  const long long nchunks = (np + kChunk - 1) / kChunk;
  auto enqueue = [&](long long k) -> cudaError_t {
    const int b = (int)(k & 1);
    const long long i0 = k * kChunk;
    const long long c = np - i0 < kChunk ? np - i0 : kChunk;
    const ParticleMinimum* src = (const ParticleMinimum*)pmin + i0;
    cudaError_t r = cudaSuccess;
    if (!on_device) {
      r = cudaMemcpyAsync(S.in[b], src, sizeof(ParticleMinimum) * c, cudaMemcpyHostToDevice,
                          S.st);
      src = (const ParticleMinimum*)S.in[b];
    }
    float* pos = (float*)S.dev[b];
    float* vel = pos + 3 * c;
    void* ids = vel + 3 * c;
    if (r == cudaSuccess) {
      prof_mark(S.st, CG_ST_OTHER);
      k_gadget_slices<<<cg_grid(c, 8), T, 0, S.st>>>(src, c, vfac, use_long_id, pos, vel, ids);
      r = cudaGetLastError();
    }
    if (r == cudaSuccess)
      r = cudaMemcpyAsync(S.host[b], S.dev[b], (24 + idb) * (size_t)c, cudaMemcpyDeviceToHost,
                          S.st);
    if (r == cudaSuccess) r = cudaEventRecord(S.done[b], S.st);
    return r;
  };
  auto drain = [&](long long k) -> bool {
    const int b = (int)(k & 1);
    const long long i0 = k * kChunk;
    const long long c = np - i0 < kChunk ? np - i0 : kChunk;
    if (cudaEventSynchronize(S.done[b]) != cudaSuccess) return false;
    const char* hb = S.host[b];
    return pwrite_all(fd, hb, 12 * (size_t)c, o_pos + 12 * (off_t)i0) &&
           pwrite_all(fd, hb + 12 * c, 12 * (size_t)c, o_vel + 12 * (off_t)i0) &&
           pwrite_all(fd, hb + 24 * c, idb * (size_t)c, o_id + (off_t)idb * i0);
  };
  bool io_ok = ok;
  for (long long k = 0; k < nchunks && e == cudaSuccess && io_ok; k++) {
    e = enqueue(k);                       // GPU: chunk k (buffer k & 1)
    if (e == cudaSuccess && k > 0 && io_ok) io_ok = drain(k - 1);   // host: chunk k-1
  }
  if (e == cudaSuccess && nchunks > 0 && io_ok) io_ok = drain(nchunks - 1);
  cudaError_t es = cudaStreamSynchronize(S.st);
  if (e == cudaSuccess) e = es;
  const bool closed = close(fd) == 0;
  if (e != cudaSuccess) return fail(CG_ECUDA, "gadget write", cudaGetErrorString(e));
  if (!io_ok || !closed) return fail(CG_EFILE, "gadget write failed", filename);
  return CG_OK;
}

extern "C" int cg_write_gadget(const char* filename, const void* pmin, long long np,
                               long long np_total, int num_files, float a, float boxsize,
                               float omega_m, float h, int use_long_id) {
  bool on_device = false;
  if (np > 0 && pmin) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, pmin) == cudaSuccess)
      on_device = at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
    cudaGetLastError();
  }
  return gadget_write(filename, pmin, on_device, np, np_total, num_files, a, boxsize, omega_m, h,
                      use_long_id, 0);
}

void cg_dropin_error(int code, const char* msg);

// write.h:7 (write.c:14-107): "<filebase>.0", one file for the one process.
// Reads the device copy of the snapshot when the last cola_set_snapshot
// left one for this Snapshot, else the host array.
extern "C" void write_snapshot(const char filebase[], Snapshot const* const snapshot,
                               int use_long_id) {
  if (!filebase || !snapshot) {
    cg_dropin_error(9000, "write_snapshot: bad arguments");
    return;
  }
  char filename[4096];
  snprintf(filename, sizeof(filename), "%s.%d", filebase, 0);
  cudaStream_t st = 0;
  const ParticleMinimum* d = dropin_device_snapshot(snapshot, &st);
  const long long np = snapshot->np_local;
  const int rc = gadget_write(filename, d ? (const void*)d : (const void*)snapshot->p, d != nullptr,
                              np, np, 1, snapshot->a, snapshot->boxsize, snapshot->omega_m,
                              snapshot->h, use_long_id, st);
  if (rc != CG_OK) {
    char msg[4200];
    snprintf(msg, sizeof(msg), "Error: Unable to write to file: %s", filename);
    cg_dropin_error(9000, msg);
  }
}
