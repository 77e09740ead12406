// Launch accounting and per-stage CUDA-event timing of the library's kernels.
//
// Every kernel launch site calls prof_mark(stream, stage) first.  The mark
// counts the launch; while a profile is open it also records a CUDA event on
// that stream, so the device time of a stage is the interval from its event
// to the next one.  Events are only read back when the profile is closed,
// so an open profile does not synchronise the stream.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <vector>

#include "../../include/colagpu.h"
#include "internal.h"

namespace {
std::atomic<long long> g_launches{0};

struct Profile {
  bool active = false;
  std::vector<cudaEvent_t> ev;
  std::vector<int> stage;
  size_t used = 0;
  cudaStream_t last = nullptr;
};
Profile g_prof;

const char* kNames[CG_ST_COUNT] = {"fill", "deposit", "fz_r2c", "fx_fwd", "green_y",
                                    "fx_inv", "zi_c2r", "interp", "wrap", "kick",
                                    "drift", "snapshot", "lpt", "other", "kick_drift",
                                    "sort"};
}  // namespace

void prof_mark(cudaStream_t st, int stage) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (!g_prof.active || g_prof.used >= g_prof.ev.size()) return;
  cudaEventRecord(g_prof.ev[g_prof.used], st);
  g_prof.stage[g_prof.used] = stage;
  g_prof.used++;
  g_prof.last = st;
}

int cg_sm_count() {
  static std::atomic<int> cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 1;
  if (dev < 64) {
    const int c = cache[dev].load(std::memory_order_relaxed);
    if (c > 0) return c;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
    sms = 1;
  if (dev < 64) cache[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

int cg_grid(long long n, int per_sm) {
  long long b = (n + CG_THREADS - 1) / CG_THREADS;
  const long long cap = (long long)cg_sm_count() * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

extern "C" long long cg_launch_count(void) { return g_launches.load(); }

extern "C" const char* cg_stage_name(int stage) {
  return (stage >= 0 && stage < CG_ST_COUNT) ? kNames[stage] : "";
}

extern "C" int cg_prof_begin(int max_marks) {
  if (max_marks <= 0) return CG_EINVAL;
  for (auto e : g_prof.ev) cudaEventDestroy(e);
  g_prof = Profile();
  g_prof.ev.resize((size_t)max_marks + 1);
  g_prof.stage.assign((size_t)max_marks + 1, -1);
  for (auto& e : g_prof.ev)
    if (cudaEventCreate(&e) != cudaSuccess) return CG_ECUDA;
  g_prof.active = true;
  return CG_OK;
}

// Closes the profile: ms[s] = summed device time of stage s, counts[s] =
// launches of stage s (arrays of nstages entries).  Returns the number of
// marks recorded, or a negative CG_E* code.
extern "C" int cg_prof_end(double* ms, int* counts, int nstages) {
  if (!g_prof.active) return CG_EINVAL;
  g_prof.active = false;
  const size_t n = g_prof.used;
  if (ms) for (int s = 0; s < nstages; s++) ms[s] = 0.0;
  if (counts) for (int s = 0; s < nstages; s++) counts[s] = 0;
  if (n == 0) return 0;
  cudaEvent_t end = g_prof.ev[n];
  if (cudaEventRecord(end, g_prof.last) != cudaSuccess) return CG_ECUDA;
  if (cudaEventSynchronize(end) != cudaSuccess) return CG_ECUDA;
  for (size_t i = 0; i < n; i++) {
    float t = 0.0f;
    cudaEventElapsedTime(&t, g_prof.ev[i], i + 1 < n ? g_prof.ev[i + 1] : end);
    const int s = g_prof.stage[i];
    if (s >= 0 && s < nstages) {
      if (ms) ms[s] += t;
      if (counts) counts[s] += 1;
    }
  }
  return (int)n;
}
