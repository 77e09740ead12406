// FFT schedule autotuner (no reference counterpart).
//
// Each mesh size from 256 up has several compiled variants of the two
// passes whose best shape depends on the size: the strided x pass (ky
// columns per CTA, maximum radix) and the fused y Green pass (lines per
// CTA, maximum radix, resident CTAs per SM).  cg_autotune times every
// variant on a plan of that size on the current device and installs the
// fastest of each; the result is kept for the process and, when
// COLAGPU_TUNE_CACHE names a file, appended to it as one line
//   <device name> TAB <ngrid> TAB <green variant> TAB <x variant>
// so that later processes on the same kind of GPU reuse it without timing.
// A cached or installed schedule also makes runs reproducible: variants
// differ in rounding (different radix orders), not in the algorithm.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <set>
#include <string>
#include <utility>

#include "../../include/colagpu.h"
#include "internal.h"

extern int cg_set_error_from_lpt(int code, const char* msg);

namespace {

std::mutex g_mu;
std::set<std::pair<std::string, int>> g_tuned;   // (device name, ngrid) done this process

int fail(int code, const char* what, cudaError_t e) {
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", what, e == cudaSuccess ? "" : cudaGetErrorString(e));
  return cg_set_error_from_lpt(code, buf);
}

std::string device_name() {
  int dev = 0;
  cudaDeviceProp prop;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
    return "unknown";
  std::string s = prop.name;
  for (auto& c : s)
    if (c == '\t' || c == '\n') c = ' ';
  return s;
}

// The last line of the cache file for (device, N), if any.
bool cache_lookup(const std::string& dev, int N, MeshSched* out) {
  const char* path = getenv("COLAGPU_TUNE_CACHE");
  if (!path || !*path) return false;
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char line[512];
  bool found = false;
  while (fgets(line, sizeof(line), f)) {
    char* tab = strchr(line, '\t');
    if (!tab) continue;
    *tab = 0;
    int n = 0, g = 0, x = 0;
    if (sscanf(tab + 1, "%d\t%d\t%d", &n, &g, &x) != 3) continue;
    if (dev == line && n == N) {
      out->green = g;
      out->fx = x;
      found = true;
    }
  }
  fclose(f);
  return found;
}

void cache_store(const std::string& dev, int N, MeshSched s) {
  const char* path = getenv("COLAGPU_TUNE_CACHE");
  if (!path || !*path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s\t%d\t%d\t%d\n", dev.c_str(), N, s.green, s.fx);
  fclose(f);
}

bool valid(int N, MeshSched s) {
  int ng = 0, nf = 0;
  if (!pm_num_variants(N, &ng, &nf)) return false;
  return s.green >= 0 && s.green < ng && s.fx >= 0 && s.fx < nf;
}

}  // namespace

extern "C" int cg_schedule_variants(int ngrid, int* n_green, int* n_fx) {
  if (!pm_num_variants(ngrid, n_green, n_fx))
    return cg_set_error_from_lpt(CG_EUNSUPPORTED, "cg_schedule_variants: mesh size not built");
  return CG_OK;
}

extern "C" int cg_get_schedule(int ngrid, int* green_variant, int* fx_variant) {
  if (!pm_supported_mesh(ngrid))
    return cg_set_error_from_lpt(CG_EUNSUPPORTED, "cg_get_schedule: mesh size not built");
  const MeshSched s = pm_get_schedule(ngrid);
  if (green_variant) *green_variant = s.green;
  if (fx_variant) *fx_variant = s.fx;
  return CG_OK;
}

extern "C" int cg_set_schedule(int ngrid, int green_variant, int fx_variant) {
  MeshSched s = pm_get_schedule(ngrid);   // keeps the deposit shape
  s.green = green_variant;
  s.fx = fx_variant;
  if (!valid(ngrid, s))
    return cg_set_error_from_lpt(CG_EINVAL, "cg_set_schedule: no such variant for this mesh size");
  pm_set_schedule(ngrid, s);
  return CG_OK;
}

extern "C" int cg_deposit_variants(void) { return PM_NUM_DEP_VARIANTS; }

extern "C" int cg_get_deposit_variant(int ngrid) {
  if (!pm_supported_mesh(ngrid))
    return cg_set_error_from_lpt(CG_EUNSUPPORTED, "cg_get_deposit_variant: mesh size not built");
  return pm_get_schedule(ngrid).dep;
}

extern "C" int cg_set_deposit_variant(int ngrid, int variant) {
  if (!pm_supported_mesh(ngrid) || variant < 0 || variant >= PM_NUM_DEP_VARIANTS)
    return cg_set_error_from_lpt(CG_EINVAL, "cg_set_deposit_variant: bad arguments");
  MeshSched s = pm_get_schedule(ngrid);
  s.dep = variant;
  pm_set_schedule(ngrid, s);
  return CG_OK;
}

extern "C" int cg_set_z_gather(int mode) {
  if (pm_set_z_gather(mode) != 0)
    return cg_set_error_from_lpt(CG_EINVAL, "cg_set_z_gather: mode must be -1, 0, 1 or 2");
  return CG_OK;
}

extern "C" int cg_set_force_deposit(int mode) {
  if (pm_set_force_deposit(mode) != 0)
    return cg_set_error_from_lpt(CG_EINVAL, "cg_set_force_deposit: mode must be -1, 0 or 1");
  return CG_OK;
}

extern "C" int cg_set_force_interp(int mode) {
  if (pm_set_force_interp(mode) != 0)
    return cg_set_error_from_lpt(CG_EINVAL, "cg_set_force_interp: mode must be -1, 0 or 1");
  return CG_OK;
}

extern "C" int cg_set_x_gather(int mode) {
  if (pm_set_x_gather(mode) != 0)
    return cg_set_error_from_lpt(CG_EINVAL, "cg_set_x_gather: mode must be -1, 0 or 1");
  return CG_OK;
}

extern "C" int cg_autotune(int ngrid, int flags, float* ms_green, float* ms_fx) {
  int ng = 0, nf = 0;
  if (!pm_num_variants(ngrid, &ng, &nf))
    return cg_set_error_from_lpt(CG_EUNSUPPORTED, "cg_autotune: mesh size not built");
  const std::string dev = device_name();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!(flags & CG_TUNE_FORCE)) {
    if (g_tuned.count({dev, ngrid})) return CG_OK;
    MeshSched c = pm_get_schedule(ngrid);
    if (cache_lookup(dev, ngrid, &c) && valid(ngrid, c)) {
      pm_set_schedule(ngrid, c);
      g_tuned.insert({dev, ngrid});
      return CG_OK;
    }
  }
  if (ng == 1 && nf == 1) {   // nothing to choose below 256
    MeshSched c = pm_get_schedule(ngrid);
    c.green = c.fx = 0;
    pm_set_schedule(ngrid, c);
    g_tuned.insert({dev, ngrid});
    return CG_OK;
  }
  PmPlan p;
  cudaError_t e = pm_plan_alloc(&p, ngrid, 1, 1.0f);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? CG_ENOMEM : CG_ECUDA, "cg_autotune: plan", e);
  MeshSched best;
  e = pm_autotune(&p, 0, &best, ms_green, ms_fx);
  pm_plan_free(&p);
  if (e != cudaSuccess) return fail(CG_ECUDA, "cg_autotune", e);
  best.dep = pm_get_schedule(ngrid).dep;
  pm_set_schedule(ngrid, best);
  g_tuned.insert({dev, ngrid});
  cache_store(dev, ngrid, best);
  return CG_OK;
}
