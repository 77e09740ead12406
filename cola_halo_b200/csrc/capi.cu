// C ABI of libcolagpu: the cg_* handle API and the drop-in replacements of
// the reference entry points (include/colagpu.h, include/colagpu_dropin.h).
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <memory>
#include <string>

#include "../../include/colagpu.h"
#include "../../include/colagpu_dropin.h"
#include "cosmo.h"
#include "internal.h"
#include "lpt.h"
#include "convnet.h"
#include "gadget.h"

#include <vector>

// ----------------------------------------------------------------- errors
static thread_local std::string g_err;

static int set_err(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

static int cuda_err(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return CG_OK;
  if (e == cudaErrorMemoryAllocation)
    return set_err(CG_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
  return set_err(CG_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CG_CHECK(expr, what)                         \
  do {                                               \
    cudaError_t _e = (expr);                         \
    if (_e != cudaSuccess) return cuda_err(_e, what); \
  } while (0)

extern "C" const char* cg_last_error(void) { return g_err.c_str(); }
extern "C" int cg_version(void) { return 1; }
extern "C" int cg_mesh_supported(int n) { return pm_supported_mesh(n) ? 1 : 0; }
extern "C" int cg_set_device(int dev) {
  CG_CHECK(cudaSetDevice(dev), "cudaSetDevice");
  return CG_OK;
}
extern "C" int cg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

extern "C" void* cg_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
    set_err(CG_ENOMEM, "cudaHostAlloc(%zu) failed", bytes);
    return nullptr;
  }
  return p;
}
extern "C" void cg_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

// ------------------------------------------------------------ cg_sim
struct cg_sim {
  int nc = 0;
  float L = 0;
  double omega_m = 0;
  std::unique_ptr<ColaTime> ct;
  PmPlan pm{};
  ParticleSoA ps{};
  float a_x = 0, a_v = 0;
  cudaStream_t st = nullptr;
  void* d_aos = nullptr;      // staging: Particle (56 B) / ParticleMinimum (32 B) arrays
  bool aos_snapshot = false;  // d_aos holds the last snapshot (ParticleMinimum[n])
  float* soa_block = nullptr; // one allocation for all SoA float arrays
  long long* id_alloc = nullptr;
  int* orig_alloc = nullptr;
  ParticleOrder order;        // cell-order sort (reorder.cu)
  int sort_every = 0;         // sort at every sort_every-th move (0: never)
  long long moves = 0;
  bool sorted = false;        // the arrays are in an order of their own
};

static void sim_free(cg_sim* s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  pm_plan_free(&s->pm);
  particle_order_free(&s->order);
  cudaFree(s->soa_block);
  cudaFree(s->id_alloc);
  cudaFree(s->orig_alloc);
  cudaFree(s->d_aos);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

static bool force_kernel_ok(int gradient, int laplacian, int deconvolve) {
  return (gradient == 0 || gradient == 2 || gradient == 4) && (laplacian == 0 || laplacian == 1) &&
         deconvolve >= 0 && deconvolve <= 2;
}

extern "C" int cg_sim_create(cg_sim** out, int nc, int ngrid, float boxsize, double omega_m,
                             long long np_capacity) {
  if (!out) return set_err(CG_EINVAL, "cg_sim_create: out is NULL");
  *out = nullptr;
  if (nc <= 0 || ngrid <= 0 || !(boxsize > 0.0f) || !(omega_m > 0.0 && omega_m <= 1.0))
    return set_err(CG_EINVAL, "cg_sim_create: bad nc=%d ngrid=%d boxsize=%g omega_m=%g", nc,
                   ngrid, boxsize, omega_m);
  if (!pm_supported_mesh(ngrid))
    return set_err(CG_EUNSUPPORTED, "mesh size %d is not built into this library", ngrid);
  const long long npl = (long long)nc * nc * nc;
  if (np_capacity < npl) np_capacity = npl;
  cg_sim* s = new cg_sim();
  s->nc = nc;
  s->L = boxsize;
  s->omega_m = omega_m;
  s->ct.reset(new ColaTime(omega_m));
  cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = pm_plan_alloc(&s->pm, ngrid, ngrid / nc > 0 ? ngrid / nc : 1, boxsize);
  // a particle's mass in mesh units, (ngrid / nc)^3 (pm.c:216 for integer
  // factors; a mesh that is no multiple of nc, e.g. 192 for 128^3, too)
  if (e == cudaSuccess) s->pm.wpar = (float)pow((double)ngrid / nc, 3.0);
  if (e == cudaSuccess) {
    s->ps.cap = np_capacity;
    e = cudaMalloc(&s->soa_block, sizeof(float) * 15 * (size_t)np_capacity);
  }
  if (e == cudaSuccess) e = cudaMalloc(&s->id_alloc, sizeof(long long) * (size_t)np_capacity);
  if (e == cudaSuccess) e = cudaMalloc(&s->orig_alloc, sizeof(int) * (size_t)np_capacity);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_aos, 56 * (size_t)np_capacity);
  s->ps.id = s->id_alloc;
  s->ps.orig = s->orig_alloc;
  // the sort pays only where the particles and meshes are far larger than
  // L2 (128^3 particles lose 0.1 ms a step), and there every sixth move:
  // 10-step runs of 256^3 particles take 11.57 ms a step against 11.89 sorting
  // every second move and 11.87 never; 512^3 on 1024^3, 38.3 against 40.6 ms
  s->sort_every = np_capacity >= (1LL << 23) ? 6 : 0;
  if (const char* ev = getenv("COLAGPU_SORT_EVERY")) s->sort_every = atoi(ev) > 0 ? atoi(ev) : 0;
  // COLAGPU_FORCE_KERNEL=g,l,d selects the force kernel of every new
  // realization (cg_sim_set_force_kernel), the drop-in's included
  if (const char* ev = getenv("COLAGPU_FORCE_KERNEL")) {
    int g = 0, l = 0, d = 0;
    if (sscanf(ev, "%d,%d,%d", &g, &l, &d) == 3 && force_kernel_ok(g, l, d)) {
      if (e == cudaSuccess) e = pm_set_force_kernel(&s->pm, g, l, d);
    } else {
      fprintf(stderr, "libcolagpu: COLAGPU_FORCE_KERNEL=%s ignored (want g,l,d)\n", ev);
    }
  }
  if (e != cudaSuccess) {
    int rc = cuda_err(e, "cg_sim_create");
    sim_free(s);
    return rc;
  }
  float* b = s->soa_block;
  const size_t c = (size_t)np_capacity;
  for (int a = 0; a < 3; a++) {
    s->ps.x[a] = b + (0 + a) * c;
    s->ps.v[a] = b + (3 + a) * c;
    s->ps.dx1[a] = b + (6 + a) * c;
    s->ps.dx2[a] = b + (9 + a) * c;
    s->ps.f[a] = b + (12 + a) * c;
  }
  cudaMemsetAsync(s->soa_block, 0, sizeof(float) * 15 * c, s->st);
  *out = s;
  return CG_OK;
}

extern "C" void cg_sim_destroy(cg_sim* s) { sim_free(s); }

static bool is_device_ptr(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

extern "C" int cg_sim_set_particles(cg_sim* s, const void* particles, long long np, float a_x,
                                    float a_v) {
  if (!s || (!particles && np > 0)) return set_err(CG_EINVAL, "cg_sim_set_particles: NULL");
  if (np < 0 || np > s->ps.cap)
    return set_err(CG_EINVAL, "cg_sim_set_particles: np=%lld exceeds capacity %lld", np,
                   s->ps.cap);
  // forces already computed keep their meaning for particles given again in
  // the same order (the caller's order, which the upload restores)
  if (s->sorted) CG_CHECK(particles_unsort_forces(&s->ps, &s->order, s->st), "unsort forces");
  s->sorted = false;
  s->ps.n = np;
  s->a_x = a_x;
  s->a_v = a_v;
  s->aos_snapshot = false;
  s->moves = 0;
  if (np == 0) return CG_OK;
  const cudaMemcpyKind kind =
      is_device_ptr(particles) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CG_CHECK(cudaMemcpyAsync(s->d_aos, particles, 56 * (size_t)np, kind, s->st), "upload particles");
  CG_CHECK(particles_aos_to_soa(s->d_aos, &s->ps, s->st), "aos_to_soa");
  return CG_OK;
}

extern "C" int cg_sim_get_particles(cg_sim* s, void* particles) {
  if (!s || !particles) return set_err(CG_EINVAL, "cg_sim_get_particles: NULL");
  if (s->ps.n == 0) return CG_OK;
  s->aos_snapshot = false;
  CG_CHECK(particles_soa_to_aos(s->d_aos, &s->ps, s->st), "soa_to_aos");
  CG_CHECK(cudaMemcpyAsync(particles, s->d_aos, 56 * (size_t)s->ps.n, cudaMemcpyDefault, s->st),
           "download particles");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");
  return CG_OK;
}

extern "C" int cg_sim_get_forces(cg_sim* s, float* f) {
  if (!s || !f) return set_err(CG_EINVAL, "cg_sim_get_forces: NULL");
  const size_t n = (size_t)s->ps.n;
  if (n == 0) return CG_OK;
  // interleave on the host side: copy three component arrays into (n,3),
  // each particle at its caller's index
  float* tmp = (float*)malloc(sizeof(float) * 3 * n);
  int* orig = (int*)malloc(sizeof(int) * n);
  if (!tmp || !orig) {
    free(tmp);
    free(orig);
    return set_err(CG_ENOMEM, "host malloc");
  }
  cudaError_t e = cudaSuccess;
  for (int a = 0; a < 3 && e == cudaSuccess; a++)
    e = cudaMemcpyAsync(tmp + a * n, s->ps.f[a], sizeof(float) * n, cudaMemcpyDeviceToHost,
                        s->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(orig, s->ps.orig, sizeof(int) * n, cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) {
    free(tmp);
    free(orig);
    return cuda_err(e, "download forces");
  }
  for (size_t i = 0; i < n; i++) {
    const size_t j = (size_t)orig[i] < n ? (size_t)orig[i] : i;
    for (int a = 0; a < 3; a++) f[3 * j + a] = tmp[a * n + i];
  }
  free(tmp);
  free(orig);
  return CG_OK;
}

extern "C" int cg_sim_get_times(cg_sim* s, float* a_x, float* a_v) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_get_times: NULL");
  if (a_x) *a_x = s->a_x;
  if (a_v) *a_v = s->a_v;
  return CG_OK;
}

extern "C" long long cg_sim_np(cg_sim* s) { return s ? s->ps.n : -1; }
extern "C" void* cg_sim_stream(cg_sim* s) { return s ? (void*)s->st : nullptr; }

extern "C" int cg_sim_move(cg_sim* s) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_move: NULL");
  CG_CHECK(dev_wrap(s->ps.x, s->ps.n, s->L, s->st), "wrap");
  if (s->sort_every > 0 && ++s->moves % s->sort_every == 0) {
    // the caller's view is unchanged: outputs go back through orig
    s->aos_snapshot = false;
    CG_CHECK(particles_sort_cells(&s->ps, &s->order, s->L, s->st), "cell-order sort");
    s->sorted = true;
  }
  return CG_OK;
}

extern "C" int cg_sim_set_force_kernel(cg_sim* s, int gradient, int laplacian, int deconvolve) {
  if (!s || !force_kernel_ok(gradient, laplacian, deconvolve))
    return set_err(CG_EINVAL, "cg_sim_set_force_kernel: bad arguments");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");    // no queued Green step reads the old tables
  CG_CHECK(pm_set_force_kernel(&s->pm, gradient, laplacian, deconvolve), "force kernel");
  return CG_OK;
}

extern "C" int cg_sim_set_force_filters(cg_sim* s, const float* knots, int n, int nsets) {
  if (!s || n < 0 || nsets < 0 || ((long long)n * nsets > 0 && !knots) || n == 1)
    return set_err(CG_EINVAL, "cg_sim_set_force_filters: bad arguments");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");    // no queued Green step reads the old table
  CG_CHECK(pm_set_filters(&s->pm, knots, n, nsets), "force filters");
  return CG_OK;
}

extern "C" int cg_sim_use_force_filter(cg_sim* s, int set) {
  if (!s || !pm_use_filter(&s->pm, set))
    return set_err(CG_EINVAL, "cg_sim_use_force_filter: no such filter");
  return CG_OK;
}

extern "C" int cg_sim_set_sort_interval(cg_sim* s, int every) {
  if (!s || every < 0) return set_err(CG_EINVAL, "cg_sim_set_sort_interval: bad arguments");
  s->sort_every = every;
  return CG_OK;
}

static int check_err_word(cg_sim* s) {
  unsigned err = 0;
  CG_CHECK(cudaMemcpyAsync(&err, s->pm.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s->st),
           "read error word");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");
  if (err & CG_ERR_TMA_WAIT) {
    cudaMemsetAsync(s->pm.err, 0, sizeof(unsigned), s->st);
    return set_err(CG_ECUDA, "z transform: a TMA gather did not complete (error word 0x%x)", err);
  }
  if (err) {
    cudaMemsetAsync(s->pm.err, 0, sizeof(unsigned), s->st);
    return set_err(CG_EPARTICLE, "particle position %s (device error word 0x%x)",
                   (err & CG_ERR_NONFINITE) ? "not finite" : "below zero in y or z", err);
  }
  return CG_OK;
}

extern "C" int cg_sim_forces(cg_sim* s, double* density_sum) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_forces: NULL");
  const float* x[3] = {s->ps.x[0], s->ps.x[1], s->ps.x[2]};
  CG_CHECK(pm_forces(&s->pm, x, s->ps.n, s->ps.f, s->st), "pm_forces");
  if (density_sum) {
    CG_CHECK(cudaMemcpyAsync(density_sum, s->pm.dsum, sizeof(double), cudaMemcpyDeviceToHost,
                             s->st), "read density sum");
    int rc = check_err_word(s);
    if (rc) return rc;
  }
  return CG_OK;
}

extern "C" int cg_sim_kick_coeffs(cg_sim* s, float dda, float q1, float q2) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_kick_coeffs: NULL");
  const float* f[3] = {s->ps.f[0], s->ps.f[1], s->ps.f[2]};
  const float* d1[3] = {s->ps.dx1[0], s->ps.dx1[1], s->ps.dx1[2]};
  const float* d2[3] = {s->ps.dx2[0], s->ps.dx2[1], s->ps.dx2[2]};
  CG_CHECK(dev_kick(s->ps.v, f, d1, d2, s->ps.n, s->ct->om32, dda, q1, q2, s->st), "kick");
  return CG_OK;
}

extern "C" int cg_sim_drift_coeffs(cg_sim* s, float dyyy, float da1, float da2) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_drift_coeffs: NULL");
  const float* v[3] = {s->ps.v[0], s->ps.v[1], s->ps.v[2]};
  const float* d1[3] = {s->ps.dx1[0], s->ps.dx1[1], s->ps.dx1[2]};
  const float* d2[3] = {s->ps.dx2[0], s->ps.dx2[1], s->ps.dx2[2]};
  CG_CHECK(dev_drift(s->ps.x, v, d1, d2, s->ps.n, dyyy, da1, da2, s->st), "drift");
  return CG_OK;
}

// kick with (dda, q1, q2), then drift with (dyyy, da1, da2) and the kicked
// velocity, in one pass
static int sim_kick_drift(cg_sim* s, float dda, float q1, float q2, float dyyy, float da1,
                          float da2) {
  const float* f[3] = {s->ps.f[0], s->ps.f[1], s->ps.f[2]};
  const float* d1[3] = {s->ps.dx1[0], s->ps.dx1[1], s->ps.dx1[2]};
  const float* d2[3] = {s->ps.dx2[0], s->ps.dx2[1], s->ps.dx2[2]};
  CG_CHECK(dev_kick_drift(s->ps.x, s->ps.v, f, d1, d2, s->ps.n, s->ct->om32, dda, q1, q2, dyyy,
                          da1, da2, s->st),
           "kick_drift");
  return CG_OK;
}

extern "C" int cg_sim_kick(cg_sim* s, float avel1) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_kick: NULL");
  float dda, q1, q2;
  s->ct->kick(s->a_v, s->a_x, avel1, &dda, &q1, &q2);
  int rc = cg_sim_kick_coeffs(s, dda, q1, q2);
  if (rc) return rc;
  s->a_v = avel1;
  return CG_OK;
}

extern "C" int cg_sim_drift(cg_sim* s, float apos1) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_drift: NULL");
  float dyyy, da1, da2;
  s->ct->drift(s->a_x, s->a_v, apos1, &dyyy, &da1, &da2);
  int rc = cg_sim_drift_coeffs(s, dyyy, da1, da2);
  if (rc) return rc;
  s->a_x = apos1;
  return CG_OK;
}

// cg_sim_kick(avel1) then cg_sim_drift(apos1) in one pass over the particles.
extern "C" int cg_sim_kick_drift(cg_sim* s, float avel1, float apos1) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_kick_drift: NULL");
  float dda, q1, q2, dyyy, da1, da2;
  s->ct->kick(s->a_v, s->a_x, avel1, &dda, &q1, &q2);
  s->ct->drift(s->a_x, avel1, apos1, &dyyy, &da1, &da2);
  const int rc = sim_kick_drift(s, dda, q1, q2, dyyy, da1, da2);
  if (rc) return rc;
  s->a_v = avel1;
  s->a_x = apos1;
  return CG_OK;
}

// cola.c:341-384: coefficients of the final half kick and drift to aout.
static int queue_snapshot(cg_sim* s, double aout, float omega_m, void* d_out) {
  ColaTime ct(omega_m);
  const float vfac = (float)(100.0 / aout);
  const float AF = (float)aout;
  float dda, q1, q2, dyyy, da1, da2;
  ct.kick(s->a_v, s->a_x, AF, &dda, &q1, &q2);
  ct.drift(s->a_x, s->a_v, AF, &dyyy, &da1, &da2);
  const float Dv = (float)ct.DprimeQ((double)AF, 1.0);
  const float Dv2 = (float)ct.D2v((double)AF);
  const float* x[3] = {s->ps.x[0], s->ps.x[1], s->ps.x[2]};
  const float* v[3] = {s->ps.v[0], s->ps.v[1], s->ps.v[2]};
  const float* f[3] = {s->ps.f[0], s->ps.f[1], s->ps.f[2]};
  const float* d1[3] = {s->ps.dx1[0], s->ps.dx1[1], s->ps.dx1[2]};
  const float* d2[3] = {s->ps.dx2[0], s->ps.dx2[1], s->ps.dx2[2]};
  CG_CHECK(dev_snapshot(x, v, f, d1, d2, s->ps.n, ct.om32, dda, q1, q2, Dv, Dv2, dyyy, da1,
                         da2, vfac, s->ps.id, s->ps.orig, d_out, s->st),
           "snapshot");
  return CG_OK;
}

extern "C" int cg_sim_snapshot(cg_sim* s, double aout, float omega_m, void* pmin_out) {
  if (!s || !pmin_out) return set_err(CG_EINVAL, "cg_sim_snapshot: NULL");
  int rc = queue_snapshot(s, aout, omega_m, s->d_aos);
  if (rc) return rc;
  s->aos_snapshot = true;
  CG_CHECK(cudaMemcpyAsync(pmin_out, s->d_aos, 32 * (size_t)s->ps.n, cudaMemcpyDefault, s->st),
           "download snapshot");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");
  return CG_OK;
}

// set_noncola_initial (cola.c:297-338) on the device: the snapshot of the
// 2LPT initial condition at a_x, downloaded into pmin_out.
extern "C" int cg_sim_initial_snapshot(cg_sim* s, float omega_m, void* pmin_out) {
  if (!s || !pmin_out) return set_err(CG_EINVAL, "cg_sim_initial_snapshot: NULL");
  const float aout = s->a_x;
  ColaTime ct(omega_m);
  const float vfac = 100.0f / aout;                              // cola.c:310
  const float Dv = (float)ct.DprimeQ((double)aout, 1.0);         // cola.c:312
  const float Dv2 = (float)ct.D2v((double)aout);                 // cola.c:313
  CG_CHECK(dev_initial_snapshot(&s->ps, vfac, Dv, Dv2, s->d_aos, s->st), "initial snapshot");
  s->aos_snapshot = true;
  CG_CHECK(cudaMemcpyAsync(pmin_out, s->d_aos, 32 * (size_t)s->ps.n, cudaMemcpyDefault, s->st),
           "download snapshot");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");
  return CG_OK;
}

extern "C" int cg_sim_write_gadget(cg_sim* s, double aout, float omega_m, float h,
                                   const char* filename, int use_long_id) {
  if (!s || !filename) return set_err(CG_EINVAL, "cg_sim_write_gadget: NULL");
  int rc = queue_snapshot(s, aout, omega_m, s->d_aos);
  if (rc) return rc;
  s->aos_snapshot = true;
  return gadget_write(filename, s->d_aos, true, s->ps.n, s->ps.n, 1, (float)aout, s->L, omega_m,
                      h, use_long_id, s->st);
}

extern "C" int cg_sim_sync(cg_sim* s) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_sync: NULL");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");
  return check_err_word(s);
}

extern "C" int cg_sim_power_spectrum(cg_sim* s, int nbins, int flags, double* k, double* pk,
                                     double* nmodes) {
  if (!s || !k || !pk || nbins < 1 || nbins > s->pm.N)
    return set_err(CG_EINVAL, "cg_sim_power_spectrum: bad arguments");
  const float* x[3] = {s->ps.x[0], s->ps.x[1], s->ps.x[2]};
  CG_CHECK(pm_power_spectrum(&s->pm, x, s->ps.n, nbins, flags & CG_PK_DECONVOLVE_CIC,
                             s->pm.pk_acc, s->st),
           "power spectrum");
  double* h = (double*)malloc(sizeof(double) * 3 * nbins);
  if (!h) return set_err(CG_ENOMEM, "host malloc");
  cudaError_t e = cudaMemcpyAsync(h, s->pm.pk_acc, sizeof(double) * 3 * nbins,
                                  cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) {
    free(h);
    return cuda_err(e, "power spectrum readback");
  }
  const double N = s->pm.N, L = s->L;
  const double kf = 2.0 * M_PI / L;
  const double norm = L * L * L / (N * N * N * N * N * N);
  const double shot = (flags & CG_PK_SUBTRACT_SHOT) && s->ps.n > 0 ? L * L * L / (double)s->ps.n
                                                                   : 0.0;
  for (int b = 0; b < nbins; b++) {
    const double w = h[b];
    k[b] = w > 0 ? kf * h[nbins + b] / w : 0.0;
    pk[b] = w > 0 ? norm * h[2 * nbins + b] / w - shot : 0.0;
    if (nmodes) nmodes[b] = w;
  }
  free(h);
  return CG_OK;
}

extern "C" int cg_sim_tune_deposit(cg_sim* s, float* ms) {
  if (!s || s->ps.n < 1) return set_err(CG_EINVAL, "cg_sim_tune_deposit: no particles");
  // the deposit takes positions inside the box, as after cg_sim_move
  CG_CHECK(dev_wrap(s->ps.x, s->ps.n, s->L, s->st), "wrap");
  const float* x[3] = {s->ps.x[0], s->ps.x[1], s->ps.x[2]};
  int best = 0;
  CG_CHECK(pm_tune_deposit(&s->pm, x, s->ps.n, s->st, &best, ms), "tune deposit");
  MeshSched m = pm_get_schedule(s->pm.N);
  m.dep = best;
  pm_set_schedule(s->pm.N, m);
  return best;
}

// ------------------------------------------------ slab decomposition
// The per-rank stages of a force split over x slabs (pm_slab_* in
// pm_kernels.cu); the caller moves the spectra and the buffer copies
// between ranks.  bx / bf: SoA device arrays of nb floats per component.

extern "C" int cg_sim_state_ptrs(cg_sim* s, float** x, float** f) {
  if (!s || !x || !f) return set_err(CG_EINVAL, "cg_sim_state_ptrs: NULL");
  for (int a = 0; a < 3; a++) {
    x[a] = s->ps.x[a];
    f[a] = s->ps.f[a];
  }
  return CG_OK;
}

extern "C" int cg_sim_spectrum_ptr(cg_sim* s, int which, void** ptr) {
  if (!s || !ptr || which < 0 || which > 3)
    return set_err(CG_EINVAL, "cg_sim_spectrum_ptr: bad arguments");
  *ptr = which == 0 ? (void*)s->pm.spec : (void*)s->pm.gsp[which - 1];
  return CG_OK;
}

static void soa3(const float* base, long long n, const float* out[3]) {
  for (int a = 0; a < 3; a++) out[a] = base ? base + a * n : nullptr;
}

extern "C" int cg_sim_slab_density(cg_sim* s, int x0, int nx, const float* bx, long long nb,
                                   double* density_sum) {
  if (!s || nb < 0 || (nb > 0 && !bx)) return set_err(CG_EINVAL, "cg_sim_slab_density: bad arguments");
  const float* x[3] = {s->ps.x[0], s->ps.x[1], s->ps.x[2]};
  const float* b[3];
  soa3(bx, nb, b);
  CG_CHECK(pm_slab_density(&s->pm, x0, nx, x, s->ps.n, b, nb, s->st), "slab density");
  if (density_sum) {
    CG_CHECK(cudaMemcpyAsync(density_sum, s->pm.dsum, sizeof(double), cudaMemcpyDeviceToHost,
                             s->st), "read density sum");
    int rc = check_err_word(s);
    if (rc) return rc;
  }
  return CG_OK;
}

extern "C" int cg_sim_slab_kspace(cg_sim* s, int kz0, int nkz) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_slab_kspace: NULL");
  CG_CHECK(pm_slab_kspace(&s->pm, kz0, nkz, s->st), "slab kspace");
  return CG_OK;
}

extern "C" int cg_sim_slab_c2r(cg_sim* s, int x0, int nx) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_slab_c2r: NULL");
  CG_CHECK(pm_slab_c2r(&s->pm, x0, nx, s->st), "slab c2r");
  return CG_OK;
}

extern "C" int cg_sim_slab_interp(cg_sim* s, int x0, int nx, const float* bx, long long nb,
                                  float* bf) {
  if (!s || nb < 0 || (nb > 0 && (!bx || !bf)))
    return set_err(CG_EINVAL, "cg_sim_slab_interp: bad arguments");
  const float* x[3] = {s->ps.x[0], s->ps.x[1], s->ps.x[2]};
  const float* b[3];
  soa3(bx, nb, b);
  float* fb[3] = {bf, bf ? bf + nb : nullptr, bf ? bf + 2 * nb : nullptr};
  CG_CHECK(pm_slab_interp(&s->pm, x0, nx, x, s->ps.n, s->ps.f, b, nb, fb, s->st),
           "slab interp");
  return CG_OK;
}

extern "C" int cg_sim_keep_density(cg_sim* s, int keep) {
  if (!s) return set_err(CG_EINVAL, "cg_sim_keep_density: null handle");
  s->pm.keep_dens = keep != 0;
  return CG_OK;
}

extern "C" int cg_sim_get_mesh(cg_sim* s, int which, float* out) {
  if (!s || !out || which < 0 || which > 3) return set_err(CG_EINVAL, "cg_sim_get_mesh: bad args");
  if (which == 0 && (s->pm.dens_reset || s->pm.dens_stale)) {
    // the force step consumed the density, or built it in shared memory
    // only: deposit the current positions again
    const float* x[3] = {s->ps.x[0], s->ps.x[1], s->ps.x[2]};
    CG_CHECK(pm_deposit(&s->pm, x, s->ps.n, s->st), "deposit");
  }
  if (which > 0) {
    // the interpolation from the z c2r's tiles wrote no force mesh
    CG_CHECK(pm_force_mesh(&s->pm, which - 1, s->st), "force mesh");
  }
  const float* src = which == 0 ? s->pm.dens : s->pm.fmesh[which - 1];
  CG_CHECK(cudaMemcpyAsync(out, src, s->pm.mesh_bytes, cudaMemcpyDeviceToHost, s->st), "get mesh");
  CG_CHECK(cudaStreamSynchronize(s->st), "sync");
  return CG_OK;
}

extern "C" int cg_sim_copy_particles(cg_sim* dst, const cg_sim* src) {
  if (!dst || !src || src->ps.n > dst->ps.cap)
    return set_err(CG_EINVAL, "cg_sim_copy_particles: bad arguments");
  CG_CHECK(cudaStreamSynchronize(src->st), "sync");
  const size_t n = (size_t)src->ps.n;
  for (int a = 0; a < 3; a++) {
    CG_CHECK(cudaMemcpyAsync(dst->ps.x[a], src->ps.x[a], 4 * n, cudaMemcpyDeviceToDevice, dst->st), "copy");
    CG_CHECK(cudaMemcpyAsync(dst->ps.v[a], src->ps.v[a], 4 * n, cudaMemcpyDeviceToDevice, dst->st), "copy");
    CG_CHECK(cudaMemcpyAsync(dst->ps.dx1[a], src->ps.dx1[a], 4 * n, cudaMemcpyDeviceToDevice, dst->st), "copy");
    CG_CHECK(cudaMemcpyAsync(dst->ps.dx2[a], src->ps.dx2[a], 4 * n, cudaMemcpyDeviceToDevice, dst->st), "copy");
  }
  CG_CHECK(cudaMemcpyAsync(dst->ps.id, src->ps.id, 8 * n, cudaMemcpyDeviceToDevice, dst->st), "copy");
  CG_CHECK(cudaMemcpyAsync(dst->ps.orig, src->ps.orig, 4 * n, cudaMemcpyDeviceToDevice, dst->st),
           "copy");
  dst->ps.n = src->ps.n;
  dst->sorted = src->sorted;
  dst->aos_snapshot = false;
  dst->a_x = src->a_x;
  dst->a_v = src->a_v;
  return CG_OK;
}

// ---------------------------------------------------- learned correction
struct cg_net {
  CNet n{};
  cudaStream_t st = nullptr;
};

extern "C" int cg_net_create(cg_net** out, int ngrid, unsigned long long seed) {
  if (!out || !pm_supported_mesh(ngrid)) return set_err(CG_EINVAL, "cg_net_create: bad mesh");
  cg_net* h = new cg_net();
  cudaError_t e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cnet_alloc(&h->n, ngrid, seed);
  if (e != cudaSuccess) {
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return cuda_err(e, "cg_net_create");
  }
  h->n.use_tc = 1;
  *out = h;
  return CG_OK;
}

extern "C" void cg_net_destroy(cg_net* h) {
  if (!h) return;
  cudaStreamSynchronize(h->st);
  cnet_free(&h->n);
  cudaStreamDestroy(h->st);
  delete h;
}

extern "C" int cg_net_set_tensor_cores(cg_net* h, int on) {
  if (!h) return set_err(CG_EINVAL, "cg_net_set_tensor_cores: NULL");
  h->n.use_tc = on ? 1 : 0;
  return CG_OK;
}

extern "C" int cg_net_set_conv_variant(int variant) {
  if (conv_tc_set_variant(variant) != 0)
    return set_err(CG_EINVAL, "cg_net_set_conv_variant: variant must be -1, 0, 1 or 2");
  return CG_OK;
}

extern "C" int cg_net_set_scales(cg_net* h, float in_delta, float in_phi, float out_scale) {
  if (!h || !(out_scale > 0)) return set_err(CG_EINVAL, "cg_net_set_scales: bad arguments");
  h->n.in_scale[0] = in_delta;
  h->n.in_scale[1] = in_phi;
  h->n.out_scale = out_scale;
  return CG_OK;
}

extern "C" int cg_net_get_params(cg_net* h, float* out) {
  if (!h || !out) return set_err(CG_EINVAL, "cg_net_get_params: NULL");
  CG_CHECK(cudaMemcpyAsync(out, h->n.params, sizeof(float) * CNET_PARAMS, cudaMemcpyDeviceToHost,
                           h->st), "get params");
  CG_CHECK(cudaStreamSynchronize(h->st), "sync");
  return CG_OK;
}

extern "C" int cg_net_set_params(cg_net* h, const float* p) {
  if (!h || !p) return set_err(CG_EINVAL, "cg_net_set_params: NULL");
  CG_CHECK(cudaMemcpyAsync(h->n.params, p, sizeof(float) * CNET_PARAMS, cudaMemcpyHostToDevice,
                           h->st), "set params");
  CG_CHECK(cnet_sync_bf16(&h->n, h->st), "bf16 weights");
  CG_CHECK(cudaStreamSynchronize(h->st), "sync");
  return CG_OK;
}

extern "C" int cg_net_num_params(void) { return CNET_PARAMS; }

// Host-array entry points (checks and tools): in2 = [v][2] features
// (already scaled), out3 = [v][3] raw network output, grad3 = dL/dout.
static int net_load_input(cg_net* h, const float* in2) {
  const size_t nv = (size_t)h->n.N * h->n.N * h->n.N;
  std::vector<__nv_bfloat16> b(nv * CNET_C, __float2bfloat16_rn(0.0f));
  for (size_t v = 0; v < nv; v++) {
    b[v * CNET_C] = __float2bfloat16_rn(in2[2 * v]);
    b[v * CNET_C + 1] = __float2bfloat16_rn(in2[2 * v + 1]);
  }
  CG_CHECK(cudaMemcpyAsync(h->n.act[0], b.data(), b.size() * sizeof(__nv_bfloat16),
                           cudaMemcpyHostToDevice, h->st), "upload input");
  CG_CHECK(cudaStreamSynchronize(h->st), "sync");
  return CG_OK;
}

static int net_check_tc() {
  if (conv_tc_error_word()) return set_err(CG_ECUDA, "tensor-core convolution wait timed out");
  return CG_OK;
}

extern "C" int cg_net_forward_host(cg_net* h, const float* in2, float* out3) {
  if (!h || !in2 || !out3) return set_err(CG_EINVAL, "cg_net_forward_host: NULL");
  int rc = net_load_input(h, in2);
  if (rc) return rc;
  CG_CHECK(cnet_forward(&h->n, h->st), "forward");
  const size_t nv = (size_t)h->n.N * h->n.N * h->n.N;
  std::vector<float> o(nv * CNET_C);
  CG_CHECK(cudaMemcpyAsync(o.data(), h->n.out, o.size() * 4, cudaMemcpyDeviceToHost, h->st), "dl");
  CG_CHECK(cudaStreamSynchronize(h->st), "sync");
  for (size_t v = 0; v < nv; v++)
    for (int c = 0; c < 3; c++) out3[3 * v + c] = o[v * CNET_C + c];
  return net_check_tc();
}

extern "C" int cg_net_backward_host(cg_net* h, const float* in2, const float* grad3,
                                    float* grads) {
  if (!h || !in2 || !grad3 || !grads) return set_err(CG_EINVAL, "cg_net_backward_host: NULL");
  int rc = net_load_input(h, in2);
  if (rc) return rc;
  CG_CHECK(cnet_forward(&h->n, h->st), "forward");
  const size_t nv = (size_t)h->n.N * h->n.N * h->n.N;
  std::vector<float> g(nv * CNET_C, 0.0f);
  for (size_t v = 0; v < nv; v++)
    for (int c = 0; c < 3; c++) g[v * CNET_C + c] = grad3[3 * v + c];
  CG_CHECK(cudaMemcpyAsync(h->n.g0, g.data(), g.size() * 4, cudaMemcpyHostToDevice, h->st), "ul");
  CG_CHECK(cnet_backward(&h->n, h->st), "backward");
  CG_CHECK(cudaMemcpyAsync(grads, h->n.grads, sizeof(float) * CNET_PARAMS, cudaMemcpyDeviceToHost,
                           h->st), "dl");
  CG_CHECK(cudaStreamSynchronize(h->st), "sync");
  return net_check_tc();
}

// One training step on the current particles of two realizations holding
// the same particles: coarse (the net's mesh) and fine (the target mesh).
extern "C" int cg_net_train_step(cg_net* h, cg_sim* coarse, cg_sim* fine, float lr,
                                 double* loss) {
  if (!h || !coarse || !fine || coarse->pm.N != h->n.N || coarse->ps.n != fine->ps.n)
    return set_err(CG_EINVAL, "cg_net_train_step: bad arguments");
  coarse->pm.keep_dens = true;   // the net's features read the density after the force
  int rc = cg_sim_forces(coarse, nullptr);
  if (!rc) rc = cg_sim_forces(fine, nullptr);
  if (rc) return rc;
  CG_CHECK(cudaStreamSynchronize(fine->st), "sync fine");
  CG_CHECK(cudaStreamSynchronize(coarse->st), "sync coarse");
  cudaStream_t st = h->st;
  const float* x[3] = {coarse->ps.x[0], coarse->ps.x[1], coarse->ps.x[2]};
  const float* ff[3] = {fine->ps.f[0], fine->ps.f[1], fine->ps.f[2]};
  const float* fc[3] = {coarse->ps.f[0], coarse->ps.f[1], coarse->ps.f[2]};
  CG_CHECK(cnet_features(&h->n, coarse->pm.dens, st), "features");
  CG_CHECK(cnet_target(&h->n, x, coarse->ps.n, coarse->L, ff, fc, st), "target");
  CG_CHECK(cnet_forward(&h->n, st), "forward");
  CG_CHECK(cnet_loss_grad(&h->n, 1.0 / (double)coarse->ps.n, st), "loss");
  CG_CHECK(cnet_backward(&h->n, st), "backward");
  if (lr > 0) CG_CHECK(cnet_adam(&h->n, lr, st), "adam");
  if (loss) {
    CG_CHECK(cudaMemcpyAsync(loss, h->n.loss, sizeof(double), cudaMemcpyDeviceToHost, st), "loss");
  }
  CG_CHECK(cudaStreamSynchronize(st), "sync");
  return net_check_tc();
}

// Forces of the coarse realization with the learned correction added.
extern "C" int cg_net_forces(cg_net* h, cg_sim* coarse) {
  if (!h || !coarse || coarse->pm.N != h->n.N) return set_err(CG_EINVAL, "cg_net_forces: bad");
  coarse->pm.keep_dens = true;   // the net's features read the density after the force
  int rc = cg_sim_forces(coarse, nullptr);
  if (rc) return rc;
  cudaStream_t st = coarse->st;   // stay on the realization's stream
  const float* x[3] = {coarse->ps.x[0], coarse->ps.x[1], coarse->ps.x[2]};
  CG_CHECK(cnet_features(&h->n, coarse->pm.dens, st), "features");
  CG_CHECK(cnet_forward(&h->n, st, false), "forward");
  CG_CHECK(cnet_apply(&h->n, x, coarse->ps.n, coarse->L, coarse->ps.f, st), "apply");
  return CG_OK;
}

// ------------------------------------------------------ mesh transforms
// Unnormalised 3-D r2c / c2r of host arrays through the device mesh passes
// (real [x][y][z], half spectrum [kx][ky][kz], kz = 0..n/2, complex
// interleaved), synchronous.  The c2r ignores Im of kz = 0 and n/2.
static int host_fft(int n, const float* in, float* out, bool forward) {
  if (!pm_supported_mesh(n) || !in || !out) return set_err(CG_EINVAL, "cg_fft: bad arguments");
  MeshFFT f;
  CG_CHECK(mesh_fft_alloc(&f, n), "mesh_fft_alloc");
  const size_t nh = (size_t)(n / 2 + 1);
  const size_t rb = sizeof(float) * (size_t)n * n * n, sb = sizeof(float2) * nh * n * n;
  float* dr = nullptr;
  float2* ds = nullptr;
  float2* hs = (float2*)malloc(sb);
  cudaError_t e = cudaMalloc(&dr, rb);
  if (e == cudaSuccess) e = cudaMalloc(&ds, sb);
  if (e == cudaSuccess && hs) {
    if (forward) {
      e = cudaMemcpy(dr, in, rb, cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = mesh_r2c(&f, dr, ds, 0);
      if (e == cudaSuccess) e = cudaMemcpy(hs, ds, sb, cudaMemcpyDeviceToHost);
      // device layout [kz][kx][ky] -> host [kx][ky][kz]
      if (e == cudaSuccess)
        for (size_t k = 0; k < nh; k++)
          for (size_t i = 0; i < (size_t)n; i++)
            for (size_t j = 0; j < (size_t)n; j++) {
              const float2 v = hs[(k * n + i) * n + j];
              out[2 * ((i * n + j) * nh + k)] = v.x;
              out[2 * ((i * n + j) * nh + k) + 1] = v.y;
            }
    } else {
      for (size_t k = 0; k < nh; k++)
        for (size_t i = 0; i < (size_t)n; i++)
          for (size_t j = 0; j < (size_t)n; j++)
            hs[(k * n + i) * n + j] = make_float2(in[2 * ((i * n + j) * nh + k)],
                                                  in[2 * ((i * n + j) * nh + k) + 1]);
      e = cudaMemcpy(ds, hs, sb, cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = mesh_c2r(&f, ds, dr, 0);
      if (e == cudaSuccess) e = cudaMemcpy(out, dr, rb, cudaMemcpyDeviceToHost);
    }
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(dr);
  cudaFree(ds);
  free(hs);
  mesh_fft_free(&f);
  return cuda_err(e, "cg_fft");
}

// Device time of the plain 3-D transforms on device-resident data (no
// host copies, no layout conversion): the mean of `reps` launches each.
extern "C" int cg_fft_time(int n, int reps, float* ms_r2c, float* ms_c2r) {
  if (!pm_supported_mesh(n) || reps < 1) return set_err(CG_EINVAL, "cg_fft_time: bad arguments");
  MeshFFT f;
  CG_CHECK(mesh_fft_alloc(&f, n), "mesh_fft_alloc");
  const size_t nh = (size_t)(n / 2 + 1);
  float* dr = nullptr;
  float2* ds = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaMalloc(&dr, sizeof(float) * (size_t)n * n * n);
  if (e == cudaSuccess) e = cudaMalloc(&ds, sizeof(float2) * nh * n * n);
  if (e == cudaSuccess) e = cudaMemset(dr, 0, sizeof(float) * (size_t)n * n * n);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  float t_r2c = 0.0f, t_c2r = 0.0f;
  for (int pass = 0; pass < 2 && e == cudaSuccess; pass++) {
    const bool fwd = pass == 0;
    e = fwd ? mesh_r2c(&f, dr, ds, 0) : mesh_c2r(&f, ds, dr, 0);      // warm-up
    if (e == cudaSuccess) e = cudaEventRecord(a, 0);
    for (int r = 0; r < reps && e == cudaSuccess; r++)
      e = fwd ? mesh_r2c(&f, dr, ds, 0) : mesh_c2r(&f, ds, dr, 0);
    if (e == cudaSuccess) e = cudaEventRecord(b, 0);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    (fwd ? t_r2c : t_c2r) = ms / reps;
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(dr);
  cudaFree(ds);
  mesh_fft_free(&f);
  if (e != cudaSuccess) return cuda_err(e, "cg_fft_time");
  if (ms_r2c) *ms_r2c = t_r2c;
  if (ms_c2r) *ms_c2r = t_c2r;
  return CG_OK;
}

extern "C" int cg_fft_r2c(int n, const float* real_in, float* spec_out) {
  return host_fft(n, real_in, spec_out, true);
}
extern "C" int cg_fft_c2r(int n, const float* spec_in, float* real_out) {
  return host_fft(n, spec_in, real_out, false);
}

// ------------------------------------------------------ host coefficients
extern "C" double cg_growth_D1(double omega_m, double a) { return ColaTime(omega_m).D1(a); }
extern "C" double cg_growth_D2(double omega_m, double a) { return ColaTime(omega_m).D2(a); }
extern "C" double cg_cola_Sq(double omega_m, double ai, double af, double aref) {
  return ColaTime(omega_m).Sq(ai, af, aref);
}
extern "C" double cg_cola_Sphi(double omega_m, double ai, double af, double aref) {
  return ColaTime(omega_m).Sphi(ai, af, aref);
}
extern "C" void cg_kick_coeffs(double omega_m, float a_v, float a_x, float avel1, float out3[3]) {
  ColaTime(omega_m).kick(a_v, a_x, avel1, &out3[0], &out3[1], &out3[2]);
}
extern "C" void cg_drift_coeffs(double omega_m, float a_x, float a_v, float apos1,
                                float out3[3]) {
  ColaTime(omega_m).drift(a_x, a_v, apos1, &out3[0], &out3[1], &out3[2]);
}

// ===================================================================
// Drop-in layer: the reference's entry points over one process-wide
// realization (the reference keeps file-static state the same way,
// pm.c:45-71, lpt.c:26-39, cola.c:58).
// ===================================================================
namespace {
struct DropIn {
  int nc_pm = 0, factor = 0;
  float boxsize = 0;
  cg_sim* sim = nullptr;
  const Particles* bound = nullptr;
  const Particle* bound_p = nullptr;
  int bound_np = -1;
  bool full_sync = false;
  bool abort_on_error = true;
  const ParticleMinimum* snap_p = nullptr;   // host array of the last cola_set_snapshot
  int snap_np = -1;
  // cola_kick is queued and run fused with the cola_drift that follows it
  // (main.c:191-201 always calls them in that order); any other call runs
  // it first
  bool kick_pending = false;
  float kick_dda = 0, kick_q1 = 0, kick_q2 = 0;
  int lpt_nc = 0;
  PowerTable power;
  bool power_ready = false;
  double power_om = 0.3, power_ol = 0.7;
  std::map<float, std::unique_ptr<ColaTime>> times;
};
DropIn g_drop;

// msg_abort (msg.c:36-45): print and exit with the reference's code.
void dropin_fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  if (g_drop.abort_on_error) {
    fprintf(stderr, "%s\n", buf);
    fflush(stderr);
    exit(code);
  }
}

const ColaTime& times_for(float om) {
  auto it = g_drop.times.find(om);
  if (it == g_drop.times.end())
    it = g_drop.times.emplace(om, std::unique_ptr<ColaTime>(new ColaTime(om))).first;
  return *it->second;
}

// Make the device state of `p` current.  Returns false on failure.
// Run a queued cola_kick.  Returns false after reporting a failure.
bool flush_kick() {
  if (!g_drop.kick_pending) return true;
  g_drop.kick_pending = false;
  if (cg_sim_kick_coeffs(g_drop.sim, g_drop.kick_dda, g_drop.kick_q1, g_drop.kick_q2)) {
    dropin_fail(4001, "cola_kick: %s", cg_last_error());
    return false;
  }
  return true;
}

bool bind(const Particles* p, bool refresh, bool keep_kick = false) {
  if (!g_drop.nc_pm) {
    dropin_fail(4001, "pm_init has not been called");
    return false;
  }
  if (!keep_kick && !flush_kick()) return false;
  const int nc = g_drop.nc_pm / g_drop.factor;
  if (!g_drop.sim) {
    long long cap = p->np_allocated > p->np_local ? p->np_allocated : p->np_local;
    int rc = cg_sim_create(&g_drop.sim, nc, g_drop.nc_pm, g_drop.boxsize, 0.3, cap);
    if (rc) {
      dropin_fail(4001, "Unable to allocate device memory for particle mesh: %s",
                  cg_last_error());
      return false;
    }
  }
  if (refresh || g_drop.full_sync || p != g_drop.bound || p->p != g_drop.bound_p ||
      p->np_local != g_drop.bound_np) {
    if (p->np_local > g_drop.sim->ps.cap) {
      // grow: recreate with the larger capacity
      cg_sim_destroy(g_drop.sim);
      g_drop.sim = nullptr;
      int rc = cg_sim_create(&g_drop.sim, nc, g_drop.nc_pm, g_drop.boxsize, 0.3, p->np_local);
      if (rc) {
        dropin_fail(4001, "Unable to allocate device memory: %s", cg_last_error());
        return false;
      }
    }
    if (cg_sim_set_particles(g_drop.sim, p->p, p->np_local, p->a_x, p->a_v)) {
      dropin_fail(4002, "particle upload failed: %s", cg_last_error());
      return false;
    }
    g_drop.bound = p;
    g_drop.bound_p = p->p;
    g_drop.bound_np = p->np_local;
  }
  g_drop.sim->a_x = p->a_x;
  g_drop.sim->a_v = p->a_v;
  return true;
}

void full_sync_download(Particles* p, bool forces) {
  if (!g_drop.full_sync) return;
  cg_sim_get_particles(g_drop.sim, p->p);
  if (forces) cg_sim_get_forces(g_drop.sim, (float*)p->force);
}
}  // namespace

extern "C" void cg_dropin_set_sync(int full) { g_drop.full_sync = full != 0; }
extern "C" void cg_dropin_set_abort(int abort_on_error) { g_drop.abort_on_error = abort_on_error != 0; }

extern "C" void cg_dropin_finalize(void) {
  g_drop.kick_pending = false;
  cg_sim_destroy(g_drop.sim);
  g_drop.sim = nullptr;
  g_drop.bound = nullptr;
  g_drop.bound_p = nullptr;
  g_drop.bound_np = -1;
  g_drop.nc_pm = 0;
  g_drop.snap_p = nullptr;
  g_drop.snap_np = -1;
  lpt_dropin_release();
}

extern "C" void cg_snapshot_invalidate(void) {
  g_drop.snap_p = nullptr;
  g_drop.snap_np = -1;
}

extern "C" int cg_particles_upload(Particles* p) {
  if (!p) return set_err(CG_EINVAL, "cg_particles_upload: NULL");
  return bind(p, true) ? CG_OK : CG_EINVAL;
}

extern "C" int cg_particles_download(Particles* p) {
  if (!p) return set_err(CG_EINVAL, "cg_particles_download: NULL");
  if (!bind(p, false)) return CG_EINVAL;
  int rc = cg_sim_get_particles(g_drop.sim, p->p);
  if (!rc && p->force) rc = cg_sim_get_forces(g_drop.sim, (float*)p->force);
  return rc;
}

extern "C" void pm_init(const int nc_pm, const int nc_pm_factor, const float boxsize,
                        const float np_alloc_factor, void* const mem1, const size_t size1,
                        void* const mem2, const size_t size2) {
  (void)np_alloc_factor; (void)mem1; (void)size1; (void)mem2; (void)size2;
  if (!pm_supported_mesh(nc_pm) || nc_pm_factor <= 0 || nc_pm % nc_pm_factor) {
    dropin_fail(4001, "pm_init: unsupported mesh %d (factor %d)", nc_pm, nc_pm_factor);
    return;
  }
  if (g_drop.sim && (g_drop.nc_pm != nc_pm || g_drop.boxsize != boxsize)) {
    cg_sim_destroy(g_drop.sim);
    g_drop.sim = nullptr;
  }
  g_drop.nc_pm = nc_pm;
  g_drop.factor = nc_pm_factor;
  g_drop.boxsize = boxsize;
  g_drop.bound = nullptr;
}

extern "C" void move_particles2(Particles* const particles, const float BoxSize, void* const buf,
                                const size_t size) {
  (void)buf; (void)size;
  if (!bind(particles, false)) return;
  g_drop.sim->L = BoxSize;
  if (cg_sim_move(g_drop.sim)) dropin_fail(6030, "move_particles2: %s", cg_last_error());
  g_drop.sim->L = g_drop.boxsize;
  full_sync_download(particles, false);
}

extern "C" void pm_calculate_forces(Particles* particles) {
  if (!bind(particles, false)) return;
  double sum = 0.0;
  int rc = cg_sim_forces(g_drop.sim, &sum);
  if (rc) {
    dropin_fail(rc == CG_EPARTICLE ? 6040 : 4001, "pm_calculate_forces: %s", cg_last_error());
    return;
  }
  // check_total_density (pm.c:548-553)
  const long long ncp = g_drop.nc_pm / g_drop.factor;
  const double tol = 1.0e-7 * pow((double)g_drop.factor, 3) * (double)(ncp * ncp * ncp);
  if (fabs(sum) > tol) {
    dropin_fail(6040, "Error: total CIC density error is large: %le > %le\n", sum, tol);
    return;
  }
  full_sync_download(particles, true);
}

extern "C" void cola_kick(Particles* const particles, const float Omega_m, const float avel1) {
  if (!bind(particles, false)) return;
  const ColaTime& ct = times_for(Omega_m);
  float dda, q1, q2;
  ct.kick(particles->a_v, particles->a_x, avel1, &dda, &q1, &q2);
  // the kick's -1.5 Omega_m factor (cola.c:105) takes this call's Omega_m
  if (!g_drop.sim->ct || g_drop.sim->ct->om32 != Omega_m) {
    g_drop.sim->omega_m = Omega_m;
    g_drop.sim->ct.reset(new ColaTime(Omega_m));
  }
  if (g_drop.full_sync) {
    if (cg_sim_kick_coeffs(g_drop.sim, dda, q1, q2)) {
      dropin_fail(4001, "cola_kick: %s", cg_last_error());
      return;
    }
  } else {
    g_drop.kick_pending = true;
    g_drop.kick_dda = dda;
    g_drop.kick_q1 = q1;
    g_drop.kick_q2 = q2;
  }
  particles->a_v = avel1;          // cola.c:115
  g_drop.sim->a_v = avel1;
  full_sync_download(particles, false);
}

extern "C" void cola_drift(Particles* const particles, const float Omega_m, const float apos1) {
  // a kick queued for these particles runs fused with this drift
  const bool fuse = g_drop.kick_pending && particles == g_drop.bound &&
                    particles->p == g_drop.bound_p && particles->np_local == g_drop.bound_np;
  if (!bind(particles, false, fuse)) return;
  const ColaTime& ct = times_for(Omega_m);
  float dyyy, da1, da2;
  ct.drift(particles->a_x, particles->a_v, apos1, &dyyy, &da1, &da2);
  int rc;
  if (fuse && g_drop.kick_pending) {
    g_drop.kick_pending = false;
    rc = sim_kick_drift(g_drop.sim, g_drop.kick_dda, g_drop.kick_q1, g_drop.kick_q2, dyyy, da1,
                        da2);
  } else {
    rc = cg_sim_drift_coeffs(g_drop.sim, dyyy, da1, da2);
  }
  if (rc) {
    dropin_fail(4001, "cola_drift: %s", cg_last_error());
    return;
  }
  particles->a_x = apos1;          // cola.c:151
  g_drop.sim->a_x = apos1;
  full_sync_download(particles, false);
}

extern "C" void cola_set_snapshot(const double aout, Particles const* const particles,
                                  Snapshot* const snapshot) {
  if (!bind(particles, false)) return;
  if (snapshot->np_allocated < particles->np_local) {
    dropin_fail(4002, "cola_set_snapshot: snapshot holds %d < %d particles",
                snapshot->np_allocated, particles->np_local);
    return;
  }
  if (cg_sim_snapshot(g_drop.sim, aout, snapshot->omega_m, snapshot->p)) {
    dropin_fail(4001, "cola_set_snapshot: %s", cg_last_error());
    return;
  }
  snapshot->np_local = particles->np_local;          // cola.c:412-414
  snapshot->np_average = particles->np_average;
  snapshot->a = (float)aout;
  g_drop.snap_p = g_drop.full_sync ? nullptr : snapshot->p;
  g_drop.snap_np = snapshot->np_local;
}

extern "C" void set_noncola_initial(Particles const* const particles, Snapshot* const snapshot) {
  if (!bind(particles, false)) return;
  if (snapshot->np_allocated < particles->np_local) {
    dropin_fail(4002, "set_noncola_initial: snapshot holds %d < %d particles",
                snapshot->np_allocated, particles->np_local);
    return;
  }
  if (cg_sim_initial_snapshot(g_drop.sim, snapshot->omega_m, snapshot->p)) {
    dropin_fail(4001, "set_noncola_initial: %s", cg_last_error());
    return;
  }
  snapshot->np_local = particles->np_local;          // cola.c:333-336
  snapshot->np_total = particles->np_total;
  snapshot->np_average = particles->np_average;
  snapshot->a = particles->a_x;
  g_drop.snap_p = g_drop.full_sync ? nullptr : snapshot->p;
  g_drop.snap_np = snapshot->np_local;
}

// The device copy of `snapshot` left by the last cola_set_snapshot (the
// drop-in sim's ParticleMinimum staging array), while it still matches:
// same host array and count, not overwritten since, no full-sync mode.
ParticleMinimum* dropin_device_snapshot(const Snapshot* snapshot, cudaStream_t* st) {
  if (!snapshot || !g_drop.sim || g_drop.full_sync || !g_drop.sim->aos_snapshot ||
      g_drop.snap_p != snapshot->p || g_drop.snap_np != snapshot->np_local)
    return nullptr;
  if (st) *st = g_drop.sim->st;
  return (ParticleMinimum*)g_drop.sim->d_aos;
}

// ---------------------------------------------------------- power.c
extern "C" void power_init(const char filename[], const double a_init, const double sigma8,
                           const double omega_m, const double omega_lambda) {
  (void)a_init;
  char err[512];
  g_drop.power_om = omega_m;
  g_drop.power_ol = omega_lambda;
  if (!g_drop.power.read(filename, err, sizeof(err))) {
    g_drop.power_ready = false;
    dropin_fail(3000, "Error: %s", err);
    return;
  }
  g_drop.power.norm = 1.0;
  const double s8 = sqrt(g_drop.power.sigma2(8.0));        // power.c:103-118
  if (fabs(s8 - sigma8) / sigma8 > 0.05) {
    g_drop.power_ready = false;
    dropin_fail(3010, "Input sigma8 %f is far from target sigma8 %f\n", s8, sigma8);
    return;
  }
  g_drop.power_ready = true;
}

extern "C" double PowerSpec(const double k) {
  return g_drop.power_ready ? g_drop.power(k) : 0.0;
}

extern "C" double GrowthFactor(double astart, double aend) {
  return linear_growth(aend, g_drop.power_om, g_drop.power_ol) /
         linear_growth(astart, g_drop.power_om, g_drop.power_ol);
}

// ------------------------------------------------------------- lpt.c
extern "C" void lpt_init(const int nc, const void* mem, const size_t size) {
  (void)mem; (void)size;
  if (nc <= 0 || nc % 2) {
    dropin_fail(2003, "lpt_init: nc=%d must be even and positive", nc);
    return;
  }
  g_drop.lpt_nc = nc;
}

extern "C" int lpt_get_local_nx(void) { return g_drop.lpt_nc; }

extern "C" int lpt_set_displacement(const double InitTime, const double omega_m, const int Seed,
                                    const double Box, Particles* particles) {
  if (!g_drop.lpt_nc) {
    dropin_fail(2003, "lpt_init has not been called");
    return -1;
  }
  if (!g_drop.power_ready) {
    dropin_fail(3000, "power_init has not been called");
    return -1;
  }
  const int nc = g_drop.lpt_nc;
  const long long np = (long long)nc * nc * nc;
  if (particles->np_allocated < np) {
    dropin_fail(2003, "lpt_set_displacement: %d particles allocated, %lld needed",
                particles->np_allocated, np);
    return -1;
  }
  const double dplus = 1.0 / GrowthFactor(InitTime, 1.0);             // lpt.c:509
  int rc = lpt_generate(nc, Box, Seed, omega_m, InitTime, dplus, g_drop.power,
                        particles->p);
  if (rc) {
    dropin_fail(2003, "lpt_set_displacement: %s", cg_last_error());
    return -1;
  }
  particles->np_local = (int)np;                                     // lpt.c:573-575
  particles->a_x = (float)InitTime;
  particles->a_v = 0.0f;
  g_drop.bound = nullptr;            // next call uploads the new particles
  return 0;
}

int cg_set_error_from_lpt(int code, const char* msg) { return set_err(code, "%s", msg); }
// The drop-in failure path (msg_abort semantics) for drop-in entry points
// defined in other translation units.
void cg_dropin_error(int code, const char* msg) { dropin_fail(code, "%s", msg); }
