// Batched realizations in one graph launch.
//
// The reference produces many realizations by looping over seeds, one after
// another (main.c:117-209).  Here a batch of realizations -- each with its
// own box size, mesh, step count and initial particles -- is recorded once
// into a single CUDA graph: the realizations are spread over a few streams
// (longest total work first), each stream runs its realizations' complete
// time loops (the reference's control flow, main.c:162-206) back to back on
// one set of mesh buffers, and the streams fork from and join into one
// capture stream.  cg_batch_run launches that graph; relaunching it reruns
// the whole batch from the stored initial particles.  All time coefficients
// are computed in double on the host while the graph is recorded.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <memory>
#include <vector>

#include "../../include/colagpu.h"
#include "cosmo.h"
#include "internal.h"

extern int cg_set_error_from_lpt(int code, const char* msg);

namespace {

struct Real {
  cg_realization_spec spec;
  ParticleSoA ps{};
  float* soa = nullptr;
  long long* id_alloc = nullptr;  // the allocations behind ps.id / ps.orig (a sort
  int* orig_alloc = nullptr;      // exchanges ps's pointers with order's scratch)
  ParticleOrder order;            // cell-order sort scratch (sorting batches only)
  void* ics = nullptr;          // initial Particle[] (device)
  void* snap = nullptr;         // ParticleMinimum[] (device)
  double* dsum = nullptr;       // one density sum per force evaluation
  double* pk = nullptr;         // 3 * ngrid doubles of P(k) sums
  int nforce = 0;
  int stream = 0;
  bool loaded = false;
};

struct StreamBufs {
  cudaStream_t st = nullptr;
  PmPlan plan{};                // buffers for the largest mesh of this stream
};

}  // namespace

struct cg_batch {
  double omega_m = 0;
  int sort_every = 0;              // cell-order sort at every sort_every-th move
  std::unique_ptr<ColaTime> ct;
  std::vector<Real> reals;
  std::vector<StreamBufs> streams;
  std::map<int, MeshFFT> tables;   // twiddle tables per mesh size
  cudaStream_t main = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<cudaEvent_t> events;
  cudaEvent_t t0 = nullptr, t1 = nullptr;   // timing of the last graph launch
  float last_ms = 0.0f;
};

namespace {

int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s%s%s", what, e != cudaSuccess ? ": " : "",
           e != cudaSuccess ? cudaGetErrorString(e) : "");
  return cg_set_error_from_lpt(code, buf);
}

// A per-realization view of a stream's mesh buffers: this realization's mesh
// size and box constants (the same float expressions as pm_plan_alloc).
PmPlan view(const PmPlan& bufs, const MeshFFT& tab, int N, int factor, float L) {
  PmPlan p = bufs;
  p.N = N;
  p.factor = factor;
  p.L = L;
  p.scale = (float)N / L;
  p.wpar = (float)pow((double)factor, 3.0);
  const float sc = (float)(2.0 * 3.1415926535897932384626433832795 / (double)L);
  p.f1 = (float)(-1.0 / pow((double)N, 3.0) / (double)sc);
  const float eps = L / (float)N;
  p.x_right = L / (float)N * (float)N - eps;
  p.shiftx = -L;
  p.twN = tab.twN;
  p.twH = tab.twH;
  p.mesh_bytes = sizeof(float) * (size_t)N * N * N;
  p.spec_bytes = sizeof(float2) * (size_t)(N / 2 + 1) * N * N;
  if (N != bufs.N) {
    // the stream's TMA maps describe its largest mesh, not this one
    p.ztm_ok = false;
    p.zsw_ok = false;
    p.xsw_ok = false;
  }
  // the realization's first deposit fills the shared buffer (dens_reset
  // false); from then on each z r2c leaves -1 behind for the next one
  p.keep_dens = false;
  p.dens_reset = false;
  return p;
}

// One realization's full time loop queued on stream st (main.c:162-206 with
// the general linear schedule: apos(i) = a_init + (i-1) da).
cudaError_t record_realization(cg_batch* b, Real& r, StreamBufs& sb) {
  const cg_realization_spec& sp = r.spec;
  cudaStream_t st = sb.st;
  PmPlan p = view(sb.plan, b->tables[sp.ngrid], sp.ngrid, sp.ngrid / sp.nc, sp.boxsize);
  cudaError_t e = particles_aos_to_soa(r.ics, &r.ps, st);
  if (e != cudaSuccess) return e;
  const double da = (sp.a_final - sp.a_init) / sp.nsteps;
  const int nloop = sp.nsteps + 1;
  float a_x = (float)sp.a_init, a_v = (float)sp.a_init;
  const float aout = sp.aout;
  bool written = false;
  // the particles' working arrays; a cell-order sort exchanges them
  const float* cx[3] = {r.ps.x[0], r.ps.x[1], r.ps.x[2]};
  const float* cv[3] = {r.ps.v[0], r.ps.v[1], r.ps.v[2]};
  const float* cf[3] = {r.ps.f[0], r.ps.f[1], r.ps.f[2]};
  const float* c1[3] = {r.ps.dx1[0], r.ps.dx1[1], r.ps.dx1[2]};
  const float* c2[3] = {r.ps.dx2[0], r.ps.dx2[1], r.ps.dx2[2]};
  int iforce = 0;
  for (int istep = 1; istep <= nloop && !written; istep++) {
    const double avel0 = sp.a_init + (istep - 1.5) * da;
    const double apos0 = sp.a_init + (istep - 1.0) * da;
    const double avel1 = sp.a_init + (istep - 0.5) * da;
    const double apos1 = sp.a_init + istep * da;
    if ((e = dev_wrap(r.ps.x, r.ps.n, sp.boxsize, st)) != cudaSuccess) return e;
    if (b->sort_every > 0 && istep % b->sort_every == 0) {
      // cell order, as cg_sim_move sorts (the pointers the captured kernels
      // get follow the exchange, so every relaunch repeats it)
      if ((e = particles_sort_cells(&r.ps, &r.order, sp.boxsize, st)) != cudaSuccess) return e;
      for (int a = 0; a < 3; a++) {
        cx[a] = r.ps.x[a];
        cv[a] = r.ps.v[a];
        cf[a] = r.ps.f[a];
        c1[a] = r.ps.dx1[a];
        c2[a] = r.ps.dx2[a];
      }
    }
    p.dsum = r.dsum + iforce++;
    if ((e = pm_forces(&p, cx, r.ps.n, r.ps.f, st)) != cudaSuccess) return e;
    auto snapshot = [&]() -> cudaError_t {
      const float vfac = (float)(100.0 / (double)aout);
      float dda, q1, q2, dyyy, da1, da2;
      b->ct->kick(a_v, a_x, aout, &dda, &q1, &q2);
      b->ct->drift(a_x, a_v, aout, &dyyy, &da1, &da2);
      const float Dv = (float)b->ct->DprimeQ((double)aout, 1.0);
      const float Dv2 = (float)b->ct->D2v((double)aout);
      written = true;
      return dev_snapshot(cx, cv, cf, c1, c2, r.ps.n, b->ct->om32, dda, q1, q2, Dv, Dv2, dyyy,
                          da1, da2, vfac, r.ps.id, r.ps.orig, r.snap, st);
    };
    if (avel0 <= aout && aout <= apos0) {
      if ((e = snapshot()) != cudaSuccess) return e;
      break;
    }
    float dda, q1, q2;
    b->ct->kick(a_v, a_x, (float)avel1, &dda, &q1, &q2);
    if (apos0 < aout && aout <= avel1) {
      // the output falls between the kick and the drift
      if ((e = dev_kick(r.ps.v, cf, c1, c2, r.ps.n, b->ct->om32, dda, q1, q2, st)) != cudaSuccess)
        return e;
      a_v = (float)avel1;
      if ((e = snapshot()) != cudaSuccess) return e;
      break;
    }
    // kick, then drift with the kicked velocity, in one pass (bit-identical
    // to the two kernels, as cg_sim_kick_drift)
    a_v = (float)avel1;
    float dyyy, da1, da2;
    b->ct->drift(a_x, a_v, (float)apos1, &dyyy, &da1, &da2);
    if ((e = dev_kick_drift(r.ps.x, r.ps.v, cf, c1, c2, r.ps.n, b->ct->om32, dda, q1, q2, dyyy,
                            da1, da2, st)) != cudaSuccess)
      return e;
    a_x = (float)apos1;
  }
  r.nforce = iforce;
  // power spectrum of the final positions (the P(k) the batch is measured by);
  // its density sum goes to the spare slot after the force evaluations
  p.dsum = r.dsum + sp.nsteps + 1;
  return pm_power_spectrum(&p, cx, r.ps.n, sp.ngrid / 2, 0, r.pk, st);
}

void free_batch(cg_batch* b) {
  if (!b) return;
  if (b->main) cudaStreamSynchronize(b->main);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto& r : b->reals) {
    cudaFree(r.soa);
    cudaFree(r.id_alloc);
    cudaFree(r.orig_alloc);
    particle_order_free(&r.order);
    cudaFree(r.ics);
    cudaFree(r.snap);
    cudaFree(r.dsum);
    cudaFree(r.pk);
  }
  for (auto& s : b->streams) {
    pm_plan_free(&s.plan);
    if (s.st) cudaStreamDestroy(s.st);
  }
  for (auto& t : b->tables) mesh_fft_free(&t.second);
  for (auto e : b->events) cudaEventDestroy(e);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->t1) cudaEventDestroy(b->t1);
  if (b->main) cudaStreamDestroy(b->main);
  delete b;
}

}  // namespace

extern "C" int cg_batch_create(cg_batch** out, int nreal, const cg_realization_spec* specs,
                               double omega_m, int nstreams) {
  if (!out || nreal < 1 || !specs || nstreams < 1)
    return fail(CG_EINVAL, "cg_batch_create: bad arguments");
  *out = nullptr;
  for (int i = 0; i < nreal; i++) {
    const cg_realization_spec& s = specs[i];
    if (s.nc <= 0 || s.ngrid % s.nc || !pm_supported_mesh(s.ngrid) || !(s.boxsize > 0) ||
        s.nsteps < 1 || !(s.a_final > s.a_init) || !(s.a_init > 0))
      return fail(CG_EINVAL, "cg_batch_create: bad realization spec");
  }
  cg_batch* b = new cg_batch();
  b->omega_m = omega_m;
  // the cell-order sort policy of cg_sim: every sixth move from 2^23
  // particles per realization (COLAGPU_SORT_EVERY overrides)
  long long npmax = 0;
  for (int i = 0; i < nreal; i++)
    npmax = std::max(npmax, (long long)specs[i].nc * specs[i].nc * specs[i].nc);
  b->sort_every = npmax >= (1LL << 23) ? 6 : 0;
  if (const char* ev = getenv("COLAGPU_SORT_EVERY")) b->sort_every = atoi(ev) > 0 ? atoi(ev) : 0;
  b->ct.reset(new ColaTime(omega_m));
  b->reals.resize(nreal);
  if (nstreams > nreal) nstreams = nreal;
  b->streams.resize(nstreams);
  cudaError_t e = cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking);
  // assign realizations to streams: longest (np * forces) first, least loaded
  std::vector<int> order(nreal);
  for (int i = 0; i < nreal; i++) order[i] = i;
  auto work = [&](int i) {
    return (double)specs[i].ngrid * specs[i].ngrid * specs[i].ngrid * (specs[i].nsteps + 1);
  };
  std::sort(order.begin(), order.end(), [&](int a, int c) { return work(a) > work(c); });
  std::vector<double> load(nstreams, 0.0);
  std::vector<int> maxN(nstreams, 0);
  for (int i : order) {
    const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[s] += work(i);
    b->reals[i].stream = s;
    maxN[s] = std::max(maxN[s], specs[i].ngrid);
  }
  for (int s = 0; s < nstreams && e == cudaSuccess; s++) {
    e = cudaStreamCreateWithFlags(&b->streams[s].st, cudaStreamNonBlocking);
    if (e == cudaSuccess && maxN[s] > 0) e = pm_plan_alloc(&b->streams[s].plan, maxN[s], 1, 1.0f);
  }
  for (int i = 0; i < nreal && e == cudaSuccess; i++) {
    Real& r = b->reals[i];
    r.spec = specs[i];
    const int N = r.spec.ngrid;
    if (!b->tables.count(N)) {
      MeshFFT t;
      e = mesh_fft_alloc(&t, N);
      if (e != cudaSuccess) break;
      b->tables[N] = t;
    }
    const long long np = (long long)r.spec.nc * r.spec.nc * r.spec.nc;
    r.ps.n = np;
    r.ps.cap = np;
    e = cudaMalloc(&r.soa, sizeof(float) * 15 * (size_t)np);
    if (e == cudaSuccess) e = cudaMalloc(&r.id_alloc, sizeof(long long) * (size_t)np);
    if (e == cudaSuccess) e = cudaMalloc(&r.orig_alloc, sizeof(int) * (size_t)np);
    r.ps.id = r.id_alloc;
    r.ps.orig = r.orig_alloc;
    if (e == cudaSuccess) e = cudaMalloc(&r.ics, 56 * (size_t)np);
    if (e == cudaSuccess) e = cudaMalloc(&r.snap, 32 * (size_t)np);
    if (e == cudaSuccess) e = cudaMalloc(&r.dsum, sizeof(double) * (r.spec.nsteps + 2));
    if (e == cudaSuccess) e = cudaMalloc(&r.pk, sizeof(double) * 3 * N);
    if (e != cudaSuccess) break;
    for (int a = 0; a < 3; a++) {
      r.ps.x[a] = r.soa + (0 + a) * (size_t)np;
      r.ps.v[a] = r.soa + (3 + a) * (size_t)np;
      r.ps.dx1[a] = r.soa + (6 + a) * (size_t)np;
      r.ps.dx2[a] = r.soa + (9 + a) * (size_t)np;
      r.ps.f[a] = r.soa + (12 + a) * (size_t)np;
    }
    e = cudaMemset(r.soa, 0, sizeof(float) * 15 * (size_t)np);
  }
  if (e != cudaSuccess) {
    int rc = fail(e == cudaErrorMemoryAllocation ? CG_ENOMEM : CG_ECUDA, "cg_batch_create", e);
    free_batch(b);
    return rc;
  }
  *out = b;
  return CG_OK;
}

extern "C" void cg_batch_destroy(cg_batch* b) { free_batch(b); }

extern "C" int cg_batch_set_particles(cg_batch* b, int i, const void* particles, long long np) {
  if (!b || i < 0 || i >= (int)b->reals.size() || !particles)
    return fail(CG_EINVAL, "cg_batch_set_particles: bad arguments");
  Real& r = b->reals[i];
  if (np != r.ps.n) return fail(CG_EINVAL, "cg_batch_set_particles: np must be nc^3");
  cudaError_t e = cudaMemcpy(r.ics, particles, 56 * (size_t)np, cudaMemcpyDefault);
  if (e != cudaSuccess) return fail(CG_ECUDA, "cg_batch_set_particles", e);
  r.loaded = true;
  return CG_OK;
}

extern "C" int cg_batch_set_sort_interval(cg_batch* b, int every) {
  if (!b || every < 0) return fail(CG_EINVAL, "cg_batch_set_sort_interval: bad arguments");
  if (b->exec) return fail(CG_EINVAL, "cg_batch_set_sort_interval: the batch is recorded already");
  b->sort_every = every;
  return CG_OK;
}

extern "C" int cg_batch_run(cg_batch* b) {
  if (!b) return fail(CG_EINVAL, "cg_batch_run: NULL");
  for (auto& r : b->reals)
    if (!r.loaded) return fail(CG_EINVAL, "cg_batch_run: a realization has no particles");
  cudaError_t e = cudaSuccess;
  if (!b->exec) {
    // the sort's scratch, allocated before the capture (which allocates nothing)
    for (auto& r : b->reals)
      if (b->sort_every > 0 && (e = particle_order_reserve(&r.order, r.ps.cap)) != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? CG_ENOMEM : CG_ECUDA,
                    "cg_batch_run: sort scratch", e);
    // the column bins of the force step's deposit and interpolation, per
    // stream for its largest realization (the views of the stream's plan
    // share them)
    for (auto& r : b->reals)
      if ((pm_force_deposit_binned() || pm_force_interp_binned()) &&
          (e = pm_colbins_reserve(&b->streams[r.stream].plan, r.ps.cap)) != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? CG_ENOMEM : CG_ECUDA,
                    "cg_batch_run: column bins", e);
    const int ns = (int)b->streams.size();
    b->events.resize(ns + 1);
    for (auto& ev : b->events)
      if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
        return fail(CG_ECUDA, "cg_batch_run: event", e);
    e = cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(CG_ECUDA, "cg_batch_run: begin capture", e);
    cudaEventRecord(b->events[ns], b->main);
    for (int s = 0; s < ns; s++) cudaStreamWaitEvent(b->streams[s].st, b->events[ns], 0);
    for (auto& r : b->reals) {
      e = record_realization(b, r, b->streams[r.stream]);
      if (e != cudaSuccess) break;
    }
    for (int s = 0; s < ns; s++) {
      cudaEventRecord(b->events[s], b->streams[s].st);
      cudaStreamWaitEvent(b->main, b->events[s], 0);
    }
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(b->main, &g);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(CG_ECUDA, "cg_batch_run: capture", e);
    }
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) return fail(CG_ECUDA, "cg_batch_run: instantiate", e);
  }
  if (!b->t0) {
    if ((e = cudaEventCreate(&b->t0)) != cudaSuccess || (e = cudaEventCreate(&b->t1)) != cudaSuccess)
      return fail(CG_ECUDA, "cg_batch_run: event", e);
  }
  prof_mark(b->main, CG_ST_OTHER);
  cudaEventRecord(b->t0, b->main);
  e = cudaGraphLaunch(b->exec, b->main);
  if (e == cudaSuccess) e = cudaEventRecord(b->t1, b->main);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->main);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&b->last_ms, b->t0, b->t1);
  if (e != cudaSuccess) return fail(CG_ECUDA, "cg_batch_run: launch", e);
  // density checks of every force evaluation (pm.c:548-553)
  for (auto& r : b->reals) {
    std::vector<double> d(r.nforce);
    e = cudaMemcpy(d.data(), r.dsum, sizeof(double) * r.nforce, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(CG_ECUDA, "cg_batch_run: density sums", e);
    const double f = (double)(r.spec.ngrid / r.spec.nc);
    const double tol = 1.0e-7 * f * f * f * (double)r.ps.n;
    for (double v : d)
      if (fabs(v) > tol) return fail(CG_EDENSITY, "cg_batch_run: CIC density sum check failed");
  }
  return CG_OK;
}

extern "C" int cg_batch_get_snapshot(cg_batch* b, int i, void* pmin_out) {
  if (!b || i < 0 || i >= (int)b->reals.size() || !pmin_out)
    return fail(CG_EINVAL, "cg_batch_get_snapshot: bad arguments");
  Real& r = b->reals[i];
  cudaError_t e = cudaMemcpy(pmin_out, r.snap, 32 * (size_t)r.ps.n, cudaMemcpyDefault);
  return e == cudaSuccess ? CG_OK : fail(CG_ECUDA, "cg_batch_get_snapshot", e);
}

extern "C" int cg_batch_power_spectrum(cg_batch* b, int i, double* k, double* pk,
                                       double* nmodes) {
  if (!b || i < 0 || i >= (int)b->reals.size() || !k || !pk)
    return fail(CG_EINVAL, "cg_batch_power_spectrum: bad arguments");
  Real& r = b->reals[i];
  const int nb = r.spec.ngrid / 2;
  std::vector<double> h(3 * (size_t)nb);
  cudaError_t e = cudaMemcpy(h.data(), r.pk, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(CG_ECUDA, "cg_batch_power_spectrum", e);
  const double N = r.spec.ngrid, L = r.spec.boxsize;
  const double kf = 2.0 * M_PI / L, norm = L * L * L / (N * N * N * N * N * N);
  for (int j = 0; j < nb; j++) {
    const double w = h[j];
    k[j] = w > 0 ? kf * h[nb + j] / w : 0.0;
    pk[j] = w > 0 ? norm * h[2 * nb + j] / w : 0.0;
    if (nmodes) nmodes[j] = w;
  }
  return CG_OK;
}

extern "C" int cg_batch_num_nodes(cg_batch* b, size_t* nodes) {
  if (!b || !b->graph || !nodes) return fail(CG_EINVAL, "cg_batch_num_nodes: not recorded");
  cudaError_t e = cudaGraphGetNodes(b->graph, nullptr, nodes);
  return e == cudaSuccess ? CG_OK : fail(CG_ECUDA, "cg_batch_num_nodes", e);
}

extern "C" int cg_batch_last_ms(cg_batch* b, float* ms) {
  if (!b || !ms) return fail(CG_EINVAL, "cg_batch_last_ms: NULL");
  *ms = b->last_ms;
  return CG_OK;
}
