// Internal declarations shared by the CUDA translation units of libcolagpu.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#define CG_THREADS 256

// Stages of the step, for launch accounting and event timing (prof.cu).
enum {
  CG_ST_FILL = 0, CG_ST_DEPOSIT, CG_ST_FZ, CG_ST_FX_FWD, CG_ST_GREEN, CG_ST_FX_INV,
  CG_ST_ZI, CG_ST_INTERP, CG_ST_WRAP, CG_ST_KICK, CG_ST_DRIFT, CG_ST_SNAPSHOT, CG_ST_LPT,
  CG_ST_OTHER, CG_ST_KICK_DRIFT, CG_ST_SORT, CG_ST_COUNT
};
// Call before every kernel launch: counts it and, while a profile is open,
// records a CUDA event on the launch stream.
void prof_mark(cudaStream_t st, int stage);

// Streaming multiprocessors of the current device (queried once per device).
int cg_sm_count();
// Grid of a grid-stride kernel of CG_THREADS threads over n items: one CTA
// per CG_THREADS items, at most per_sm CTAs for every SM of the device.
int cg_grid(long long n, int per_sm);
inline int grid_for(long long n) { return cg_grid(n, 16); }

// Device error word bits (set by kernels, read by the host after a step).
enum {
  CG_ERR_BAD_CELL = 1,      // a particle's y or z cell index was negative
  CG_ERR_NONFINITE = 2,     // a particle position was NaN or infinite
  CG_ERR_TMA_WAIT = 4,      // a TMA gather of the z transform did not complete
};

// Mesh transform plan: every buffer of one PM mesh size.
struct PmPlan {
  int N;                    // mesh cells per dimension
  int factor;               // PM factor (mesh/particle per dimension)
  float L;                  // box size
  float scale;              // (float)N / (float)L                 pm.c:215
  float wpar;               // factor^3                            pm.c:216
  float f1;                 // -1/N^3/(2 pi/L) as float            pm.c:315-317
  float x_right;            // buffer-particle threshold           pm.c:422-423
  float shiftx;             // -L                                  pm.c:434
  float* dens;              // real mesh [x][y][z], N^3
  float2* spec;             // half spectrum [kz][kx][ky], (N/2+1) N N
  float2* gsp[3];           // force spectra, same layout
  float* fmesh[3];          // real force meshes [x][y][z]
  float2* twN;              // exp(-2 pi i k/N), k < N
  float2* twH;              // exp(-2 pi i k/(N/2)), k < N/2
  double* dsum;             // device: sum of the density mesh (check)
  double* pk_acc;           // device: 3 N doubles of power-spectrum bin sums
  unsigned* err;            // device: error word
  size_t mesh_bytes;        // bytes of one real mesh
  size_t spec_bytes;        // bytes of one half spectrum
  float* kfilt;             // device: force transfer functions, kfilt_sets x kfilt_n knots
  size_t kfilt_cap;         //   floats allocated
  int kfilt_n;              //   knots per function
  int kfilt_sets;           //   functions held
  int kfilt_cur;            //   the one the Green step applies; -1 = none
  float kfilt_inv_dn;       //   knots per unit of |n|
  float* ktab;              // device: gradient | Laplacian | window tables (N each), or
                            //   NULL for the reference's spectral kernel
  bool keep_dens;           // the density must survive the force step (else the z r2c
                            //   resets it to -1 for the next deposit)
  bool dens_reset;          // dens holds -1 everywhere, not the last density
  CUtensorMap ztm[3];       // TMA maps of gsp[0..2] for the z transform's gather
  bool ztm_ok;              //   valid, landing-area form k_zi_tma
  bool zsw_ok;              //   valid, swizzled-tile form k_zi_sw (else, with neither,
                            //   the cp.async gather runs)
  CUtensorMap xtm[3];       // TMA maps of spec, gsp[1], gsp[2] for the x pass's gather
  bool xsw_ok;              //   valid (else the x pass loads directly)
  int xtm_tk;               //   the columns per CTA the maps were encoded for
  bool dens_stale;          // dens does not hold the last force step's density (the
                            //   column-binned deposit built it in shared memory only)
  // Column bins of the force step's clouds (pm_colbins_reserve): per key
  // (lower-corner column) a count, then its start; per particle the rank of
  // its cloud and of its buffer copy; one 16-byte entry per cloud.
  long long cb_cap;         //   particles the rank / entry arrays hold
  long long cb_keys;        //   keys the count array holds (+1 for the total)
  unsigned* cb_cnt;
  unsigned* cb_bsum;        //   prefix-sum scratch
  unsigned* cb_rank;        //   2 cb_cap
  float4* cb_ent;           //   2 cb_cap
  float* cb_part;           //   interpolation partials: 6 x 2 cb_cap (slots i0 / i1 of
                            //   the x, y, z components)
  bool fmesh_stale;         // fmesh does not hold the last force step's force meshes (the
                            //   interpolation read them from shared memory only)
};

// Plain 3-D real transforms on the mesh layouts above (unnormalised, FFTW
// sign and c2r conventions).  mesh_c2r overwrites its input spectrum.
struct MeshFFT {
  int N;
  float2* twN;
  float2* twH;
  double* dsum;             // scratch: receives the sum of the r2c input
};
cudaError_t mesh_fft_alloc(MeshFFT* f, int N);
void mesh_fft_free(MeshFFT* f);
cudaError_t mesh_r2c(const MeshFFT* f, const float* real, float2* spec, cudaStream_t st);
cudaError_t mesh_c2r(const MeshFFT* f, float2* spec, float* real, cudaStream_t st);

// Schedule of the FFT passes of one mesh size: which compiled variant of the
// strided x pass and of the fused Green pass runs (pm_kernels.cu kFxCfg,
// kGreenCfg).  Variants other than 0 exist from 256 up (Green: up to 768).
#define PM_NUM_FX_VARIANTS 3
#define PM_NUM_GREEN_VARIANTS 7
#define PM_NUM_DEP_VARIANTS 6
struct MeshSched {
  int green = 0;
  int fx = 0;
  int dep = 0;   // deposit shape (pm_kernels.cu kDepCfg)
};

// pm_kernels.cu
bool pm_supported_mesh(int N);
// Gather of the z c2r for plans created afterwards: -1 by mesh size, 0
// cp.async, 1 TMA landing area, 2 TMA swizzled tile.  -1 on a bad mode.
int pm_set_z_gather(int mode);
// Gather of the x pass for plans created afterwards: -1 default, 0 direct
// loads, 1 TMA into a swizzled tile.  -1 on a bad mode.
int pm_set_x_gather(int mode);
// Number of schedule variants compiled for mesh size N (1 below 256).
int pm_num_variants(int N, int* n_green, int* n_fx);
MeshSched pm_get_schedule(int N);
void pm_set_schedule(int N, MeshSched s);
// Time every Green and x-pass variant of the plan's mesh size on its own
// buffers (their contents are overwritten) and return the fastest of each;
// ms_green / ms_fx receive the best time of each variant (may be NULL).
// Does not install the result.
cudaError_t pm_autotune(PmPlan* p, cudaStream_t st, MeshSched* best, float* ms_green,
                        float* ms_fx);
cudaError_t pm_plan_alloc(PmPlan* p, int N, int factor, float L);
// Force transfer functions T(|n|) for the Green step: nsets functions of n
// knots each at |n| = j (sqrt(3) N / 2) / (n - 1), copied from a host array
// (synchronous); set 0 becomes current.  n = 0 removes them.
cudaError_t pm_set_filters(PmPlan* p, const float* knots, int n, int nsets);
// Make set `set` current (-1: none, the reference's force).  False when the
// plan holds no such set.
bool pm_use_filter(PmPlan* p, int set);
// Force kernel of the Green step: gradient 0 spectral (the reference), 2 or
// 4 the 2- or 4-point central difference; laplacian 0 exact |n|^2 (the
// reference), 1 the 7-point discrete Laplacian; deconvolve 0, 1 or 2 times
// the CIC window.  All 0: the reference's kernel, no tables.
cudaError_t pm_set_force_kernel(PmPlan* p, int gradient, int laplacian, int deconvolve);
void pm_plan_free(PmPlan* p);
// Full PM force: deposit -> r2c -> Green/gradient -> 3 c2r -> interpolation.
// Positions and forces are SoA device arrays of n floats per component.
// With the column-binned deposit selected (pm_set_force_deposit(1)) and a
// plan that does not keep its density (keep_dens), the deposit and the r2c
// along z run as k_dfz, which needs the plan's column bins for n particles
// (allocated here on first use; pm_colbins_reserve beforehand for a stream
// capture).
cudaError_t pm_forces(PmPlan* p, const float* const x[3], long long n,
                      float* const f[3], cudaStream_t st);
// Deposit of the force step for the plans' next pm_forces calls: 0 (the
// default) the mesh deposit + k_fz, 1 column bins + k_dfz.  -1 on a bad mode.
int pm_set_force_deposit(int mode);
// The column-binned deposit is selected.
bool pm_force_deposit_binned();
// Interpolation of the force step for the plans' next pm_forces calls: 0
// (the default) from the force meshes (k_zi + k_interp), 1 from the z c2r's
// shared tiles through the column bins (k_zi_interp).  The forces are the
// same bit for bit.  -1 on a bad mode.
int pm_set_force_interp(int mode);
// The interpolation from the column bins is selected.
bool pm_force_interp_binned();
// The force mesh of component a (0..2) of the last force step in fmesh[a]
// (a z c2r of its spectrum when the interpolation did not write it).
cudaError_t pm_force_mesh(PmPlan* p, int a, cudaStream_t st);
// Column bins for up to n particles on the plan's mesh (no-op when held).
cudaError_t pm_colbins_reserve(PmPlan* p, long long n);
// Slab decomposition of the force over ranks (pm_kernels.cu): the density
// and r2c along z of planes [x0, x0+nx) from the rank's particles and the
// buffer copies it received (bx, nb: SoA device positions); the x, Green
// and inverse x passes of kz planes [kz0, kz0+nkz); the three z c2r of
// planes [x0, x0+nx); the interpolation of the rank's particles and buffer
// copies from its own planes.  The spectra move between the x and the kz
// slabs in between (the caller's exchange).
cudaError_t pm_slab_density(PmPlan* p, int x0, int nx, const float* const x[3], long long n,
                            const float* const bx[3], long long nb, cudaStream_t st);
cudaError_t pm_slab_kspace(PmPlan* p, int kz0, int nkz, cudaStream_t st);
cudaError_t pm_slab_c2r(PmPlan* p, int x0, int nx, cudaStream_t st);
cudaError_t pm_slab_interp(PmPlan* p, int x0, int nx, const float* const x[3], long long n,
                           float* const f[3], const float* const bx[3], long long nb,
                           float* const bf[3], cudaStream_t st);
// Individual stages (exposed for tests and timing).
cudaError_t pm_deposit(PmPlan* p, const float* const x[3], long long n, cudaStream_t st);
// Time every deposit variant on these positions (best of 3, each after a
// fill) and return the fastest in *best, the times in ms[PM_NUM_DEP_VARIANTS]
// (may be NULL).  Does not install it; leaves a deposit in the mesh.
cudaError_t pm_tune_deposit(PmPlan* p, const float* const x[3], long long n, cudaStream_t st,
                            int* best, float* ms);
// dens -> spec transformed along z and x (+ density sum into dsum)
cudaError_t pm_r2c(PmPlan* p, cudaStream_t st);
// spec -> y transform, Green/gradient -> three force meshes fmesh[a]
cudaError_t pm_green_c2r(PmPlan* p, cudaStream_t st);
// Power spectrum of the CIC density of x: deposit, r2c, shell sums into
// acc[3 * nbins] (device doubles: sum w, sum w |n|, sum w |delta_k|^2).
cudaError_t pm_power_spectrum(PmPlan* p, const float* const x[3], long long n, int nbins,
                              int deconv, double* acc, cudaStream_t st);
cudaError_t pm_interp(PmPlan* p, const float* const x[3], long long n,
                      float* const f[3], cudaStream_t st);

// Particle state on the device, structure of arrays (one array per
// component).  The arrays may be kept in an order of their own (cell
// order, reorder.cu); orig[i] is then the caller's index of particle i, and
// everything handed back to the caller is put in the caller's order by it.
// orig == NULL means the caller's order.
struct ParticleSoA {
  long long n;              // particles held
  long long cap;            // capacity
  float* x[3];
  float* v[3];
  float* dx1[3];
  float* dx2[3];
  float* f[3];
  long long* id;
  int* orig;
};

// cola_kernels.cu
cudaError_t dev_wrap(float* const x[3], long long n, float L, cudaStream_t st);
cudaError_t dev_kick(float* const v[3], const float* const f[3],
                      const float* const dx1[3], const float* const dx2[3],
                      long long n, float omega_m, float dda, float q1, float q2,
                      cudaStream_t st);
cudaError_t dev_drift(float* const x[3], const float* const v[3],
                       const float* const dx1[3], const float* const dx2[3],
                       long long n, float dyyy, float da1, float da2, cudaStream_t st);
// dev_kick then dev_drift (with the kicked velocity) in one kernel.
cudaError_t dev_kick_drift(float* const x[3], float* const v[3], const float* const f[3],
                           const float* const dx1[3], const float* const dx2[3], long long n,
                           float omega_m, float dda, float q1, float q2, float dyyy, float da1,
                           float da2, cudaStream_t st);
cudaError_t dev_snapshot(const float* const x[3], const float* const v[3],
                          const float* const f[3], const float* const dx1[3],
                          const float* const dx2[3], long long n,
                          float omega_m, float dda, float q1, float q2,
                          float Dv, float Dv2, float dyyy, float da1, float da2,
                          float vfac, const long long* id, const int* orig, void* out_aos,
                          cudaStream_t st);
// set_noncola_initial (cola.c:297-338): ParticleMinimum of the positions and
// the 2LPT velocities vfac (dx1 Dv + dx2 Dv2), in the caller's order.
cudaError_t dev_initial_snapshot(const ParticleSoA* s, float vfac, float Dv, float Dv2,
                                 void* out_aos, cudaStream_t st);
// AoS (reference Particle, 56 B) <-> SoA conversion on the device.  The
// upload resets orig to the caller's order; the download writes particle i
// at orig[i].
cudaError_t particles_aos_to_soa(const void* aos, ParticleSoA* s, cudaStream_t st);
cudaError_t particles_soa_to_aos(void* aos, const ParticleSoA* s, cudaStream_t st);

// reorder.cu: cell order of the particles.  Particles are sorted by the
// cell of a grid of about eight particles per cell (x slowest, z fastest), so
// that consecutive threads of the deposit and the interpolation touch
// neighbouring mesh cells.  A counting sort: bin counts (each particle's
// rank in its bin from the same atomic), a prefix sum, and one scatter of x, v, dx1, dx2, f, id and orig into a second set of
// arrays, which then becomes the working set.
struct ParticleOrder {
  long long cap = 0;        // particles the arrays hold
  long long nbins = 0;      // bins the counts hold
  float* alloc = nullptr;   // owned: 15 floats per particle
  long long* alloc_id = nullptr;
  int* alloc_orig = nullptr;
  // the scratch set (a sort writes here, then exchanges it with the
  // particles' working set, so these point into either allocation)
  float* x[3] = {nullptr, nullptr, nullptr};
  float* v[3] = {nullptr, nullptr, nullptr};
  float* dx1[3] = {nullptr, nullptr, nullptr};
  float* dx2[3] = {nullptr, nullptr, nullptr};
  float* f[3] = {nullptr, nullptr, nullptr};
  long long* id = nullptr;
  int* orig = nullptr;
  unsigned* key = nullptr;  // per particle: its bin, then (cap on) its rank in the bin
  unsigned* cnt = nullptr;  // per bin: count, then start
  unsigned* bsum = nullptr; // scan scratch
};
void particle_order_free(ParticleOrder* o);
// Allocate o's arrays for up to cap particles now (before a stream capture,
// which must not allocate); a later sort of at most cap particles then
// allocates nothing.
cudaError_t particle_order_reserve(ParticleOrder* o, long long cap);
// Sort s into cell order, allocating o's arrays on first use (o's
// capacity is s->cap).  s's array pointers are exchanged with o's scratch
// set, so the owner of s must free its arrays through the allocations it
// made, not through s's current pointers.
cudaError_t particles_sort_cells(ParticleSoA* s, ParticleOrder* o, float L, cudaStream_t st);
// Put s's forces back in the caller's order (before the particles
// themselves are replaced in that order); o holds the scratch arrays.
cudaError_t particles_unsort_forces(ParticleSoA* s, ParticleOrder* o, cudaStream_t st);
