/*
 * libcolagpu -- B200 particle-mesh force, COLA time step and 2LPT setup for
 * cola_halo, behind a plain C ABI.
 *
 * Two layers:
 *
 *   1. Drop-in entry points with the reference's own names and signatures
 *      (declared in colagpu_dropin.h).  A caller built against the
 *      reference's pm.h / cola.h / lpt.h / power.h / move.h links this
 *      library instead of pm.o cola.o lpt.o power.o move.o.
 *
 *   2. The handle API below (cg_*): one cg_sim holds the device particle
 *      state (structure of arrays) and the PM mesh plan of one realization,
 *      so a process can run several meshes or realizations at once.
 *
 * All cg_* functions return 0 on success and a negative CG_E* code on
 * failure; cg_last_error() describes the last failure of the calling thread.
 * Work is queued on the handle's own CUDA stream: functions that hand data
 * back to host memory synchronise that stream, the others return as soon as
 * the work is queued.
 *
 * Particle layouts exchanged with the host are the reference's
 * (particle.h:6-48): Particle (56 B: x, dx1, dx2, v, id) and ParticleMinimum
 * (32 B: x, v, id).
 */
#ifndef COLAGPU_H
#define COLAGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CG_OK 0
#define CG_EINVAL (-1)      /* bad argument */
#define CG_ECUDA (-2)       /* CUDA runtime error (message has the details) */
#define CG_ENOMEM (-3)      /* device or pinned-host allocation failed */
#define CG_EDENSITY (-4)    /* CIC density sum check failed (pm.c:548-553) */
#define CG_EPARTICLE (-5)   /* a particle position was non-finite or below 0 */
#define CG_EUNSUPPORTED (-6)/* mesh size not built into this library */
#define CG_EFILE (-7)       /* file unreadable or unwritable */

typedef struct cg_sim cg_sim;

/* Library / error information. */
const char* cg_last_error(void);
int cg_version(void);
/* 1 if mesh size n (cells per dimension) is supported: n in
 * {16, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024}. */
int cg_mesh_supported(int n);
/* Number of visible CUDA devices (0 when there is none or no driver). */
int cg_device_count(void);
/* Make device `dev` current for the calling host thread (one process per
 * GPU: call once before any other cg_* / drop-in call). */
int cg_set_device(int dev);

/* Pinned host memory for fast host<->device particle transfers. */
void* cg_host_alloc(size_t bytes);
void cg_host_free(void* p);

/* Create a realization: nc^3 particles capacity np_capacity (>= nc^3),
 * PM mesh of ngrid^3 cells (ngrid = factor * nc in the reference; any
 * built mesh size here, a particle weighing (ngrid/nc)^3 mesh units),
 * periodic box boxsize.  Replaces pm_init (pm.c:87-198) for one handle. */
int cg_sim_create(cg_sim** out, int nc, int ngrid, float boxsize, double omega_m,
                  long long np_capacity);
void cg_sim_destroy(cg_sim* s);

/* Load particles from a host (or device) array of reference Particle
 * structs; a_x / a_v are the position and velocity scale factors
 * (particle.h:18). */
int cg_sim_set_particles(cg_sim* s, const void* particles, long long np, float a_x, float a_v);
/* Copy the state back into a host array of reference Particle structs. */
int cg_sim_get_particles(cg_sim* s, void* particles);
/* Copy the last computed forces (np x 3 floats, particle order) to host. */
int cg_sim_get_forces(cg_sim* s, float* f);
int cg_sim_get_times(cg_sim* s, float* a_x, float* a_v);
long long cg_sim_np(cg_sim* s);

/* move_particles2 on one GPU (move.c:34-41): periodic wrap of x, y, z. */
int cg_sim_move(cg_sim* s);
/* Cell order (no reference counterpart): every `every`-th cg_sim_move
 * (default 2 for simulations of at least 2^23 particles, else 0 = never;
 * the environment variable COLAGPU_SORT_EVERY sets the default) sorts the
 * particles on the device by a grid of about eight
 * particles per cell, so that the deposit and the interpolation keep the
 * memory locality of the initial lattice as structure forms.  Results are
 * unchanged up to the order of the deposit's float additions: every output
 * (cg_sim_get_particles, cg_sim_get_forces, snapshots) is in the order the
 * particles were given in. */
int cg_sim_set_sort_interval(cg_sim* s, int every);
/* Force kernel of the Green step (no reference counterpart; the
 * reference's kernel, pm.c:304-346, is the default: exact spectral gradient
 * i n_a, exact 1/|n|^2, no window correction).  gradient: 0 spectral, 2 the
 * 2-point or 4 the 4-point central difference of the potential (applied in
 * Fourier space as the difference operator's transfer function, identical
 * to the real-space stencil on the periodic mesh); laplacian: 0 exact, 1 the
 * 7-point discrete Laplacian; deconvolve: divide the force by the CIC
 * window sinc^2 per axis 0, 1 (deposit) or 2 (deposit and interpolation)
 * times.  The environment variable COLAGPU_FORCE_KERNEL=g,l,d sets it for
 * every realization created afterwards, the drop-in's included.
 * CG_EINVAL for other values. */
int cg_sim_set_force_kernel(cg_sim* s, int gradient, int laplacian, int deconvolve);

/* Isotropic transfer functions of the PM force (no reference counterpart;
 * the Fourier-space learned correction): the Green step multiplies the
 * force spectrum by T(|n|), |n| in units of the fundamental mode, given at
 * n >= 2 equally spaced knots from 0 to sqrt(3) ngrid / 2 (linear between
 * knots).  cg_sim_set_force_filters copies nsets such functions (host
 * array, nsets x n floats) to the device and makes set 0 current; n = 0
 * removes them.  cg_sim_use_force_filter selects the set the following
 * force evaluations apply (-1: none, the reference's force); it copies
 * nothing, so a time loop can switch sets per step. */
int cg_sim_set_force_filters(cg_sim* s, const float* knots, int n, int nsets);
int cg_sim_use_force_filter(cg_sim* s, int set);
/* pm_calculate_forces (pm.c:565-596).  If density_sum is non-NULL the
 * stream is synchronised and the mesh sum (check_total_density) returned. */
int cg_sim_forces(cg_sim* s, double* density_sum);
/* cola_kick (cola.c:73-117) / cola_drift (cola.c:119-153) with the time
 * coefficients computed on the host in double precision. */
int cg_sim_kick(cg_sim* s, float avel1);
int cg_sim_drift(cg_sim* s, float apos1);
/* The same updates with caller-supplied single-precision coefficients
 * (dda, q1, q2) / (dyyy, da1, da2); they do not change a_x / a_v. */
/* cg_sim_kick(avel1) followed by cg_sim_drift(apos1) in one pass over the
 * particles (no reference counterpart; the same results bit for bit, with
 * one read of the particle state instead of two). */
int cg_sim_kick_drift(cg_sim* s, float avel1, float apos1);
int cg_sim_kick_coeffs(cg_sim* s, float dda, float q1, float q2);
int cg_sim_drift_coeffs(cg_sim* s, float dyyy, float da1, float da2);
/* cola_set_snapshot (cola.c:341-416) into a host ParticleMinimum array. */
int cg_sim_snapshot(cg_sim* s, double aout, float omega_m, void* pmin_out);
/* Wait for all queued work of the handle; reports device-side errors. */
int cg_sim_sync(cg_sim* s);
/* Power spectrum of the particles' CIC density on the PM mesh (no
 * reference counterpart; the reference writes only a coarse density grid,
 * coarse_grid.c).  delta_k = r2c(delta)/ngrid^3, P = L^3 |delta_k|^2
 * averaged over shells: bin b has |n| in [b+1/2, b+3/2) in units of the
 * fundamental 2 pi/L.  Outputs nbins values each of mean k (h/Mpc), P(k)
 * ((Mpc/h)^3) and the number of modes.  nbins <= ngrid.  Overwrites the
 * density mesh; synchronous. */
#define CG_PK_DECONVOLVE_CIC 1   /* divide by the CIC window squared */
#define CG_PK_SUBTRACT_SHOT 2    /* subtract L^3 / np */
int cg_sim_power_spectrum(cg_sim* s, int nbins, int flags, double* k, double* pk,
                          double* nmodes);
/* The shell sums of cg_sim_power_spectrum for a half spectrum the caller
 * already holds in device memory, without allocating anything (no reference
 * counterpart).  For callers that cannot allocate device memory where they
 * measure P(k): a caller whose memory pool or arena owns the whole device,
 * or a program that has given all of HBM to its meshes, where cudaMalloc
 * would fail or take memory the pool counts as its own.
 * d_spec: device, n*n*(n/2+1) interleaved complex [x][y][kz], unnormalised
 * r2c of delta (the cg_fft_r2c layout); n even.  Same bins, flags and units
 * as cg_sim_power_spectrum; np is the particle count for
 * CG_PK_SUBTRACT_SHOT.  stream: a cudaStream_t, or NULL for the default
 * stream; synchronous on it.
 * Scratch is a fixed device array compiled into the library: at most
 * CG_PK_NOALLOC_MAX_BINS bins (larger nbins returns CG_EINVAL).  Every call
 * on a device shares that one array, so calls that overlap (from two host
 * threads, or on two streams at once) race and must not be made.  The first
 * call on each device, made with that device current, looks the array's
 * device address up; make it before any stream capture.  A later call looks
 * it up again if the device's context has changed (cudaDeviceReset). */
#define CG_PK_NOALLOC_MAX_BINS 1024
int cg_pk_bins_noalloc(const void* d_spec, int n, float boxsize, int nbins, int flags,
                       double* k, double* pk, double* nmodes, long long np, void* stream);
/* Copy one mesh to host: which = 0 density (delta), 1..3 force x, y, z;
 * ngrid^3 floats, [x][y][z] order.  The force step's z transform resets the
 * density mesh to -1 for the next deposit, so after cg_sim_forces (unless
 * the handle keeps its density, cg_sim_keep_density) which = 0 deposits the
 * particles' CURRENT positions again: after a kick/drift that is not the
 * density behind the force meshes 1..3 of the same step. */
int cg_sim_get_mesh(cg_sim* s, int which, float* out);
/* keep = 1: the force step leaves the density mesh in place (its z transform
 * does not reset it), so cg_sim_get_mesh(s, 0, ..) returns the density the
 * last force step used; the next deposit then fills the mesh with -1 first
 * (one more pass over the mesh).  keep = 0 (the default): the reset. */
int cg_sim_keep_density(cg_sim* s, int keep);
/* The CUDA stream (cudaStream_t) the handle queues its work on. */
void* cg_sim_stream(cg_sim* s);

/* Copy the particle state (x, v, dx1, dx2, id, a_x, a_v) of src into dst
 * (device to device), e.g. to evaluate two meshes on the same particles. */
int cg_sim_copy_particles(cg_sim* dst, const cg_sim* src);

/* Learned small-scale force correction (no reference counterpart).  A
 * three-layer 3x3x3 periodic conv net on a coarse mesh (2 -> 16 -> 16 -> 3
 * channels, leaky-ReLU 0.1, bf16 weights and activations, fp32
 * accumulation; convolutions on tcgen05 tensor cores when the mesh is a
 * multiple of 128) maps (delta, phi) of the coarse mesh to a force residual
 * that is CIC-interpolated to the particles and added to the coarse PM
 * force.  Trained by the library's own forward/backward kernels and Adam on
 * pairs generated by the PM method: the fine-mesh minus coarse-mesh force
 * at the same particles, deposited on the coarse mesh (mass-weighted MSE).
 * Parameters: 3 layers x (27*16*16 weights W[tap][ci][cout] + 16 biases). */
typedef struct cg_net cg_net;
int cg_net_create(cg_net** out, int ngrid, unsigned long long seed);
void cg_net_destroy(cg_net* h);
int cg_net_num_params(void);
int cg_net_get_params(cg_net* h, float* params);
int cg_net_set_params(cg_net* h, const float* params);
int cg_net_set_scales(cg_net* h, float in_delta, float in_phi, float out_scale);
/* 1: tcgen05 convolutions (default); 0: CUDA-core convolutions. */
int cg_net_set_tensor_cores(cg_net* h, int on);
/* Pipeline of the tensor-core convolutions, for every net: -1 by mesh size
 * (the default), 0 two stages, 1 one stage, 2 the line ring that reuses
 * input lines along y (128^3 meshes).  All give bit-identical outputs. */
int cg_net_set_conv_variant(int variant);
/* Host-array forward / backward (checks): in2 [v][2] scaled features,
 * out3 [v][3] raw outputs, grad3 = dLoss/dout3, grads [num_params]. */
int cg_net_forward_host(cg_net* h, const float* in2, float* out3);
int cg_net_backward_host(cg_net* h, const float* in2, const float* grad3, float* grads);
/* Training step on two realizations holding the same particles; returns the
 * loss before the update.  lr <= 0 evaluates without updating. */
int cg_net_train_step(cg_net* h, cg_sim* coarse, cg_sim* fine, float lr, double* loss);
/* cg_sim_forces of the coarse realization plus the learned correction. */
int cg_net_forces(cg_net* h, cg_sim* coarse);

/* Batched realizations in one CUDA graph launch (no reference counterpart:
 * the reference loops over seeds one at a time, main.c:117-209).  Each
 * realization has its own particles, mesh, box size and schedule: nsteps
 * drifts linear in a from a_init to a_final (nsteps + 1 force
 * evaluations), one snapshot at aout, and the P(k) of its final positions
 * (ngrid/2 bins, as cg_sim_power_spectrum without flags).  The whole batch
 * is recorded into one graph on the first cg_batch_run and relaunched on
 * later calls; every launch restarts from the stored initial particles. */
typedef struct {
  int nc;            /* particles per dimension */
  int ngrid;         /* mesh cells per dimension (a multiple of nc) */
  float boxsize;     /* Mpc/h */
  double a_init, a_final;
  int nsteps;
  float aout;        /* snapshot scale factor */
} cg_realization_spec;
typedef struct cg_batch cg_batch;
int cg_batch_create(cg_batch** out, int nreal, const cg_realization_spec* specs,
                    double omega_m, int nstreams);
void cg_batch_destroy(cg_batch* b);
/* Initial particles of realization i: nc^3 reference Particle structs. */
int cg_batch_set_particles(cg_batch* b, int i, const void* particles, long long np);
/* Cell-order sort of every realization's particles at every every-th move,
 * inside the graph (0: never).  Default: the cg_sim policy (every sixth
 * move from 2^23 particles).  Only before the first cg_batch_run. */
int cg_batch_set_sort_interval(cg_batch* b, int every);
/* Launch (recording first if needed) and wait; checks every density sum. */
int cg_batch_run(cg_batch* b);
int cg_batch_get_snapshot(cg_batch* b, int i, void* pmin_out);
int cg_batch_power_spectrum(cg_batch* b, int i, double* k, double* pk, double* nmodes);
/* Number of nodes of the recorded graph (after the first run). */
int cg_batch_num_nodes(cg_batch* b, size_t* nodes);
/* Device time (CUDA events around the graph launch) of the last
 * cg_batch_run, in milliseconds. */
int cg_batch_last_ms(cg_batch* b, float* ms);

/* Unnormalised 3-D real transforms of host arrays on the device, FFTW sign
 * convention (replaces the fftwf_mpi r2c / c2r plans of pm.c:141-147 and
 * lpt.c:118-134 for one process).  real: n^3 floats [x][y][z]; spec:
 * n*n*(n/2+1) interleaved complex [x][y][kz].  The c2r is c2c over x and y
 * followed by a c2r over z that ignores Im of kz = 0 and kz = n/2, as
 * FFTW's c2r does.  Synchronous; allocates its own scratch. */
int cg_fft_r2c(int n, const float* real_in, float* spec_out);
int cg_fft_c2r(int n, const float* spec_in, float* real_out);
/* Device time in ms of one r2c and one c2r of an n^3 mesh held in device
 * memory (the mean of `reps` launches after a warm-up); for comparing the
 * transforms with other FFT implementations. */
int cg_fft_time(int n, int reps, float* ms_r2c, float* ms_c2r);

/* Friends-of-friends halos (fof.c:427-1181 on one process).  pmin: np
 * reference ParticleMinimum structs (32 B: x, v, id) in host or device
 * memory, positions within one box length of [0, L).  Particles closer than
 * ll are linked (periodic box of side boxsize); groups of at least
 * nfof_min members are halos: member count, centre (a member plus the mean
 * minimum-image offset, wrapped into [0, L)) and mean velocity.  Halos come
 * in the order of each group's smallest particle index.  Up to max_halos
 * are written to `halos` (may be NULL); *nhalo receives the total count.
 * Synchronous; allocates and frees its own device scratch. */
typedef struct {
  int nfof;
  float x[3];
  float v[3];
} cg_halo;
int cg_fof(const void* pmin, long long np, float boxsize, float ll, int nfof_min,
           cg_halo* halos, long long max_halos, long long* nhalo);

/* Coarse density grid (coarse_grid.c:17-121): CIC assignment of np
 * ParticleMinimum (host or device memory) onto an nc^3 grid [x][y][z] of a
 * periodic box, then delta = nc^3 / np_total * rho - 1, all in float with
 * the reference's weight arithmetic.  delta_out (nc^3 floats, host or
 * device) receives the contrast; *mass_sum (may be NULL) the sum of rho in
 * double.  1 <= nc <= 1024.  Grids of up to 16384 cells are accumulated
 * per CTA in shared memory first.  Synchronous; allocates and frees its own
 * device grid. */
int cg_coarse_grid(const void* pmin, long long np, long long np_total, float boxsize, int nc,
                   float* delta_out, double* mass_sum);

/* GADGET-1 snapshot file (write.c:14-107, one file): header, positions,
 * velocities times 1/sqrt(a), ids (4-byte unsigned, or 8-byte with
 * use_long_id), each record framed by its int byte length.  pmin holds np
 * ParticleMinimum in host or device memory; the header's particle mass uses
 * np_total.  Device input is formatted on the GPU chunk by chunk and
 * downloaded through pinned buffers while the previous chunk is written.
 * Synchronous.  CG_EFILE when the file cannot be written. */
int cg_write_gadget(const char* filename, const void* pmin, long long np, long long np_total,
                    int num_files, float a, float boxsize, float omega_m, float h,
                    int use_long_id);
/* The snapshot at aout (as cg_sim_snapshot) written straight from the
 * device as a GADGET-1 file, with no host copy of the particles. */
/* set_noncola_initial (cola.c:297-338): the snapshot of the 2LPT initial
 * condition at the current a_x (positions, velocities 100/a (dx1 D1' +
 * dx2 D2')) into pmin_out (np ParticleMinimum, host or device). */
int cg_sim_initial_snapshot(cg_sim* s, float omega_m, void* pmin_out);
int cg_sim_write_gadget(cg_sim* s, double aout, float omega_m, float h, const char* filename,
                        int use_long_id);

/* FFT schedule autotuner (no reference counterpart).  From 256 up each
 * mesh size has several compiled variants of the strided x pass (ky columns
 * per CTA, maximum radix) and, up to 768, of the fused y Green pass (lines
 * per CTA, maximum radix, CTAs per SM).  cg_autotune times them on a
 * temporary plan of that size on the current device, installs the fastest
 * of each for the process, and appends the choice to the file named by
 * COLAGPU_TUNE_CACHE (if set), which later calls read instead of timing.
 * ms_green / ms_fx (may be NULL; cg_schedule_variants entries each) receive
 * the best time of every variant when they were timed.  CG_TUNE_FORCE
 * re-times.  The variants agree to float rounding; a fixed schedule
 * (cached, or set with cg_set_schedule) makes runs bit-reproducible.
 * Variant 0 is the default; sizes below 256 have only variant 0.  Tune
 * outside stream capture. */
#define CG_TUNE_FORCE 1
int cg_autotune(int ngrid, int flags, float* ms_green, float* ms_fx);
int cg_schedule_variants(int ngrid, int* n_green, int* n_fx);
int cg_get_schedule(int ngrid, int* green_variant, int* fx_variant);
int cg_set_schedule(int ngrid, int green_variant, int fx_variant);
/* How the z c2r of the force step gathers its transposed input, for the
 * handles created afterwards: 0 cp.async, 1 TMA into a landing area, 2 TMA
 * into the transform's own swizzled tile, -1 (the default) by mesh size.
 * The three give bit-identical forces; COLAGPU_ZI=0/1/2 overrides. */
int cg_set_z_gather(int mode);
/* Deposit of the force step (PtoMesh + the r2c along z, pm.c:229-301), for
 * every handle from the next force step on: 0 (the default, also -1)
 * deposits into the mesh and then transforms it; 1 bins the particles'
 * clouds by mesh column with warp-aggregated atomics, and each CTA of the z
 * transform builds its own density lines in shared memory from its
 * columns' clouds, so the density mesh never goes through HBM.  The two
 * agree to float rounding (only the order of the deposit's float additions
 * differs); 1 adds them in an order that changes from run to run, so its
 * forces are not bit-reproducible.  A handle that keeps its density
 * (cg_sim_keep_density) always takes 0.  COLAGPU_FUSED_DEPOSIT=0/1
 * overrides. */
int cg_set_force_deposit(int mode);
/* Interpolation of the force step (force_at_particle_locations ×3 + the
 * buffer copies' forces, pm.c:359-412, 505-532), for every handle from the
 * next force step on: 0 (the default, also -1) writes the force meshes and
 * interpolates from them; 1 bins the particles' clouds by mesh column, and
 * each CTA of the z c2r interpolates the clouds of its plane from the force
 * lines it has just transformed in shared memory, so the three force
 * meshes never go through HBM.  The forces are the same bit for bit.  After
 * a step with 1, cg_sim_get_mesh(s, 1..3, ..) transforms the requested
 * force mesh from its spectrum first.  COLAGPU_FUSED_INTERP=0/1 overrides. */
int cg_set_force_interp(int mode);

/* Slab decomposition of one realization's PM force over ranks (one GPU per
 * rank).  It replaces the reference's MPI slabs: comm_init's x slabs
 * (comm.c:35-111), the FFTW-MPI transposes inside pm.c:282-355, the buffer
 * particles of send_buffer_positions / add_buffer_forces (pm.c:416-532) and
 * move_particles2's exchange (move.c:15-175).  Every rank's handle holds full-size
 * meshes; rank r owns mesh planes [x0, x0 + nx) and kz planes [kz0, kz0 +
 * nkz) of the spectra.  Per force evaluation:
 *   cg_sim_slab_density  density of the rank's particles and of the buffer
 *                        copies it received (bx: 3 x nb floats, SoA, device;
 *                        copies keep their own weights, shifted by -L across
 *                        the periodic face), its r2c along z for planes
 *                        [x0, x0+nx); density_sum (may be NULL) receives the
 *                        slab's part of check_total_density's sum;
 *   (caller)             spectrum x slabs -> kz slabs (cg_sim_spectrum_ptr 0);
 *   cg_sim_slab_kspace   x, Green and inverse x passes of kz planes [kz0,
 *                        kz0+nkz) into the three force spectra;
 *   (caller)             force spectra kz slabs -> x slabs (ptr 1..3);
 *   cg_sim_slab_c2r      the three z c2r of planes [x0, x0+nx);
 *   cg_sim_slab_interp   forces of the rank's particles and of the buffer
 *                        copies (bf: 3 x nb floats) from planes [x0, x0+nx);
 *   (caller)             buffer forces back to their owners, added to theirs.
 * cg_sim_state_ptrs gives the device arrays of positions and forces (three
 * each); cg_sim_spectrum_ptr the half spectrum (0) or the force spectra
 * (1..3), laid out [kz][kx][ky].  cola_halo_b200/slab.py drives them over
 * torch.distributed. */
int cg_sim_state_ptrs(cg_sim* s, float** x, float** f);
int cg_sim_spectrum_ptr(cg_sim* s, int which, void** ptr);
int cg_sim_slab_density(cg_sim* s, int x0, int nx, const float* bx, long long nb,
                        double* density_sum);
int cg_sim_slab_kspace(cg_sim* s, int kz0, int nkz);
int cg_sim_slab_c2r(cg_sim* s, int x0, int nx);
int cg_sim_slab_interp(cg_sim* s, int x0, int nx, const float* bx, long long nb, float* bf);
/* Shape of the CIC deposit per mesh size (no reference counterpart; the
 * reference's PtoMesh is pm.c:209-279): variant v of cg_deposit_variants()
 * sets the particles per CTA and the shared-memory box (512 / 3,072 cells,
 * 256 / 3,072, 1,024 / 6,144, 2,048 / 12,288, 512 / 6,144, or global
 * atomics only).  cg_sim_tune_deposit times every variant on the handle's
 * current particles (best of 3 CUDA-event timings), installs the fastest
 * for the handle's mesh size and returns it (or a negative CG_E* code); ms
 * (may be NULL) receives each variant's time.  It wraps the positions into
 * the box first (move_particles2's wrap) and leaves a deposit of them in
 * the density mesh.  All variants give the same density to float
 * rounding. */
int cg_deposit_variants(void);
int cg_get_deposit_variant(int ngrid);
int cg_set_deposit_variant(int ngrid, int variant);
int cg_sim_tune_deposit(cg_sim* s, float* ms);
/* How the strided x pass of the force step gathers its columns, for the
 * handles created afterwards: 0 direct loads, 1 TMA into the transform's
 * own swizzled tile, -1 (the default) by mesh size.  Bit-identical forces;
 * COLAGPU_FXG=0/1 overrides. */
int cg_set_x_gather(int mode);

/* Kernel accounting (no reference counterpart; the reference's wall-clock
 * timers are timer.c).  cg_launch_count: kernels launched by this library
 * since load.  cg_prof_begin / cg_prof_end bracket a region: every launch in
 * between records a CUDA event; cg_prof_end synchronises, and fills
 * ms[stage] (device time) and counts[stage] (launches) for nstages stages
 * named by cg_stage_name(stage).  Returns the number of launches timed. */
long long cg_launch_count(void);
const char* cg_stage_name(int stage);
int cg_prof_begin(int max_marks);
int cg_prof_end(double* ms, int* counts, int nstages);

/* Host time coefficients (double-precision restatement of cola.c:156-292). */
double cg_growth_D1(double omega_m, double a);
double cg_growth_D2(double omega_m, double a);
double cg_cola_Sq(double omega_m, double ai, double af, double aref);
double cg_cola_Sphi(double omega_m, double ai, double af, double aref);
void cg_kick_coeffs(double omega_m, float a_v, float a_x, float avel1, float out3[3]);
void cg_drift_coeffs(double omega_m, float a_x, float a_v, float apos1, float out3[3]);

#ifdef __cplusplus
}
#endif
#endif
