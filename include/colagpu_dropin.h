/*
 * Drop-in replacements for the cola_halo hot-path entry points.
 *
 * Each function has the name, signature and argument meaning of the
 * reference function it replaces (cited below), so the reference's driver
 * (main.c) links against libcolagpu instead of pm.o, cola.o, lpt.o, power.o,
 * move.o, fof.o, coarse_grid.o and write.o.  The data types are the
 * reference's (particle.h:6-48).
 *
 * Errors: like the reference (msg_abort -> MPI_Abort, msg.c:36-45) a failure
 * prints a message and exits the process with the reference's error code
 * (4001 mesh allocation, 6040 density check, 3000 power table, 3010 sigma8,
 * 7000/7050 halo finding, 8110 halo file, 10010/10021 coarse grid, 9000
 * GADGET file),
 * unless cg_dropin_set_abort(0) was called, in which case the call returns
 * and cg_last_error() describes the failure.
 *
 * Particle residency: the first call that sees a Particles object uploads its
 * particles to the GPU; from then on the device copy is the working state and
 * the host array p[] is not read again.  cola_set_snapshot writes its result
 * to the host Snapshot as the reference does.  A caller that changes p[]
 * itself calls cg_particles_upload(); one that wants p[] / force[] on the
 * host calls cg_particles_download().  With cg_dropin_set_sync(1) every call
 * instead reads its inputs from, and writes its outputs to, the host arrays
 * (the reference's exact memory behaviour, at PCIe cost).
 */
#ifndef COLAGPU_DROPIN_H
#define COLAGPU_DROPIN_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* particle.h:6-48.  The reference's `typedef float float3[3]` is kept for C
 * callers; CUDA's own float3 vector type has the same name, so inside a CUDA
 * translation unit the force member is spelled float (*)[3] (same ABI). */
#if !defined(__CUDACC__) && !defined(__VECTOR_TYPES_H__)
typedef float float3[3];
#endif

typedef struct {
  float x[3];
  float dx1[3]; /* ZA displacement */
  float dx2[3]; /* 2LPT displacement */
  float v[3];   /* velocity */
  long long id;
} Particle;

typedef struct {
  Particle* p;
  float (*force)[3];
  float a_x, a_v;
  int np_local, np_allocated;
  long long np_total;
  float np_average;
} Particles;

typedef struct {
  float x[3];
  float v[3];
  long long id;
} ParticleMinimum;

typedef struct {
  ParticleMinimum* p;
  int np_local;
  int np_allocated;
  long long np_total;
  float np_average;
  float a;
  float boxsize;
  int nc;
  float omega_m, h;
  int seed;
  char* filename;
} Snapshot;

/* pm.h:6-9 (pm.c:87-198).  mem1 / mem2 are accepted and not used: the
 * meshes live in device memory. */
void pm_init(const int nc_pm, const int nc_pm_factor, const float boxsize,
             const float np_alloc_factor, void* const mem1, const size_t size1,
             void* const mem2, const size_t size2);
/* pm.h:11 (pm.c:565-596) */
void pm_calculate_forces(Particles* particles);
/* cola.h:7-8 (cola.c:73-117) */
void cola_kick(Particles* const particles, const float Omega_m, const float avel1);
/* cola.h:9-10 (cola.c:119-153) */
void cola_drift(Particles* const particles, const float Omega_m, const float apos1);
/* cola.h:18 (cola.c:341-416) */
void cola_set_snapshot(const double aout, Particles const* const particles,
                       Snapshot* const snapshot);
/* cola.h:16 (cola.c:297-338): snapshot of the 2LPT initial condition at
 * particles->a_x (positions, 2LPT velocities in km/s), for the initial
 * condition file of main.c:131-137. */
void set_noncola_initial(Particles const* const particles, Snapshot* const snapshot);
/* move.h:7 (move.c:15-98); one process: the periodic wrap (move.c:34-41). */
void move_particles2(Particles* const particles, const float BoxSize, void* const buf,
                     const size_t size);
/* lpt.h:6 (lpt.c:46-143).  mem / size are accepted and not used. */
void lpt_init(const int nc, const void* mem, const size_t size);
/* lpt.h:7 (lpt.c:145-578).  Declared void in lpt.h but defined int in
 * lpt.c (returns 0); exported as int. */
int lpt_set_displacement(const double InitTime, const double omega_m, const int Seed,
                         const double Box, Particles* particles);
/* lpt.h:8 (lpt.c:611-614) */
int lpt_get_local_nx(void);
/* power.h:5 (power.c:36-60) */
void power_init(const char filename[], const double a_init, const double sigma8,
                const double omega_m, const double omega_lambda);
/* power.h:4 (power.c:120-151) */
double PowerSpec(const double k);
/* power.h:6 (power.c:199-202) */
double GrowthFactor(double astart, double aend);

/* fof.h:6 (fof.c:973-988): bytes the reference wants in mem1 for the halo
 * finder.  Returned for callers that size their arena with it; the GPU
 * finder keeps its own device buffers. */
size_t fof_calc_memory(const int np_alloc, const int nc);
/* fof.h:7 (fof.c:990-1033).  mem / mem_size are accepted and not used. */
void fof_init(const int np_alloc, const int nc, void* mem, size_t mem_size);
/* fof.h:8 (fof.c:1035-1084): friends-of-friends halos of the snapshot's
 * particles with linking length ll, on the GPU.  Wraps the snapshot's
 * positions into the box in place, as the reference does; unlike the
 * reference it leaves the particle order unchanged (the reference sorts
 * them into its k-d tree). */
void fof_find_halos(Snapshot* snapshot, const float ll);
/* fof.h:10 (fof.c:1086-1181): the halos of the last fof_find_halos with
 * at least 32 members, one line each, "nfof x y z vx vy vz" in the
 * reference's format. */
void fof_write_halos(char filename[]);

/* coarse_grid.h:6 (coarse_grid.c:17-121): CIC density contrast of the
 * snapshot's particles on an nc^3 grid, written as [float boxsize][int nc]
 * [nc^3 float delta, x slowest][int nc].  The grid is assigned on the GPU;
 * mem1 / size1 are accepted and not used. */
void coarse_grid2(const char filename[], Snapshot const* const snapshot, const int nc,
                  void* const mem1, const size_t size1);

/* write.h:7 (write.c:14-107): GADGET-1 file "<filebase>.0" of the
 * snapshot (one process), the reference's bytes.  Error 9000 when the file
 * cannot be written. */
void write_snapshot(const char filebase[], Snapshot const* const snapshot, int use_long_id);

/* Residency and error controls of the drop-in layer (no reference
 * counterpart). */
/* Snapshot residency: cola_set_snapshot leaves its result on the device as
 * well as in snapshot->p, and fof_find_halos, coarse_grid2 and
 * write_snapshot read that device copy while the Snapshot's array and
 * np_local are unchanged (fof_find_halos wraps both copies).  A caller that
 * edits snapshot->p in between calls cg_snapshot_invalidate() first; the
 * next call then reads the host array. */
void cg_snapshot_invalidate(void);
int cg_particles_upload(Particles* particles);
int cg_particles_download(Particles* particles);
void cg_dropin_set_sync(int full);
void cg_dropin_set_abort(int abort_on_error);
/* Release every device buffer of the drop-in layer. */
void cg_dropin_finalize(void);

#ifdef __cplusplus
}
#endif
#endif
