// Snapshot output shared by the handle API and the drop-in layer: the
// GADGET writer and the device copy of the drop-in snapshot.
#pragma once
#include <cuda_runtime.h>

#include "../../include/colagpu_dropin.h"

// Write np ParticleMinimum particles (device memory when on_device, else
// host) as a GADGET-1 file.  Device input is read after the work queued on
// `upstream` so far.  Returns a CG_* code; the message is set on failure.
int gadget_write(const char* filename, const void* pmin, bool on_device, long long np,
                 long long np_total, int num_files, float a, float boxsize, float omega_m,
                 float h, int use_long_id, cudaStream_t upstream);

// capi.cu: the device copy (ParticleMinimum[np_local]) of `snapshot` left by
// the last cola_set_snapshot while it still matches the host array, else
// NULL; *st receives the stream its producer ran on.
ParticleMinimum* dropin_device_snapshot(const Snapshot* snapshot, cudaStream_t* st);
