"""ctypes binding of libcolagpu.so (the C ABI declared in include/colagpu.h
and include/colagpu_dropin.h).

The library is built in-tree by ``cola_halo_b200.build``; ``load()`` builds
it when it is missing and nvcc is available, and raises otherwise -- there is
no CPU fallback for any entry point.
"""
import ctypes
import os

from . import build as _build

_lib = None

P = ctypes.c_void_p
f32 = ctypes.c_float
f64 = ctypes.c_double
i32 = ctypes.c_int
i64 = ctypes.c_longlong
sz = ctypes.c_size_t
fptr = ctypes.POINTER(ctypes.c_float)
dptr = ctypes.POINTER(ctypes.c_double)

# name: (restype, argtypes)
SIGNATURES = {
    # handle API (colagpu.h)
    "cg_last_error": (ctypes.c_char_p, []),
    "cg_version": (i32, []),
    "cg_mesh_supported": (i32, [i32]),
    "cg_device_count": (i32, []),
    "cg_set_device": (i32, [i32]),
    "cg_host_alloc": (P, [sz]),
    "cg_host_free": (None, [P]),
    "cg_sim_create": (i32, [ctypes.POINTER(P), i32, i32, f32, f64, i64]),
    "cg_sim_destroy": (None, [P]),
    "cg_sim_set_particles": (i32, [P, P, i64, f32, f32]),
    "cg_sim_get_particles": (i32, [P, P]),
    "cg_sim_get_forces": (i32, [P, P]),
    "cg_sim_get_times": (i32, [P, fptr, fptr]),
    "cg_sim_np": (i64, [P]),
    "cg_sim_move": (i32, [P]),
    "cg_sim_forces": (i32, [P, dptr]),
    "cg_sim_kick": (i32, [P, f32]),
    "cg_sim_drift": (i32, [P, f32]),
    "cg_sim_kick_drift": (i32, [P, f32, f32]),
    "cg_sim_kick_coeffs": (i32, [P, f32, f32, f32]),
    "cg_sim_drift_coeffs": (i32, [P, f32, f32, f32]),
    "cg_sim_snapshot": (i32, [P, f64, f32, P]),
    "cg_sim_sync": (i32, [P]),
    "cg_sim_get_mesh": (i32, [P, i32, P]),
    "cg_sim_keep_density": (i32, [P, i32]),
    "cg_sim_power_spectrum": (i32, [P, i32, i32, P, P, P]),
    "cg_pk_bins_noalloc": (i32, [P, i32, f32, i32, i32, P, P, P, i64, P]),
    "cg_sim_stream": (P, [P]),
    "cg_sim_copy_particles": (i32, [P, P]),
    "cg_sim_set_sort_interval": (i32, [P, i32]),
    "cg_sim_set_force_filters": (i32, [P, P, i32, i32]),
    "cg_sim_use_force_filter": (i32, [P, i32]),
    "cg_sim_set_force_kernel": (i32, [P, i32, i32, i32]),
    "cg_net_create": (i32, [ctypes.POINTER(P), i32, ctypes.c_ulonglong]),
    "cg_net_destroy": (None, [P]),
    "cg_net_num_params": (i32, []),
    "cg_net_get_params": (i32, [P, P]),
    "cg_net_set_params": (i32, [P, P]),
    "cg_net_set_scales": (i32, [P, f32, f32, f32]),
    "cg_net_set_tensor_cores": (i32, [P, i32]),
    "cg_net_set_conv_variant": (i32, [i32]),
    "cg_net_forward_host": (i32, [P, P, P]),
    "cg_net_backward_host": (i32, [P, P, P, P]),
    "cg_net_train_step": (i32, [P, P, P, f32, dptr]),
    "cg_net_forces": (i32, [P, P]),
    "cg_batch_create": (i32, [ctypes.POINTER(P), i32, P, f64, i32]),
    "cg_batch_destroy": (None, [P]),
    "cg_batch_set_particles": (i32, [P, i32, P, i64]),
    "cg_batch_run": (i32, [P]),
    "cg_batch_set_sort_interval": (i32, [P, i32]),
    "cg_batch_get_snapshot": (i32, [P, i32, P]),
    "cg_batch_power_spectrum": (i32, [P, i32, P, P, P]),
    "cg_batch_num_nodes": (i32, [P, ctypes.POINTER(sz)]),
    "cg_batch_last_ms": (i32, [P, fptr]),
    "cg_fof": (i32, [P, i64, f32, f32, i32, P, i64, ctypes.POINTER(i64)]),
    "cg_coarse_grid": (i32, [P, i64, i64, f32, i32, P, ctypes.POINTER(f64)]),
    "cg_write_gadget": (i32, [ctypes.c_char_p, P, i64, i64, i32, f32, f32, f32, f32, i32]),
    "cg_sim_write_gadget": (i32, [P, f64, f32, f32, ctypes.c_char_p, i32]),
    "cg_sim_initial_snapshot": (i32, [P, f32, P]),
    "cg_snapshot_invalidate": (None, []),
    "cg_autotune": (i32, [i32, i32, P, P]),
    "cg_schedule_variants": (i32, [i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
    "cg_get_schedule": (i32, [i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
    "cg_set_schedule": (i32, [i32, i32, i32]),
    "cg_set_z_gather": (i32, [i32]),
    "cg_set_x_gather": (i32, [i32]),
    "cg_set_force_deposit": (i32, [i32]),
    "cg_set_force_interp": (i32, [i32]),
    "cg_sim_state_ptrs": (i32, [P, ctypes.POINTER(P), ctypes.POINTER(P)]),
    "cg_sim_spectrum_ptr": (i32, [P, i32, ctypes.POINTER(P)]),
    "cg_sim_slab_density": (i32, [P, i32, i32, P, i64, dptr]),
    "cg_sim_slab_kspace": (i32, [P, i32, i32]),
    "cg_sim_slab_c2r": (i32, [P, i32, i32]),
    "cg_sim_slab_interp": (i32, [P, i32, i32, P, i64, P]),
    "cg_deposit_variants": (i32, []),
    "cg_get_deposit_variant": (i32, [i32]),
    "cg_set_deposit_variant": (i32, [i32, i32]),
    "cg_sim_tune_deposit": (i32, [P, P]),
    "cg_fft_r2c": (i32, [i32, P, P]),
    "cg_fft_c2r": (i32, [i32, P, P]),
    "cg_fft_time": (i32, [i32, i32, fptr, fptr]),
    "cg_launch_count": (i64, []),
    "cg_stage_name": (ctypes.c_char_p, [i32]),
    "cg_prof_begin": (i32, [i32]),
    "cg_prof_end": (i32, [P, P, i32]),
    "cg_growth_D1": (f64, [f64, f64]),
    "cg_growth_D2": (f64, [f64, f64]),
    "cg_cola_Sq": (f64, [f64, f64, f64, f64]),
    "cg_cola_Sphi": (f64, [f64, f64, f64, f64]),
    "cg_kick_coeffs": (None, [f64, f32, f32, f32, fptr]),
    "cg_drift_coeffs": (None, [f64, f32, f32, f32, fptr]),
    # drop-in layer (colagpu_dropin.h)
    "pm_init": (None, [i32, i32, f32, f32, P, sz, P, sz]),
    "pm_calculate_forces": (None, [P]),
    "cola_kick": (None, [P, f32, f32]),
    "cola_drift": (None, [P, f32, f32]),
    "cola_set_snapshot": (None, [f64, P, P]),
    "set_noncola_initial": (None, [P, P]),
    "move_particles2": (None, [P, f32, P, sz]),
    "lpt_init": (None, [i32, P, sz]),
    "lpt_set_displacement": (i32, [f64, f64, i32, f64, P]),
    "lpt_get_local_nx": (i32, []),
    "power_init": (None, [ctypes.c_char_p, f64, f64, f64, f64]),
    "PowerSpec": (f64, [f64]),
    "GrowthFactor": (f64, [f64, f64]),
    "fof_calc_memory": (sz, [i32, i32]),
    "fof_init": (None, [i32, i32, P, sz]),
    "fof_find_halos": (None, [P, f32]),
    "fof_write_halos": (None, [ctypes.c_char_p]),
    "coarse_grid2": (None, [ctypes.c_char_p, P, i32, P, sz]),
    "write_snapshot": (None, [ctypes.c_char_p, P, i32]),
    "cg_particles_upload": (i32, [P]),
    "cg_particles_download": (i32, [P]),
    "cg_dropin_set_sync": (None, [i32]),
    "cg_dropin_set_abort": (None, [i32]),
    "cg_dropin_finalize": (None, []),
}


class ColaGpuError(RuntimeError):
    pass


def lib_path():
    return _build.LIB


def load(build_if_missing=True):
    """Load libcolagpu.so (building it first if needed)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise ColaGpuError("libcolagpu.so is not built: run python -m cola_halo_b200.build")
        _build.build(verbose=False)
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


NSTAGES = 16   # CG_ST_COUNT in csrc/internal.h


def check(rc, what=""):
    if rc != 0:
        msg = load().cg_last_error()
        raise ColaGpuError("%s failed (%d): %s" % (what, rc, msg.decode() if msg else ""))
    return rc
