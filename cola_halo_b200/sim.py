"""Python host mirror of the reference's hot-path interface over libcolagpu.

``Simulation`` wraps one ``cg_sim`` handle: a realization's particles held on
the GPU plus its PM mesh plan.  Its methods are the reference's per-step
operations (``move_particles2``, ``pm_calculate_forces``, ``cola_kick``,
``cola_drift``, ``cola_set_snapshot``) and ``run`` drives them with the
reference time loop (main.c:117-206).  All arithmetic runs in the CUDA
library; this module only moves arguments and host arrays.
"""
import ctypes

import numpy as np

from . import _lib
from .schedule import output_scale_factors, run_time_loop
from .types import PARTICLE_DTYPE, PARTICLE_MIN_DTYPE


class Simulation:
    def __init__(self, nc, ngrid, boxsize, omega_m, np_capacity=None):
        self.lib = _lib.load()
        self.nc, self.ngrid, self.boxsize, self.omega_m = nc, ngrid, float(boxsize), float(omega_m)
        h = ctypes.c_void_p()
        cap = np_capacity or nc ** 3
        _lib.check(self.lib.cg_sim_create(ctypes.byref(h), nc, ngrid, self.boxsize,
                                          self.omega_m, cap), "cg_sim_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.cg_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ---------------------------------------------------------
    def set_particles(self, particles, a_x, a_v):
        """particles: numpy array of PARTICLE_DTYPE (reference Particle)."""
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        _lib.check(self.lib.cg_sim_set_particles(self.h, p.ctypes.data, len(p), a_x, a_v),
                   "cg_sim_set_particles")
        self._keep = p

    def set_particles_ptr(self, ptr, n, a_x, a_v):
        """Load n reference Particle structs from a host or device address."""
        _lib.check(self.lib.cg_sim_set_particles(self.h, ptr, n, a_x, a_v),
                   "cg_sim_set_particles")

    def set_state(self, x, dx1, dx2, v=None, ids=None, a_x=0.0, a_v=0.0):
        n = x.shape[0]
        p = np.zeros(n, dtype=PARTICLE_DTYPE)
        p["x"], p["dx1"], p["dx2"] = x, dx1, dx2
        if v is not None:
            p["v"] = v
        p["id"] = np.arange(1, n + 1) if ids is None else ids
        self.set_particles(p, a_x, a_v)

    def get_particles(self):
        n = self.lib.cg_sim_np(self.h)
        out = np.zeros(n, dtype=PARTICLE_DTYPE)
        _lib.check(self.lib.cg_sim_get_particles(self.h, out.ctypes.data), "cg_sim_get_particles")
        return out

    def get_forces(self):
        n = self.lib.cg_sim_np(self.h)
        out = np.zeros((n, 3), dtype=np.float32)
        _lib.check(self.lib.cg_sim_get_forces(self.h, out.ctypes.data), "cg_sim_get_forces")
        return out

    def get_mesh(self, which):
        out = np.zeros((self.ngrid,) * 3, dtype=np.float32)
        _lib.check(self.lib.cg_sim_get_mesh(self.h, which, out.ctypes.data), "cg_sim_get_mesh")
        return out

    def keep_density(self, keep=True):
        """Keep the density the force step used (get_mesh(0) then returns it);
        by default the force step resets the mesh for the next deposit."""
        _lib.check(self.lib.cg_sim_keep_density(self.h, 1 if keep else 0), "cg_sim_keep_density")

    def power_spectrum(self, nbins=None, deconvolve_cic=False, subtract_shot=False):
        """(k, P(k), modes) of the current positions' CIC density."""
        nb = nbins or self.ngrid // 2
        k = np.zeros(nb)
        p = np.zeros(nb)
        m = np.zeros(nb)
        flags = (1 if deconvolve_cic else 0) | (2 if subtract_shot else 0)
        _lib.check(self.lib.cg_sim_power_spectrum(self.h, nb, flags, k.ctypes.data,
                                                  p.ctypes.data, m.ctypes.data),
                   "cg_sim_power_spectrum")
        return k, p, m

    def times(self):
        ax, av = ctypes.c_float(), ctypes.c_float()
        self.lib.cg_sim_get_times(self.h, ctypes.byref(ax), ctypes.byref(av))
        return ax.value, av.value

    # -- reference operations ---------------------------------------------
    def move(self):
        _lib.check(self.lib.cg_sim_move(self.h), "cg_sim_move")

    def forces(self, check_density=False):
        if check_density:
            s = ctypes.c_double()
            _lib.check(self.lib.cg_sim_forces(self.h, ctypes.byref(s)), "cg_sim_forces")
            return s.value
        _lib.check(self.lib.cg_sim_forces(self.h, None), "cg_sim_forces")
        return None

    def kick(self, avel1):
        _lib.check(self.lib.cg_sim_kick(self.h, avel1), "cg_sim_kick")

    def drift(self, apos1):
        _lib.check(self.lib.cg_sim_drift(self.h, apos1), "cg_sim_drift")

    def kick_drift(self, avel1, apos1):
        """kick(avel1) then drift(apos1) in one pass (bit-identical)."""
        _lib.check(self.lib.cg_sim_kick_drift(self.h, avel1, apos1), "cg_sim_kick_drift")

    def kick_coeffs(self, dda, q1, q2):
        _lib.check(self.lib.cg_sim_kick_coeffs(self.h, dda, q1, q2), "cg_sim_kick_coeffs")

    def drift_coeffs(self, dyyy, da1, da2):
        _lib.check(self.lib.cg_sim_drift_coeffs(self.h, dyyy, da1, da2), "cg_sim_drift_coeffs")

    def snapshot(self, aout, omega_m=None):
        n = self.lib.cg_sim_np(self.h)
        out = np.zeros(n, dtype=PARTICLE_MIN_DTYPE)
        om = self.omega_m if omega_m is None else omega_m
        _lib.check(self.lib.cg_sim_snapshot(self.h, aout, om, out.ctypes.data), "cg_sim_snapshot")
        return out

    def write_gadget(self, filename, aout, h=0.7, use_long_id=False, omega_m=None):
        """The snapshot at aout written as a GADGET-1 file straight from the
        device (cg_sim_write_gadget)."""
        om = self.omega_m if omega_m is None else omega_m
        _lib.check(self.lib.cg_sim_write_gadget(self.h, aout, om, h, str(filename).encode(),
                                                int(bool(use_long_id))), "cg_sim_write_gadget")

    def set_force_kernel(self, gradient=0, laplacian=0, deconvolve=0):
        """Green-step options: gradient 0 (spectral, the reference), 2 or 4
        (central differences); laplacian 0 (exact) or 1 (discrete);
        deconvolve 0, 1 or 2 (times the CIC window)."""
        _lib.check(self.lib.cg_sim_set_force_kernel(self.h, gradient, laplacian, deconvolve),
                   "force kernel")

    def set_force_filters(self, knots):
        """Force transfer functions T(|n|): an (nsets, n) array of knots,
        equally spaced from 0 to sqrt(3) ngrid / 2; set 0 becomes current.
        None removes them."""
        if knots is None:
            _lib.check(self.lib.cg_sim_set_force_filters(self.h, None, 0, 0), "force filters")
            return
        k = np.ascontiguousarray(np.atleast_2d(knots), dtype=np.float32)
        _lib.check(self.lib.cg_sim_set_force_filters(self.h, k.ctypes.data, k.shape[1],
                                                     k.shape[0]), "force filters")

    def use_force_filter(self, i):
        """Apply set i in the following force evaluations (-1: none)."""
        _lib.check(self.lib.cg_sim_use_force_filter(self.h, int(i)), "use force filter")

    def set_sort_interval(self, every):
        """Sort the particles into cell order at every `every`-th move (0:
        never); outputs keep the order the particles were given in."""
        _lib.check(self.lib.cg_sim_set_sort_interval(self.h, int(every)),
                   "cg_sim_set_sort_interval")

    def sync(self):
        _lib.check(self.lib.cg_sim_sync(self.h), "cg_sim_sync")

    def run(self, sched, zout=(0.0,), check_density=False):
        """The reference time loop; returns the list of snapshots."""
        snaps = []
        aout = output_scale_factors(zout)
        run_time_loop(sched, aout, move=self.move,
                      force=lambda: self.forces(check_density),
                      kick=self.kick, drift=self.drift,
                      snapshot=lambda a, i: snaps.append((a, self.snapshot(a))),
                      kick_drift=self.kick_drift)
        return snaps


def kick_coeffs(omega_m, a_v, a_x, avel1):
    lib = _lib.load()
    out = (ctypes.c_float * 3)()
    lib.cg_kick_coeffs(omega_m, a_v, a_x, avel1, out)
    return np.float32(out[0]), np.float32(out[1]), np.float32(out[2])


def drift_coeffs(omega_m, a_x, a_v, apos1):
    lib = _lib.load()
    out = (ctypes.c_float * 3)()
    lib.cg_drift_coeffs(omega_m, a_x, a_v, apos1, out)
    return np.float32(out[0]), np.float32(out[1]), np.float32(out[2])


def fft_r2c(real):
    """Device r2c of a host (n,n,n) float32 array -> (n,n,n/2+1) complex64."""
    lib = _lib.load()
    n = real.shape[0]
    a = np.ascontiguousarray(real, dtype=np.float32)
    out = np.zeros((n, n, n // 2 + 1), dtype=np.complex64)
    _lib.check(lib.cg_fft_r2c(n, a.ctypes.data, out.ctypes.data), "cg_fft_r2c")
    return out


def fft_c2r(spec):
    lib = _lib.load()
    n = spec.shape[0]
    a = np.ascontiguousarray(spec, dtype=np.complex64)
    out = np.zeros((n, n, n), dtype=np.float32)
    _lib.check(lib.cg_fft_c2r(n, a.ctypes.data, out.ctypes.data), "cg_fft_c2r")
    return out
