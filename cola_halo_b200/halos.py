"""Friends-of-friends halos (cg_fof in colagpu.h; the reference's fof.c)."""
import ctypes

import numpy as np

from . import _lib
from .types import PARTICLE_MIN_DTYPE

HALO_DTYPE = np.dtype([("nfof", np.int32), ("x", np.float32, 3), ("v", np.float32, 3)])


def fof(particles, boxsize, ll, nfof_min=32, np_count=None):
    """Halos of reference ParticleMinimum particles: a host structured array
    (PARTICLE_MIN_DTYPE) or a device address with `np_count` particles.
    Returns a HALO_DTYPE array in the order of each group's smallest
    particle index."""
    lib = _lib.load()
    if isinstance(particles, int):
        ptr, n = particles, int(np_count)
    else:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_MIN_DTYPE)
        ptr, n = arr.ctypes.data, len(arr)
    cap = n // max(nfof_min, 1) + 1
    out = np.zeros(cap, dtype=HALO_DTYPE)
    nh = ctypes.c_longlong()
    _lib.check(lib.cg_fof(ptr, n, boxsize, ll, nfof_min, out.ctypes.data, cap, ctypes.byref(nh)),
               "cg_fof")
    return out[: nh.value].copy()


def mass_function(nfof, particle_mass, edges):
    """Halo counts in log10-mass bins (edges in log10 of the mass unit)."""
    m = np.log10(np.asarray(nfof, dtype=np.float64) * particle_mass)
    return np.histogram(m, bins=edges)[0]
