"""Coarse density grid of a snapshot (cg_coarse_grid in colagpu.h; the
reference's coarse_grid.c)."""
import ctypes

import numpy as np

from . import _lib
from .types import PARTICLE_MIN_DTYPE


def coarse_grid(particles, boxsize, nc, np_total=None, np_count=None, out=None):
    """CIC density contrast delta[nc, nc, nc] ([x][y][z], float32) of
    reference ParticleMinimum particles: a host structured array
    (PARTICLE_MIN_DTYPE) or a device address with `np_count` particles.
    `np_total` (default: the particle count) sets the mean density.  `out`
    may be a device address of nc^3 floats, which then receives the grid
    (the return value is then None).  Returns (delta, mass sum)."""
    lib = _lib.load()
    if isinstance(particles, int):
        ptr, n = particles, int(np_count)
    else:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_MIN_DTYPE)
        ptr, n = arr.ctypes.data, len(arr)
    total = ctypes.c_double()
    if out is None:
        delta = np.empty((nc, nc, nc), dtype=np.float32)
        dst = delta.ctypes.data
    else:
        delta, dst = None, int(out)
    _lib.check(lib.cg_coarse_grid(ptr, n, n if np_total is None else int(np_total), boxsize, nc,
                                  dst, ctypes.byref(total)), "cg_coarse_grid")
    return delta, total.value


def read_grid_file(path):
    """(boxsize, delta[nc, nc, nc]) of a coarse-grid file written by
    coarse_grid2: float boxsize, int nc, nc^3 float delta (x slowest), int nc
    (coarse_grid.c:46-91)."""
    raw = open(path, "rb").read()
    L = float(np.frombuffer(raw, np.float32, 1, 0)[0])
    nc = int(np.frombuffer(raw, np.int32, 1, 4)[0])
    ng = nc * nc * nc
    if len(raw) != 12 + 4 * ng or int(np.frombuffer(raw, np.int32, 1, 8 + 4 * ng)[0]) != nc:
        raise ValueError("%s: not a coarse-grid file" % path)
    return L, np.frombuffer(raw, np.float32, ng, 8).reshape(nc, nc, nc).copy()
