"""Batched realizations in one CUDA graph launch (cg_batch_* in colagpu.h)."""
import ctypes

import numpy as np

from . import _lib
from .types import PARTICLE_DTYPE, PARTICLE_MIN_DTYPE


class RealizationSpec(ctypes.Structure):
    _fields_ = [("nc", ctypes.c_int), ("ngrid", ctypes.c_int), ("boxsize", ctypes.c_float),
                ("a_init", ctypes.c_double), ("a_final", ctypes.c_double),
                ("nsteps", ctypes.c_int), ("aout", ctypes.c_float)]


class Batch:
    def __init__(self, specs, omega_m, nstreams=4):
        self.lib = _lib.load()
        self.specs = list(specs)
        arr = (RealizationSpec * len(self.specs))()
        for i, s in enumerate(self.specs):
            arr[i] = RealizationSpec(s["nc"], s["ngrid"], s["boxsize"], s["a_init"],
                                     s.get("a_final", 1.0), s["nsteps"], s.get("aout", 1.0))
        h = ctypes.c_void_p()
        _lib.check(self.lib.cg_batch_create(ctypes.byref(h), len(self.specs), arr, omega_m,
                                            nstreams), "cg_batch_create")
        self.h = h

    def set_particles(self, i, particles):
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        _lib.check(self.lib.cg_batch_set_particles(self.h, i, p.ctypes.data, len(p)),
                   "cg_batch_set_particles")

    def set_sort_interval(self, every):
        """Cell-order sort at every `every`-th move inside the graph (0:
        never); before the first run."""
        _lib.check(self.lib.cg_batch_set_sort_interval(self.h, int(every)),
                   "cg_batch_set_sort_interval")

    def run(self):
        _lib.check(self.lib.cg_batch_run(self.h), "cg_batch_run")

    def snapshot(self, i):
        n = self.specs[i]["nc"] ** 3
        out = np.zeros(n, dtype=PARTICLE_MIN_DTYPE)
        _lib.check(self.lib.cg_batch_get_snapshot(self.h, i, out.ctypes.data), "snapshot")
        return out

    def power_spectrum(self, i):
        nb = self.specs[i]["ngrid"] // 2
        k, p, m = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        _lib.check(self.lib.cg_batch_power_spectrum(self.h, i, k.ctypes.data, p.ctypes.data,
                                                    m.ctypes.data), "power_spectrum")
        return k, p, m

    def last_ms(self):
        """Device time of the last run (CUDA events around the graph launch)."""
        t = ctypes.c_float()
        _lib.check(self.lib.cg_batch_last_ms(self.h, ctypes.byref(t)), "last_ms")
        return t.value

    def num_nodes(self):
        n = ctypes.c_size_t()
        _lib.check(self.lib.cg_batch_num_nodes(self.h, ctypes.byref(n)), "num_nodes")
        return n.value

    def close(self):
        if self.h:
            self.lib.cg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
