"""ctypes / numpy mirrors of the reference's particle data types.

Byte-for-byte the structs of ``particle.h:6-48`` in cola_halo, so that one
process can hand the same ``Particles`` / ``Snapshot`` to the reference's C
entry points and to this library's drop-in C-ABI:

* ``Particle``  {float x[3], dx1[3], dx2[3], v[3]; long long id}   56 bytes
* ``Particles`` {Particle* p; float3* force; float a_x, a_v;
                 int np_local, np_allocated; long long np_total;
                 float np_average}
* ``ParticleMinimum`` {float x[3], v[3]; long long id}               32 bytes
* ``Snapshot``  {ParticleMinimum* p; int np_local, np_allocated;
                 long long np_total; float np_average, a, boxsize; int nc;
                 float omega_m, h; int seed; char* filename}
"""
import ctypes

import numpy as np

PARTICLE_DTYPE = np.dtype(
    [("x", "<f4", 3), ("dx1", "<f4", 3), ("dx2", "<f4", 3), ("v", "<f4", 3),
     ("id", "<i8")], align=True)
assert PARTICLE_DTYPE.itemsize == 56

PARTICLE_MIN_DTYPE = np.dtype(
    [("x", "<f4", 3), ("v", "<f4", 3), ("id", "<i8")], align=True)
assert PARTICLE_MIN_DTYPE.itemsize == 32


class Particles(ctypes.Structure):
    _fields_ = [("p", ctypes.c_void_p), ("force", ctypes.c_void_p),
                ("a_x", ctypes.c_float), ("a_v", ctypes.c_float),
                ("np_local", ctypes.c_int), ("np_allocated", ctypes.c_int),
                ("np_total", ctypes.c_longlong), ("np_average", ctypes.c_float)]


class Snapshot(ctypes.Structure):
    _fields_ = [("p", ctypes.c_void_p), ("np_local", ctypes.c_int),
                ("np_allocated", ctypes.c_int), ("np_total", ctypes.c_longlong),
                ("np_average", ctypes.c_float), ("a", ctypes.c_float),
                ("boxsize", ctypes.c_float), ("nc", ctypes.c_int),
                ("omega_m", ctypes.c_float), ("h", ctypes.c_float),
                ("seed", ctypes.c_int), ("filename", ctypes.c_char_p)]


class HostParticles:
    """Host-side particle storage laid out exactly as ``mem.c:11-39``
    (``allocate_particles``): an AoS ``Particle`` array and a separate
    ``float3`` force array, ``np_alloc_factor`` slack for buffer particles."""

    def __init__(self, nc, np_alloc_factor=1.25, nnode=1):
        npl = nc * nc * nc
        np_alloc = int(np_alloc_factor * nc * nc * (nc + 1))
        self.nc = nc
        self.p = np.zeros(np_alloc, dtype=PARTICLE_DTYPE)
        self.force = np.zeros((np_alloc, 3), dtype=np.float32)
        self.struct = Particles()
        self.struct.p = self.p.ctypes.data
        self.struct.force = self.force.ctypes.data
        self.struct.np_allocated = np_alloc
        self.struct.np_total = npl
        self.struct.np_average = float(npl) / nnode
        self.struct.np_local = 0

    @property
    def ptr(self):
        return ctypes.byref(self.struct)

    @property
    def np_local(self):
        return self.struct.np_local

    def local(self):
        return self.p[: self.struct.np_local]


class HostSnapshot:
    """``Snapshot`` plus its ``ParticleMinimum`` array (``mem.c:41-53``)."""

    def __init__(self, nc, np_alloc, boxsize, omega_m, h=0.705, seed=0):
        self.p = np.zeros(np_alloc, dtype=PARTICLE_MIN_DTYPE)
        self.struct = Snapshot()
        self.struct.p = self.p.ctypes.data
        self.struct.np_allocated = np_alloc
        self.struct.np_total = nc * nc * nc
        self.struct.nc = nc
        self.struct.boxsize = boxsize
        self.struct.omega_m = omega_m
        self.struct.h = h
        self.struct.seed = seed
        self.struct.a = 0.0

    @property
    def ptr(self):
        return ctypes.byref(self.struct)

    def local(self):
        return self.p[: self.struct.np_local]
