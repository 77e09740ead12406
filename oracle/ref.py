"""ctypes binding of oracle/_ref/libcolaref.so -- TEST INFRASTRUCTURE.

The library is the reference's own C code (unchanged) linked against the
project's shims; see oracle/Makefile.  The functions bound here are the
reference's public hot-path entry points (pm.h:6-11, cola.h:7-18,
lpt.h:6-8, power.h:4-6, move.h:7, comm.h:8, msg.h:4-9, timer.h:4-10) and the
friends-of-friends halo finder (fof.h:6-10).
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcolaref.so")

_lib = None


def build(ref_dir=None):
    """Compile the reference from its sources in ref_dir (default: the
    COLA_REF_DIR environment variable).  Without the sources (GPU hosts) the
    prebuilt library is used if present."""
    ref_dir = ref_dir or os.environ.get("COLA_REF_DIR")
    if not ref_dir or not os.path.isdir(ref_dir):
        return os.path.exists(LIB_PATH)
    subprocess.run(["make", "-s", "-C", HERE, "REF=" + ref_dir], check=True)
    return True


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    f, d, i = ctypes.c_float, ctypes.c_double, ctypes.c_int
    sz = ctypes.c_size_t
    sig = {
        "msg_init": (None, []),
        "msg_set_loglevel": (None, [i]),
        "timer_set_category": (None, [i]),
        "timer_print": (None, []),
        "comm_init": (None, [i, i, f]),
        "power_init": (None, [ctypes.c_char_p, d, d, d, d]),
        "PowerSpec": (d, [d]),
        "GrowthFactor": (d, [d, d]),
        "lpt_init": (None, [i, P, sz]),
        "lpt_set_displacement": (i, [d, d, i, d, P]),
        "lpt_get_local_nx": (i, []),
        "pm_init": (None, [i, i, f, f, P, sz, P, sz]),
        "pm_calculate_forces": (None, [P]),
        "cola_kick": (None, [P, f, f]),
        "cola_drift": (None, [P, f, f]),
        "cola_set_snapshot": (None, [d, P, P]),
        "move_particles2": (None, [P, f, P, sz]),
        "fof_calc_memory": (sz, [i, i]),
        "fof_init": (None, [i, i, P, sz]),
        "fof_find_halos": (None, [P, f]),
        "fof_write_halos": (None, [ctypes.c_char_p]),
        "coarse_grid2": (None, [ctypes.c_char_p, P, i, P, sz]),
        "write_snapshot": (None, [ctypes.c_char_p, P, i]),
        "growthD": (f, [f]),
        "growthD2": (f, [f]),
        "Sq": (d, [d, d, d]),
        "Sphi": (d, [d, d, d]),
        "Qfactor": (f, [f]),
        "gsl_rng_alloc": (P, [P]),
        "gsl_rng_set": (None, [P, ctypes.c_ulong]),
        "gsl_rng_uniform": (d, [P]),
        "gsl_rng_free": (None, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib.msg_init()
    lib.msg_set_loglevel(7)          # silent
    lib.timer_set_category(0)
    _lib = lib
    return lib


def ranlxd1_stream(seed, n):
    """First n draws of the shim's gsl_rng_ranlxd1 after gsl_rng_set(seed)."""
    lib = load()
    rtype = ctypes.c_void_p.in_dll(lib, "gsl_rng_ranlxd1")
    r = lib.gsl_rng_alloc(rtype)
    lib.gsl_rng_set(r, seed)
    out = [lib.gsl_rng_uniform(r) for _ in range(n)]
    lib.gsl_rng_free(r)
    return out


def set_cola_omega(omega_m):
    """cola.c keeps Omega_m in a file-static (cola.c:58) that cola_kick sets;
    the growth functions read it.  Kick zero particles to set it."""
    from cola_halo_b200.types import Particles
    lib = load()
    p = Particles()
    p.np_local = 0
    p.a_x = 0.5
    p.a_v = 0.5
    lib.cola_kick(ctypes.byref(p), omega_m, 0.5)


def fof_catalog(pmin, boxsize, nc, ll, workdir):
    """Halos of ParticleMinimum array `pmin` by the reference's own
    fof_find_halos + fof_write_halos (fof.c:1035-1181, one rank), read back
    from the text file it writes: an array of (nfof, x[3], v[3]) rows in
    the file's order.  `pmin` is not modified."""
    import numpy as np
    from cola_halo_b200.types import HostSnapshot
    lib = load()
    n = len(pmin)
    lib.comm_init(nc, nc, boxsize)
    np_alloc = int(1.25 * n) + 16
    size = lib.fof_calc_memory(np_alloc, nc)
    mem = np.zeros(size + 64, dtype=np.uint8)
    lib.fof_init(np_alloc, nc, mem.ctypes.data, size)
    snap = HostSnapshot(nc, np_alloc, boxsize, 0.3)
    snap.p[:n] = pmin
    snap.struct.np_local = n
    lib.fof_find_halos(snap.ptr, ll)
    path = os.path.join(workdir, "fof_ref.txt")
    lib.fof_write_halos(path.encode())
    rows = np.loadtxt(path, ndmin=2) if os.path.getsize(path) else np.zeros((0, 7))
    return rows


def read_grid_file(path):
    """(boxsize, delta[nc, nc, nc]) of a coarse-grid file (coarse_grid.c:46-91:
    float boxsize, int nc, nc^3 float delta with x slowest, int nc)."""
    import numpy as np
    raw = open(path, "rb").read()
    L = np.frombuffer(raw, np.float32, 1, 0)[0]
    nc = int(np.frombuffer(raw, np.int32, 1, 4)[0])
    ng = nc * nc * nc
    assert len(raw) == 12 + 4 * ng, "coarse grid file size"
    assert int(np.frombuffer(raw, np.int32, 1, 8 + 4 * ng)[0]) == nc, "coarse grid trailer"
    return L, np.frombuffer(raw, np.float32, ng, 8).reshape(nc, nc, nc).copy()


def coarse_grid_file(pmin, boxsize, nc, path, np_total=None):
    """The reference's coarse_grid2 (coarse_grid.c:17-93, one rank) on
    ParticleMinimum array `pmin`, written to `path`; returns read_grid_file."""
    import numpy as np
    from cola_halo_b200.types import HostSnapshot
    lib = load()
    n = len(pmin)
    lib.comm_init(max(nc, 1), max(nc, 1), boxsize)
    snap = HostSnapshot(nc, max(n, 1), boxsize, 0.3)
    snap.p[:n] = pmin
    snap.struct.np_local = n
    snap.struct.np_total = n if np_total is None else np_total
    size = 4 * nc * nc * (nc + 16)
    mem = np.zeros(size // 4 + 16, dtype=np.float32)
    lib.coarse_grid2(path.encode(), snap.ptr, nc, mem.ctypes.data, size)
    return read_grid_file(path)


def gadget_file(pmin, boxsize, omega_m, h, a, filebase, use_long_id=0):
    """The bytes of the reference's write_snapshot (write.c:14-107, one rank)
    for ParticleMinimum array `pmin`: it writes "<filebase>.0"."""
    from cola_halo_b200.types import HostSnapshot
    lib = load()
    n = len(pmin)
    lib.comm_init(16, 16, boxsize)
    snap = HostSnapshot(16, max(n, 1), boxsize, omega_m, h=h)
    snap.p[:n] = pmin
    snap.struct.np_local = n
    snap.struct.a = a
    lib.write_snapshot(filebase.encode(), snap.ptr, int(use_long_id))
    with open(filebase + ".0", "rb") as f:
        return f.read()
