"""GADGET-1 snapshot files (cg_write_gadget in colagpu.h; the reference's
write.c) and a reader for them."""
import numpy as np

from . import _lib
from .types import PARTICLE_MIN_DTYPE

# gadget_file.h:4-24 as a numpy record (no padding: every field is aligned)
HEADER_DTYPE = np.dtype([
    ("np", "<i4", 6), ("mass", "<f8", 6), ("time", "<f8"), ("redshift", "<f8"),
    ("flag_sfr", "<i4"), ("flag_feedback", "<i4"), ("np_total", "<u4", 6),
    ("flag_cooling", "<i4"), ("num_files", "<i4"), ("boxsize", "<f8"), ("omega0", "<f8"),
    ("omega_lambda", "<f8"), ("hubble_param", "<f8"), ("flag_stellarage", "<i4"),
    ("flag_metals", "<i4"), ("np_total_highword", "<u4", 6),
    ("flag_entropy_instead_u", "<i4"), ("fill", "V60")])
assert HEADER_DTYPE.itemsize == 256


def write_gadget(filename, particles, a, boxsize, omega_m, h, use_long_id=False, np_count=None,
                 np_total=None, num_files=1):
    """Write ParticleMinimum particles -- a host structured array
    (PARTICLE_MIN_DTYPE) or a device address with `np_count` particles --
    as a GADGET-1 file."""
    lib = _lib.load()
    if isinstance(particles, int):
        ptr, n = particles, int(np_count)
    else:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_MIN_DTYPE)
        ptr, n = arr.ctypes.data, len(arr)
    _lib.check(lib.cg_write_gadget(str(filename).encode(), ptr, n,
                                   n if np_total is None else int(np_total), num_files, a,
                                   boxsize, omega_m, h, int(bool(use_long_id))),
               "cg_write_gadget")


def read_gadget(path):
    """(header record, pos[n, 3], vel[n, 3], ids[n]) of a GADGET-1 file; the
    id width (4 or 8 bytes) follows from its record length."""
    raw = open(path, "rb").read()
    off = 0

    def record():
        nonlocal off
        n0 = int(np.frombuffer(raw, "<i4", 1, off)[0])
        size = n0 & 0xFFFFFFFF
        body = raw[off + 4: off + 4 + size]
        n1 = int(np.frombuffer(raw, "<i4", 1, off + 4 + size)[0])
        if n1 != n0 or len(body) != size:
            raise ValueError("%s: bad record framing at byte %d" % (path, off))
        off += 8 + size
        return body
    hdr = np.frombuffer(record(), HEADER_DTYPE, 1)[0]
    n = int(hdr["np"][1])
    pos = np.frombuffer(record(), "<f4").reshape(n, 3)
    vel = np.frombuffer(record(), "<f4").reshape(n, 3)
    idb = record()
    ids = np.frombuffer(idb, "<u8" if n and len(idb) == 8 * n else "<u4")
    return hdr, pos, vel, ids
