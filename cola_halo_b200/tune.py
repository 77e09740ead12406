"""Run-level tuning of a realization's schedule choices that depend on the
particles, not only on the mesh size (no reference counterpart).

The FFT pass variants are tuned per mesh size on an empty plan
(``cg_autotune``).  Two choices depend on how clustered the particles are,
so they are tuned on a running realization:

* the deposit shape (particles per CTA and shared-memory box,
  ``cg_sim_tune_deposit``), timed on the particles of a partly evolved
  realization;
* the cell-order sort interval (``cg_sim_set_sort_interval``), which trades
  the sort's cost against the locality it gives the deposit and the
  interpolation over a whole realization.
"""
import ctypes
import json
import os

import numpy as np

from . import _lib


def _cache_get(cache, key):
    """A choice stored by an earlier run in the JSON file `cache` (or None)."""
    if not cache or not os.path.exists(cache):
        return None
    with open(cache) as f:
        return json.load(f).get(key)


def _cache_put(cache, key, value):
    if not cache:
        return
    d = {}
    if os.path.exists(cache):
        with open(cache) as f:
            d = json.load(f)
    d[key] = value
    with open(cache, "w") as f:
        json.dump(d, f)


def _device_ms(lib, fn, max_marks):
    """Device time of the library's kernels queued by fn() (event profile)."""
    lib.cg_prof_begin(max_marks)
    fn()
    ms = (ctypes.c_double * _lib.NSTAGES)()
    cnt = (ctypes.c_int * _lib.NSTAGES)()
    lib.cg_prof_end(ms, cnt, _lib.NSTAGES)
    return float(np.sum(np.frombuffer(ms, dtype=np.float64)))


def tune_deposit(sim, cache=None):
    """Time every deposit shape on sim's current particles; installs the
    fastest for sim's mesh size.  Returns (variant, ms per variant).  With
    `cache` (a JSON file), a choice stored there by an earlier run for this
    mesh size is installed without timing, and a new one is stored."""
    lib = sim.lib
    key = "deposit_%d" % sim.ngrid
    got = _cache_get(cache, key)
    if got is not None:
        _lib.check(lib.cg_set_deposit_variant(sim.ngrid, int(got)), "cg_set_deposit_variant")
        return int(got), []
    nv = lib.cg_deposit_variants()
    ms = (ctypes.c_float * nv)()
    best = lib.cg_sim_tune_deposit(sim.h, ms)
    if best < 0:
        raise RuntimeError("cg_sim_tune_deposit: %s" % lib.cg_last_error().decode())
    _cache_put(cache, key, best)
    return best, [float(t) for t in ms]


def tune_sort_interval(sim, reset, sched, candidates=(0, 2, 3, 4, 6, 8, 10), reps=3,
                       cache=None, margin=0.01):
    """Run whole realizations per candidate sort interval and keep the
    fastest.  reset() puts the initial particles back; sched is the
    realization's Schedule.  Steps are move, force, fused kick + drift (the
    loop of main.c:162-206 without outputs).  Each candidate is timed as
    the best of `reps` realizations (the differences between intervals are
    a few per cent, close to the spread of single runs).  The library's
    default interval for this particle count (every sixth move from 2^23
    particles, else never) is kept unless another candidate is faster by
    more than `margin`.  Returns (interval, ms per candidate); the choice is
    installed on sim.  `cache` as for tune_deposit (keyed by particle count
    and mesh size)."""
    lib = sim.lib
    nsteps = sched.nloop - 1
    times = {}
    key = "sort_%d_%d" % (sim.nc, sim.ngrid)
    got = _cache_get(cache, key)
    if got is not None:
        sim.set_sort_interval(int(got))
        reset()
        return int(got), times

    def realization():
        for j in range(nsteps):
            _, _, avel1, apos1 = sched.times(j + 1)
            sim.move()
            sim.forces()
            sim.kick_drift(avel1, apos1)

    for every in candidates:
        sim.set_sort_interval(every)
        reset()
        realization()           # warm: first use allocates the sort's scratch
        best = None
        for _ in range(reps):
            reset()
            t = _device_ms(lib, realization, 64 * nsteps)
            best = t if best is None else min(best, t)
        times[every] = best
    default = 6 if sim.nc ** 3 >= (1 << 23) else 0
    best = min(times, key=times.get)
    if default in times and times[best] > (1.0 - margin) * times[default]:
        best = default
    sim.set_sort_interval(best)
    reset()
    _cache_put(cache, key, best)
    return best, times
