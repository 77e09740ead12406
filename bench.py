#!/usr/bin/env python
"""Throughput benchmark of the COLA step: particle-steps/s.

Workload (default): 256^3 particles, 768^3 PM mesh (factor 3), box
600 Mpc/h, BBKS no-wiggle P(k) (Omega_m 0.273, h 0.705, n_s 0.96,
sigma_8 0.81), 2LPT at z = 49, 10 COLA steps linear in a to z = 0.  Inputs
are seeded synthetic initial conditions (no dataset is involved).

A "step" is one COLA time step: periodic wrap, PM force (deposit, r2c,
Green/gradient, three c2r, interpolation), kick, drift.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  Under torchrun each rank runs its own
realization (seed + rank) on its own GPU: realizations are independent, so
the N-GPU number is weak-scaled replicas with no collective on the data path.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import shutil
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CONFIGS = {
    # 1 x B200 plain COLA run
    "c2": dict(nc=256, factor=3, L=600.0, om=0.273, a_init=0.02, nsteps=10, seed=100),
    # the CPU-runnable case
    "c1": dict(nc=64, factor=3, L=200.0, om=0.273, a_init=0.02, nsteps=10, seed=100),
    # one realization of the batched config (128^3, 384^3 mesh)
    "c3": dict(nc=128, factor=3, L=300.0, om=0.273, a_init=0.02, nsteps=10, seed=100),
    # the large single-GPU case: 512^3 particles on a 1024^3 mesh (factor 2),
    # the same mean particle spacing as c2
    "c5": dict(nc=512, factor=2, L=1200.0, om=0.273, a_init=0.02, nsteps=10, seed=100),
}

METRIC = "particle-steps/s"
HBM_FALLBACK_GBS = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


# ----------------------------------------------------------------- CUDA events
class Cudart:
    def __init__(self):
        for name in ("libcudart.so.12", "libcudart.so"):
            try:
                self.lib = ctypes.CDLL(name)
                break
            except OSError:
                continue
        else:
            self.lib = ctypes.CDLL("/usr/local/cuda/lib64/libcudart.so")
        L = self.lib
        L.cudaEventCreate.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
        L.cudaEventRecord.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.cudaEventSynchronize.argtypes = [ctypes.c_void_p]
        L.cudaEventElapsedTime.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_void_p,
                                           ctypes.c_void_p]
        L.cudaStreamSynchronize.argtypes = [ctypes.c_void_p]

    def event(self):
        e = ctypes.c_void_p()
        assert self.lib.cudaEventCreate(ctypes.byref(e)) == 0
        return e

    def record(self, ev, stream):
        assert self.lib.cudaEventRecord(ev, stream) == 0

    def elapsed_ms(self, a, b):
        assert self.lib.cudaEventSynchronize(b) == 0
        t = ctypes.c_float()
        assert self.lib.cudaEventElapsedTime(ctypes.byref(t), a, b) == 0
        return float(t.value)

    def sync_device(self):
        self.lib.cudaDeviceSynchronize()

    def device_copy_of(self, host_array):
        """A device buffer holding a copy of a contiguous host array."""
        p = ctypes.c_void_p()
        self.lib.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
        self.lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.c_int]
        assert self.lib.cudaMalloc(ctypes.byref(p), host_array.nbytes) == 0
        assert self.lib.cudaMemcpy(p, host_array.ctypes.data, host_array.nbytes, 1) == 0
        return p


# --------------------------------------------------------------- clock sampler
class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.lines = []
        self.n0 = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-i", str(self.dev), "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: let its first sample arrive
            # before the timed region opens, and keep only later samples
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0:
                time.sleep(0.01)
            self.n0 = len(self.lines)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        # a region shorter than the sampling period: take the sample that
        # follows its end
        t0 = time.time()
        while len(self.lines) <= self.n0 and time.time() - t0 < 0.5:
            time.sleep(0.005)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.n0:] or self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ helpers
def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def algorithmic_bytes(stage, N, npart, reset=True):
    """Algorithmic bytes per launch of each stage (each tensor counted once):
    the deposit reads the positions and writes the mesh once; the z r2c reads
    the mesh, writes the half spectrum and (reset) writes -1 back over the
    mesh for the next deposit."""
    Mr = 4.0 * N ** 3
    Ms = 8.0 * (N // 2 + 1) * N * N
    return {
        "fill": Mr,
        "deposit": 12.0 * npart + Mr,
        "fz_r2c": Mr + Ms + (Mr if reset else 0.0),
        "fx_fwd": 2 * Ms,
        "green_y": 3 * Ms,
        "fx_inv": 2 * Ms,
        "zi_c2r": Ms + Mr,
        "interp": 12.0 * npart + 3 * Mr + 12.0 * npart,
        "wrap": 24.0 * npart,
        "kick": 60.0 * npart,
        "drift": 60.0 * npart,
        "kick_drift": 84.0 * npart,
    }.get(stage)


def load_traffic():
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def _ref_cola_timers(lib):
    """The reference's own timer breakdown of the COLA category (timer.c:62-83,
    timer_print), read from what timer_print writes to stdout: seconds per
    subcategory (fft, assign, force_mesh, pforce, check, comm, evolve).  The
    timers accumulate over the process; callers difference two readings."""
    import re
    fd, path = tempfile.mkstemp()
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(fd, 1)
        lib.msg_set_loglevel(3)          # info
        lib.timer_print()
        lib.msg_set_loglevel(7)          # silent again
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)
        os.close(fd)
    text = open(path).read()
    os.unlink(path)
    out, cat = {}, None
    for line in text.splitlines():
        m = re.match(r"^(\S+)\s+([0-9.]+)\s", line)
        if m:
            cat = m.group(1)
            if cat == "COLA":
                out["all"] = float(m.group(2))
            continue
        m = re.match(r"^\s+(\S+)\s+([0-9.]+)\s", line)
        if m and cat == "COLA":
            out[m.group(1)] = float(m.group(2))
    lib.timer_set_category(2)            # timer_print leaves the Init category; back to COLA
    return out


def cpu_reference_step_time(cfg, parts_aos, table, steps=1, warmup=0):
    """Time the reference's own CPU code (oracle/_ref: pm.c, cola.c, move.c
    built unchanged against the project's MPI/FFTW/GSL shims) for `steps`
    COLA steps of the schedule, starting from the initial particles, after
    `warmup` untimed steps that are then undone (the particles are put back
    to the initial conditions), so the timed steps are steps 1..`steps` of a
    realization, as the GPU arm's are.  parts_aos: initial particles
    (reference Particle layout), or None to generate them with the
    reference's own lpt.c.  Returns (seconds per step, cores, the reference's
    timer breakdown of the timed steps in seconds)."""
    from cola_halo_b200.schedule import Schedule
    from cola_halo_b200.types import HostParticles
    from oracle import ref
    lib = ref.load()
    nc, factor, L, om = cfg["nc"], cfg["factor"], cfg["L"], cfg["om"]
    sched = Schedule.linear(cfg["a_init"], 1.0, cfg["nsteps"])
    lib.power_init(table.encode(), sched.a_init, 0.81, om, 1 - om)
    lib.comm_init(nc * factor, nc, L)
    lib.pm_init(nc * factor, factor, L, 1.25, None, 0, None, 0)
    hp = HostParticles(nc)
    if parts_aos is None:
        lib.lpt_init(nc, None, 0)
        lib.lpt_set_displacement(sched.a_init, om, cfg["seed"], L, hp.ptr)
    else:
        hp.p[: nc ** 3] = parts_aos
        hp.struct.np_local = nc ** 3
        hp.struct.a_x = sched.a_init
    hp.struct.a_v = sched.a_init
    ics = hp.p[: nc ** 3].copy()
    lib.timer_set_category(2)            # COLA (timer.h)

    def one(i):
        _, _, avel1, apos1 = sched.times(i % (sched.nloop - 1) + 1)
        lib.move_particles2(hp.ptr, L, None, 0)
        lib.pm_calculate_forces(hp.ptr)
        lib.cola_kick(hp.ptr, om, avel1)
        lib.cola_drift(hp.ptr, om, apos1)
    for i in range(warmup):
        one(i)
    if warmup:
        hp.p[: nc ** 3] = ics
        hp.struct.np_local = nc ** 3
        hp.struct.a_x = sched.a_init
        hp.struct.a_v = sched.a_init
    t_before = _ref_cola_timers(lib)
    t0 = time.perf_counter()
    for i in range(steps):
        one(i)
    dt = (time.perf_counter() - t0) / steps
    t_after = _ref_cola_timers(lib)
    breakdown = {k: round(t_after[k] - t_before.get(k, 0.0), 3) for k in t_after}
    cores = len(os.sched_getaffinity(0))
    return dt, cores, breakdown


# --------------------------------------------------------------- reference arm
def run_reference(args, cfg):
    rank, world, local = dist_setup(args)
    if rank != 0:
        return 0
    from cola_halo_b200.bbks import write_bbks_table
    npart = cfg["nc"] ** 3
    base = {"metric": METRIC, "unit": "particle-steps/s", "impl": "reference",
            "higher_is_better": True, "n_gpus": args.gpus}
    try:
        from oracle import ref
        if not os.path.exists(ref.LIB_PATH):
            raise RuntimeError("oracle/_ref/libcolaref.so not built")
    except Exception as e:
        print(json.dumps(dict(base, unavailable="reference build missing: %s" % e)))
        return 0
    table = write_bbks_table(os.path.join(tempfile.mkdtemp(), "bbks.dat"))
    # one whole realization: the timed steps are steps 1..nsteps of the
    # schedule, the same step indices the GPU arm averages over
    nsteps = cfg["nsteps"]
    k_ref = max(1, min(args.steps, nsteps))
    w_ref = min(args.warmup, 1)
    dt, cores, timers = cpu_reference_step_time(cfg, None, table, steps=k_ref, warmup=w_ref)
    value = npart / dt
    fft_share = (timers.get("fft", 0.0) / timers["all"]) if timers.get("all") else None
    out = dict(base, value=value, n_gpus=args.gpus, steps=k_ref, warmup=w_ref,
               ms_per_step=dt * 1e3, scaling="weak", vs_baseline=None, dtype="f32",
               data="synthetic (seeded 2LPT initial conditions, BBKS P(k))",
               config=dict(workload=args.config_desc, particles=npart,
                           mesh=cfg["nc"] * cfg["factor"], boxsize=cfg["L"],
                           steps_timed="steps 1..%d of the %d-step schedule (z = 49 -> 0), "
                                       "from the 2LPT initial conditions" % (k_ref, nsteps),
                           parallelism="1 host, %d OpenMP threads" % cores),
               reference_timers_s=timers,
               reference_fft_share=fft_share,
               cpu_baseline={"value": value, "unit": "particle-steps/s", "cores": cores,
                             "kind": "reference",
                             "sample": "steps 1..%d of one realization of the %s workload "
                                       "after %d warm-up step (undone); the reference's FFT "
                                       "is the project's double-precision shim, not FFTW "
                                       "(its share of the step time: %s)"
                                       % (k_ref, args.config, w_ref,
                                          "%.0f%%" % (100 * fft_share) if fft_share else "n/a")},
               e2e={"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0})
    print(json.dumps(out))
    return 0


# -------------------------------------------------------------------- B200 arm
def run_b200(args, cfg):
    rank, world, local = dist_setup(args)
    dist = None
    if world > 1:
        import torch
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", device_id=torch.device("cuda", local),
                              timeout=__import__("datetime").timedelta(seconds=600))
        dist = td

    def barrier():
        if dist:
            dist.barrier()

    from cola_halo_b200 import replicas

    def allmax(v):
        return replicas.allmax(v, dist)

    from cola_halo_b200 import Simulation, _lib
    from cola_halo_b200.bbks import write_bbks_table
    from cola_halo_b200.schedule import Schedule
    from cola_halo_b200.types import PARTICLE_DTYPE, PARTICLE_MIN_DTYPE, Particles, Snapshot

    lib = _lib.load()
    _lib.check(lib.cg_set_device(local), "cg_set_device")
    cuda = Cudart()
    nc, factor, L, om = cfg["nc"], cfg["factor"], cfg["L"], cfg["om"]
    N = nc * factor
    npart = nc ** 3
    sched = Schedule.linear(cfg["a_init"], 1.0, cfg["nsteps"])
    seed = replicas.replica_seed(cfg["seed"], rank)
    table = write_bbks_table(os.path.join(tempfile.mkdtemp(), "bbks.dat"))

    # ---- 2LPT initial conditions on the GPU through the drop-in API,
    # into pinned host memory (reference Particle layout)
    nbytes = 56 * npart
    hp_ptr = lib.cg_host_alloc(nbytes)
    assert hp_ptr, "pinned host allocation failed"
    host_parts = np.ctypeslib.as_array((ctypes.c_uint8 * nbytes).from_address(hp_ptr)).view(
        PARTICLE_DTYPE)
    P = Particles()
    P.p = hp_ptr
    P.force = None
    P.np_allocated = npart
    P.np_total = npart
    P.np_average = float(npart)
    lib.cg_dropin_set_abort(0)
    lib.power_init(table.encode(), sched.a_init, 0.81, om, 1 - om)
    lib.lpt_init(nc, None, 0)
    t0 = time.perf_counter()
    rc = lib.lpt_set_displacement(sched.a_init, om, seed, L, ctypes.byref(P))
    lpt_s = time.perf_counter() - t0
    assert rc == 0, lib.cg_last_error()
    ics = host_parts.copy()

    # ---- FFT schedule for this mesh size (untimed; cached across runs when
    # COLAGPU_TUNE_CACHE names a file)
    ms_green = (ctypes.c_float * 8)(*([-1.0] * 8))
    ms_fx = (ctypes.c_float * 8)(*([-1.0] * 8))
    _lib.check(lib.cg_autotune(N, 0, ms_green, ms_fx), "cg_autotune")
    sg, sf = ctypes.c_int(), ctypes.c_int()
    _lib.check(lib.cg_get_schedule(N, ctypes.byref(sg), ctypes.byref(sf)), "cg_get_schedule")
    ng_v, nf_v = ctypes.c_int(), ctypes.c_int()
    lib.cg_schedule_variants(N, ctypes.byref(ng_v), ctypes.byref(nf_v))
    tuned_ms = {"green": [round(ms_green[v], 4) for v in range(ng_v.value) if ms_green[v] >= 0],
                "x": [round(ms_fx[v], 4) for v in range(nf_v.value) if ms_fx[v] >= 0]}

    # ---- device-resident step loop (value)
    sim = Simulation(nc, N, L, om)
    stream = lib.cg_sim_stream(sim.h)
    nsteps_run = sched.nloop - 1

    # the initial particles stay on the device: a realization restarts with a
    # device-to-device copy (56 B / particle), not a host upload
    d_ics = cuda.device_copy_of(ics)

    def reset():
        sim.set_particles_ptr(d_ics, npart, sched.a_init, sched.a_init)

    def step(i):
        j = i % nsteps_run
        if j == 0:
            reset()
        _, _, avel1, apos1 = sched.times(j + 1)
        sim.move()
        sim.forces()
        sim.kick_drift(avel1, apos1)

    for i in range(args.warmup):
        step(i)
    sim.sync()
    # the schedule choices that depend on the particles, tuned on this run:
    # the deposit shape on the warm-up's partly evolved particles, the sort
    # interval over whole realizations; then the warm-up again, so the timed
    # steps continue the schedule from the same point
    from cola_halo_b200.tune import tune_deposit, tune_sort_interval
    # COLAGPU_RUN_TUNE_CACHE=file keeps these choices for later runs, as
    # COLAGPU_TUNE_CACHE keeps the FFT schedule (a profiled rerun then
    # launches what the plain run chose)
    run_cache = os.environ.get("COLAGPU_RUN_TUNE_CACHE")
    dep_best, dep_ms = tune_deposit(sim, cache=run_cache)
    sort_best, sort_ms = tune_sort_interval(sim, reset, sched, cache=run_cache)
    os.environ["COLAGPU_SORT_EVERY"] = str(sort_best)      # the drop-in run below too
    for i in range(args.warmup):
        step(i)
    sim.sync()
    # one density check outside the timed region (pm.c:535-562)
    sim.move()
    dsum = sim.forces(check_density=True)
    ev0, ev1 = cuda.event(), cuda.event()
    clocks = Clocks(local)
    prof_n = lib.cg_prof_begin(64 * (args.steps + 1))
    barrier()
    sim.sync()
    clocks.start()
    launches0 = lib.cg_launch_count()
    cuda.record(ev0, stream)
    for i in range(args.steps):
        step(args.warmup + i)
    cuda.record(ev1, stream)
    launches = lib.cg_launch_count() - launches0
    # close the stage profile right behind ev1 (its end event follows ev1 on
    # the stream, so the last stage is not charged for host time)
    stage_ms = (ctypes.c_double * _lib.NSTAGES)()
    stage_n = (ctypes.c_int * _lib.NSTAGES)()
    lib.cg_prof_end(stage_ms, stage_n, _lib.NSTAGES)
    ms = cuda.elapsed_ms(ev0, ev1)
    clk = clocks.stop()
    sim.sync()
    barrier()
    ms_max = allmax(ms)
    value = replicas.whole_job_rate(npart, args.steps, ms_max, world)

    stages = {}
    for s in range(_lib.NSTAGES):
        if stage_n[s]:
            name = lib.cg_stage_name(s).decode()
            stages[name] = {"ms": stage_ms[s], "launches": stage_n[s]}
    # dominant kernel and its roofline
    hbm, peak_kind = peaks()
    dom = max(stages, key=lambda k: stages[k]["ms"])
    per_launch_ms = stages[dom]["ms"] / stages[dom]["launches"]
    ab = algorithmic_bytes(dom, N, npart)
    traffic = load_traffic().get("%s@%d" % (dom, N))
    roofline = {"kernel": dom, "bound": "hbm",
                "achieved": ab / (per_launch_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": ab / (per_launch_ms / 1e3) / 1e9 / hbm, "traffic": traffic,
                "algorithmic_bytes": ab, "peak_source": peak_kind}
    # the same figures for every stage with an algorithmic-byte count
    stage_roofline = {}
    for name, st in stages.items():
        b = algorithmic_bytes(name, N, npart)
        if b is None or not st["launches"]:
            continue
        t = st["ms"] / st["launches"] / 1e3
        stage_roofline[name] = {"ms_per_launch": round(t * 1e3, 4),
                                "gbs": round(b / t / 1e9, 1), "frac": round(b / t / 1e9 / hbm, 3)}
    roofline["stages"] = stage_roofline

    # ---- end to end through the drop-in C ABI with host buffers
    sim.close()
    snap_bytes = 32 * npart
    sp_ptr = lib.cg_host_alloc(snap_bytes)
    S = Snapshot()
    S.p = sp_ptr
    S.np_allocated = npart
    S.np_total = npart
    S.boxsize = L
    S.nc = nc
    S.omega_m = om
    lib.pm_init(N, factor, L, 1.25, None, 0, None, 0)
    runs = max(1, int(math.ceil(args.steps / float(sched.nloop))))

    # the pinned host Particle[] holds the initial conditions; the drop-in
    # layer never writes p[] back (the device copy is the working state), so
    # every realization below starts from the same host input
    host_parts[:] = ics

    def e2e_run():
        P.np_local = npart
        P.a_x = sched.a_init
        P.a_v = sched.a_init
        _lib.check(lib.cg_particles_upload(ctypes.byref(P)), "upload")
        from cola_halo_b200.schedule import run_time_loop
        run_time_loop(sched, [1.0],
                      move=lambda: lib.move_particles2(ctypes.byref(P), L, None, 0),
                      force=lambda: lib.pm_calculate_forces(ctypes.byref(P)),
                      kick=lambda a: lib.cola_kick(ctypes.byref(P), om, a),
                      drift=lambda a: lib.cola_drift(ctypes.byref(P), om, a),
                      snapshot=lambda a, i: lib.cola_set_snapshot(a, ctypes.byref(P),
                                                                  ctypes.byref(S)))
        err = lib.cg_last_error()
        if err:
            raise RuntimeError(err.decode())

    e2e_run()   # warm-up
    assert np.array_equal(host_parts["x"], ics["x"]), "the drop-in wrote the host particles"
    barrier()
    t0 = time.perf_counter()
    for _ in range(runs):
        e2e_run()
    e2e_s = allmax(time.perf_counter() - t0)
    e2e_value = world * npart * sched.nloop * runs / e2e_s
    snap = np.ctypeslib.as_array((ctypes.c_uint8 * snap_bytes).from_address(sp_ptr)).view(
        PARTICLE_MIN_DTYPE)
    assert np.isfinite(snap["x"]).all()
    lib.cg_dropin_finalize()

    # ---- CPU baseline: the reference's own code on this host, 1 step
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            dt, cores, timers = cpu_reference_step_time(cfg, ics, table, steps=2)
            cpu = {"value": npart / dt, "unit": "particle-steps/s", "cores": cores,
                   "kind": "reference",
                   "sample": "steps 1-2 of the %s workload's schedule (same 2LPT particles) "
                             "with the reference pm.c/cola.c/move.c; shim-FFT, not FFTW "
                             "(fft %.1f s of %.1f s)" % (args.config, timers.get("fft", 0.0),
                                                         timers.get("all", 0.0))}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": "particle-steps/s", "cores": None,
                   "kind": "reference", "sample": "unavailable: %s" % e}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 2LPT initial conditions, BBKS P(k))",
            "config": {"workload": args.config_desc, "particles": npart, "mesh": N,
                       "boxsize": L, "schedule": "10 COLA steps linear in a, z=49 -> 0",
                       "parallelism": "replicas x%d (one realization per GPU)" % world,
                       "l2": "inputs larger than L2 (%.2f GB per mesh)" % (4.0 * N ** 3 / 1e9),
                       "fft_schedule": {"green_variant": sg.value, "x_variant": sf.value,
                                        "chosen_by": "cg_autotune",
                                        "ms": tuned_ms},
                       "deposit_variant": {"chosen": dep_best,
                                           "ms": [round(t, 4) for t in dep_ms],
                                           "chosen_by": "cg_sim_tune_deposit"},
                       "sort_every": {"chosen": sort_best,
                                      "realization_ms": {str(k): round(v, 3)
                                                         for k, v in sort_ms.items()},
                                      "chosen_by": "tune_sort_interval"}},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": 56 * npart // sched.nloop,
                    "d2h_bytes_per_step": snap_bytes // sched.nloop,
                    "what": "whole realizations through the drop-in C ABI "
                            "(cg_particles_upload, then per step move_particles2, "
                            "pm_calculate_forces, cola_kick, cola_drift, and "
                            "cola_set_snapshot) from a pinned host Particle[] (56 B per "
                            "particle up) to a host Snapshot (32 B per particle down); "
                            "%d force evaluations per realization, bytes averaged per "
                            "step" % sched.nloop},
            "gpu_launches": int(launches),
            "gpu_launches_before_timed": int(launches0),
            "clocks": clk,
            "stages_ms": {k: round(v["ms"] / args.steps, 4) for k, v in stages.items()},
            "lpt_ms": lpt_s * 1e3,
            "density_sum": dsum,
        }
        print(json.dumps(out))
    lib.cg_host_free(sp_ptr)
    lib.cg_host_free(hp_ptr)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned", action="store_true",
                    help="second metric: learned coarse mesh vs plain factor-3 PM")
    ap.add_argument("--train-seeds", type=int, default=64)
    ap.add_argument("--eval-seeds", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--cufft", action="store_true",
                    help="the mesh r2c / c2r transforms beside cuFFT's at 384^3 and 768^3")
    ap.add_argument("--fof", action="store_true",
                    help="friends-of-friends halo finding on the z = 0 snapshot (b = 0.2)")
    ap.add_argument("--batch-streams", type=int, default=4,
                    help="streams the batch graph spreads its realizations over")
    ap.add_argument("--batch", action="store_true",
                    help="batched realizations: 32 x 128^3 particles / 384^3 meshes, uneven "
                         "boxes and step counts, one CUDA graph per run")
    ap.add_argument("--slab", action="store_true",
                    help="one realization split over the ranks by x slabs (cola_halo_b200.slab; "
                         "NCCL between the ranks of a torchrun job)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.learned and args.config == "c5":
        return run_learned_large(args)
    if args.learned:
        return run_learned(args)
    if args.batch:
        return run_batch(args)
    if args.fof:
        return run_fof(args)
    if args.cufft:
        return run_cufft(args)
    cfg = CONFIGS[args.config]
    args.config_desc = "%d^3 particles, %d^3 mesh, L=%g Mpc/h, BBKS, 2LPT z=49, 10 steps" % (
        cfg["nc"], cfg["nc"] * cfg["factor"], cfg["L"])
    if args.impl == "reference":
        return run_reference(args, cfg)
    if args.slab:
        return run_slab(args, cfg)
    return run_b200(args, cfg)


def run_slab(args, cfg):
    """One realization split over the job's ranks by x slabs of the mesh
    (the reference's MPI decomposition, cola_halo_b200.slab): per step the
    wrap, the particles' moves to their slabs, the slab-decomposed force and
    the kick + drift.  Strong scaling: the realization is the same for every
    N.  Device time from CUDA events around the steps, max over ranks."""
    rank, world, local = dist_setup(args)
    import torch
    from cola_halo_b200 import Simulation, _lib
    from cola_halo_b200.bbks import write_bbks_table
    from cola_halo_b200.schedule import Schedule
    from cola_halo_b200.slab import GpuRank, LocalComm, SlabPM, TorchComm
    from cola_halo_b200.types import PARTICLE_DTYPE, Particles
    lib = _lib.load()
    _lib.check(lib.cg_set_device(local), "cg_set_device")
    torch.cuda.set_device(local)
    td = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", device_id=torch.device("cuda", local),
                              timeout=datetime.timedelta(seconds=600))
    nc, factor, L, om = cfg["nc"], cfg["factor"], cfg["L"], cfg["om"]
    N, npart = nc * factor, nc ** 3
    sched = Schedule.linear(cfg["a_init"], 1.0, cfg["nsteps"])
    table = write_bbks_table(os.path.join(tempfile.mkdtemp(), "bbks.dat"))
    # the same 2LPT initial conditions on every rank (the GPU lpt of the
    # drop-in layer); each rank keeps the particles of its slab
    nbytes = 56 * npart
    hp = lib.cg_host_alloc(nbytes)
    host = np.ctypeslib.as_array((ctypes.c_uint8 * nbytes).from_address(hp)).view(PARTICLE_DTYPE)
    P = Particles()
    P.p, P.force, P.np_allocated, P.np_total, P.np_average = hp, None, npart, npart, float(npart)
    lib.cg_dropin_set_abort(0)
    lib.power_init(table.encode(), sched.a_init, 0.81, om, 1 - om)
    lib.lpt_init(nc, None, 0)
    assert lib.lpt_set_displacement(sched.a_init, om, cfg["seed"], L, ctypes.byref(P)) == 0
    rows = torch.from_numpy(np.ascontiguousarray(host).view(np.float32).reshape(npart, 14).copy())
    lib.cg_dropin_finalize()
    comm = TorchComm(device="cuda") if world > 1 else LocalComm(1)
    cap = int(2.0 * npart / world) + 1024
    sim = Simulation(nc, N, L, om, np_capacity=cap)
    rk = GpuRank(sim)
    pm = SlabPM([rk], comm, "cuda")
    x0 = pm.xs[rank][0] * np.float32(L) / N
    x1 = (pm.xs[rank][0] + pm.xs[rank][1]) * np.float32(L) / N
    xw = torch.remainder(rows[:, 0], L)
    mine = rows[(xw >= x0) & (xw < x1)].cuda()
    nsteps_run = sched.nloop - 1

    def step(i):
        j = i % nsteps_run
        if j == 0:       # a realization restarts from the initial conditions
            sim.set_particles_ptr(mine.data_ptr(), mine.shape[0], sched.a_init, sched.a_init)
        _, _, avel1, apos1 = sched.times(j + 1)
        sim.move()
        pm.exchange_particles()
        pm.forces()
        sim.kick_drift(avel1, apos1)

    def barrier():
        if td:
            td.barrier()
    steps = args.steps
    for i in range(args.warmup):
        step(i)
    sim.sync()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for i in range(steps):
        step(args.warmup + i)
    sim.sync()
    ev1.record()
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    if td:
        t = torch.tensor([ms], device="cuda")
        td.all_reduce(t, op=td.ReduceOp.MAX)
        ms = float(t.item())
    barrier()
    if rank == 0:
        out = {"metric": METRIC, "value": npart * steps / (ms / 1e3), "unit": "particle-steps/s",
               "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
               "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
               "dtype": "f32", "data": "synthetic (seeded 2LPT initial conditions, BBKS P(k))",
               "config": {"workload": args.config_desc, "particles": npart, "mesh": N,
                          "boxsize": L, "parallelism": "slab x%d (one realization split by "
                                                      "x slabs)" % world,
                          "l2": "inputs larger than L2 (%.2f GB per mesh)" % (4.0 * N ** 3 / 1e9)},
               "density_sum": pm.density_sum,
               "note": "the slab-decomposed path (exchanges through torch); the default "
                       "bench line runs whole realizations per GPU"}
        print(json.dumps(out))
    sim.close()
    lib.cg_host_free(hp)
    if td:
        td.destroy_process_group()
    return 0


def _z0_snapshot(lib, cfg, table):
    """The z = 0 snapshot (host ParticleMinimum array) of one realization."""
    from cola_halo_b200 import Simulation
    from cola_halo_b200.learned import _lpt_particles
    from cola_halo_b200.schedule import Schedule
    nc, L, om = cfg["nc"], cfg["L"], cfg["om"]
    sched = Schedule.linear(cfg["a_init"], 1.0, cfg["nsteps"])
    p = _lpt_particles(nc, L, cfg["seed"], om, sched.a_init, table)
    sim = Simulation(nc, nc * cfg["factor"], L, om)
    sim.set_particles(p, sched.a_init, sched.a_init)
    snap = sim.run(sched)[-1][1]
    sim.close()
    return snap


def run_fof(args):
    """Friends-of-friends (b = 0.2, >= 32 members) on the z = 0 snapshot of
    the 256^3 and 128^3 workloads: particles per second of one synchronous
    cg_fof call on a device-resident snapshot (its scratch allocation and
    the catalogue download included; median of the timed calls), and the
    reference's own fof.c on the 128^3 snapshot on one host core."""
    rank, world, local = dist_setup(args)
    if rank != 0:
        return 0
    from cola_halo_b200 import _lib
    from cola_halo_b200.bbks import write_bbks_table
    from cola_halo_b200.halos import fof
    lib = _lib.load()
    _lib.check(lib.cg_set_device(local), "cg_set_device")
    cuda = Cudart()
    table = write_bbks_table(os.path.join(tempfile.mkdtemp(), "bbks.dat"))
    out = {"metric": "FoF particles/s", "unit": "particles/s", "higher_is_better": True,
           "n_gpus": 1, "dtype": "f32", "data": "synthetic (seeded 2LPT initial conditions, "
           "BBKS P(k), 10 COLA steps to z = 0)", "runs": {}}
    for name in ("c2", "c3"):
        cfg = CONFIGS[name]
        nc, L = cfg["nc"], cfg["L"]
        ll = float(np.float32(0.2 * L / nc))
        snap = _z0_snapshot(lib, cfg, table)
        d = cuda.device_copy_of(snap)
        for _ in range(max(args.warmup, 1)):
            halos = fof(d.value, L, ll, np_count=len(snap))
        times = []
        for _ in range(args.steps):
            cuda.sync_device()
            t0 = time.perf_counter()
            halos = fof(d.value, L, ll, np_count=len(snap))
            times.append(time.perf_counter() - t0)
        wall_s = float(np.median(times))
        run = {"particles": len(snap), "boxsize": L, "ll": ll, "halos": int(len(halos)),
               "largest": int(halos["nfof"].max()) if len(halos) else 0,
               "wall_s": wall_s, "particles_per_s": len(snap) / wall_s}
        run["coarse_grid"] = _time_coarse_grid(cuda, d, snap, L, args)
        run["gadget"] = _time_gadget(cuda, d, snap, L, args)
        if name == "c3" and not args.no_cpu_baseline:
            try:
                from oracle import ref
                if os.path.exists(ref.LIB_PATH):
                    for cg in run["coarse_grid"]:
                        t0 = time.perf_counter()
                        ref.coarse_grid_file(snap, L, cg["nc"], os.path.join(tempfile.mkdtemp(),
                                                                             "grid.bin"))
                        cg["cpu_reference_s"] = time.perf_counter() - t0
                    gdir = tempfile.mkdtemp()
                    t0 = time.perf_counter()
                    ref.gadget_file(snap, L, 0.273, 0.705, 1.0, os.path.join(gdir, "snp"), 0)
                    run["gadget"]["cpu_reference_s"] = time.perf_counter() - t0
                    shutil.rmtree(gdir, ignore_errors=True)
                    t0 = time.perf_counter()
                    rows = ref.fof_catalog(snap, L, nc, np.float32(ll), tempfile.mkdtemp())
                    cpu_s = time.perf_counter() - t0
                    run["cpu_reference_s"] = cpu_s
                    run["cpu_reference_halos"] = int(len(rows))
                    out["cpu_baseline"] = {"value": len(snap) / cpu_s, "unit": "particles/s",
                                           "cores": 1, "kind": "reference",
                                           "sample": "fof.c (k-d tree, one thread) on the "
                                                     "128^3 z = 0 snapshot"}
            except Exception as e:  # reported, not fatal
                run["cpu_reference_error"] = str(e)
        out["runs"][name] = run
    out["value"] = out["runs"]["c2"]["particles_per_s"]
    out["config"] = {"workload": "FoF b = 0.2 on the 256^3 / L = 600 z = 0 snapshot "
                                 "(value) and the 128^3 / L = 300 one"}
    print(json.dumps(out))
    return 0


def _time_coarse_grid(cuda, d, snap, L, args, grids=(16, 64, 256)):
    """One synchronous cg_coarse_grid call on the device-resident snapshot
    per grid size (nc = 16 is the reference's default coarse_grid_nc): its
    grid allocation, the CIC pass, delta and the download of the grid
    included; median over the timed calls."""
    from cola_halo_b200.coarse import coarse_grid
    out = []
    for nc in grids:
        for _ in range(max(args.warmup, 1)):
            coarse_grid(d.value, L, nc, np_count=len(snap))
        times = []
        for _ in range(args.steps):
            cuda.sync_device()
            t0 = time.perf_counter()
            _, total = coarse_grid(d.value, L, nc, np_count=len(snap))
            times.append(time.perf_counter() - t0)
        wall_s = float(np.median(times))
        out.append({"nc": nc, "wall_s": wall_s, "particles_per_s": len(snap) / wall_s,
                    "mass_sum": total})
    return out


def _time_gadget(cuda, d, snap, L, args):
    """One synchronous cg_write_gadget call (4-byte ids) of the
    device-resident snapshot to a file in a fresh temporary directory:
    formatting, download and the writes into the page cache, median over the
    timed calls (the file is deleted between calls)."""
    from cola_halo_b200.gadget import write_gadget
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, "snp.0")
    times = []
    for k in range(max(args.warmup, 1) + args.steps):
        if os.path.exists(path):
            os.remove(path)
        cuda.sync_device()
        t0 = time.perf_counter()
        write_gadget(path, d.value, 1.0, L, 0.273, 0.705, np_count=len(snap))
        if k >= max(args.warmup, 1):
            times.append(time.perf_counter() - t0)
    size = os.path.getsize(path)
    shutil.rmtree(tmp, ignore_errors=True)
    wall_s = float(np.median(times))
    return {"bytes": size, "wall_s": wall_s, "GB_per_s": size / wall_s / 1e9,
            "dir": os.path.dirname(tmp)}


def run_cufft(args):
    """Device time of one 3-D r2c and one c2r of an N^3 float mesh held in
    HBM: this library's transforms (cg_fft_time: z, x, y passes, layout
    [kz][kx][ky]) beside cuFFT's (torch.fft.rfftn / irfftn, layout
    [x][y][kz]), each the mean of the timed launches after a warm-up."""
    rank, world, local = dist_setup(args)
    if rank != 0:
        return 0
    import torch
    from cola_halo_b200 import _lib
    lib = _lib.load()
    _lib.check(lib.cg_set_device(local), "cg_set_device")
    reps = max(args.steps, 1)
    out = {"metric": "3-D real FFT device time", "unit": "ms", "higher_is_better": False,
           "n_gpus": 1, "dtype": "f32", "runs": {},
           "library": "cuFFT (torch %s) through torch.fft.rfftn / irfftn" % torch.__version__}
    for n in (384, 768):
        r2c, c2r = ctypes.c_float(), ctypes.c_float()
        _lib.check(lib.cg_fft_time(n, reps, ctypes.byref(r2c), ctypes.byref(c2r)), "cg_fft_time")
        x = torch.zeros((n, n, n), device="cuda:%d" % local, dtype=torch.float32)
        spec = torch.fft.rfftn(x)
        y = torch.empty_like(x)

        def timed(f):
            f()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                f()
            b.record()
            b.synchronize()
            return a.elapsed_time(b) / reps
        cr = timed(lambda: torch.fft.rfftn(x, out=spec))
        cc = timed(lambda: torch.fft.irfftn(spec, s=(n, n, n), out=y))
        out["runs"][str(n)] = {"r2c_ms": r2c.value, "c2r_ms": c2r.value, "cufft_r2c_ms": cr,
                               "cufft_c2r_ms": cc, "r2c_speedup": cr / r2c.value,
                               "c2r_speedup": cc / c2r.value}
        del x, spec, y
        torch.cuda.empty_cache()
    print(json.dumps(out))
    return 0


def run_batch(args):
    """Throughput of batched realizations: 32 realizations of 128^3
    particles on 384^3 meshes with box sizes L ~ U[250, 400] Mpc/h and step
    counts ~ U[5, 20] drawn from a fixed meta-seed, 2LPT at z = 49, recorded
    into one CUDA graph over --batch-streams streams; a particle-step is one COLA step of
    one particle.  Device time from CUDA events around each graph launch."""
    rank, world, local = dist_setup(args)
    if rank != 0:
        return 0
    from cola_halo_b200 import _lib
    from cola_halo_b200.batch import Batch
    from cola_halo_b200.bbks import write_bbks_table
    from cola_halo_b200.types import PARTICLE_DTYPE, Particles
    lib = _lib.load()
    _lib.check(lib.cg_set_device(local), "cg_set_device")
    nreal, nc, N, om, a_init = 32, 128, 384, 0.273, 0.02
    meta = np.random.default_rng(2024)
    specs = [dict(nc=nc, ngrid=N, boxsize=float(meta.uniform(250.0, 400.0)), a_init=a_init,
                  nsteps=int(meta.integers(5, 21)), aout=1.0) for _ in range(nreal)]
    table = write_bbks_table(os.path.join(tempfile.mkdtemp(), "bbks.dat"))
    _lib.check(lib.cg_autotune(N, 0, None, None), "cg_autotune")
    npart = nc ** 3
    nbytes = 56 * npart
    hp_ptr = lib.cg_host_alloc(nbytes)
    host = np.ctypeslib.as_array((ctypes.c_uint8 * nbytes).from_address(hp_ptr)).view(
        PARTICLE_DTYPE)
    P = Particles()
    P.p = hp_ptr
    P.force = None
    P.np_allocated = npart
    P.np_total = npart
    P.np_average = float(npart)
    lib.cg_dropin_set_abort(0)
    lib.power_init(table.encode(), a_init, 0.81, om, 1 - om)
    lib.lpt_init(nc, None, 0)
    b = Batch(specs, om, nstreams=args.batch_streams)
    dep = None
    for i, sp in enumerate(specs):
        rc = lib.lpt_set_displacement(a_init, om, 1000 + i, sp["boxsize"], ctypes.byref(P))
        assert rc == 0, lib.cg_last_error()
        b.set_particles(i, host)
        if i == 0:
            # the deposit shape for 384^3, tuned on the first realization five
            # steps in (installed per mesh size, so the graph records it)
            from cola_halo_b200 import Simulation
            from cola_halo_b200.schedule import Schedule
            from cola_halo_b200.tune import tune_deposit
            sched = Schedule.linear(a_init, 1.0, sp["nsteps"])
            sim = Simulation(nc, N, sp["boxsize"], om)
            sim.set_particles(host, a_init, a_init)
            for j in range(min(5, sp["nsteps"])):
                _, _, avel1, apos1 = sched.times(j + 1)
                sim.move()
                sim.forces()
                sim.kick_drift(avel1, apos1)
            dep = tune_deposit(sim)[0]
            sim.close()
    for _ in range(args.warmup):
        b.run()
    times = []
    for _ in range(args.steps):
        b.run()
        times.append(b.last_ms())
    ms = sum(times)
    psteps = sum(npart * sp["nsteps"] for sp in specs)
    value = psteps * len(times) / (ms / 1e3)
    # a realization of n steps evaluates the force n + 1 times (main.c:162-206)
    # and ends with its P(k): per force evaluation the rate is
    pforces = sum(npart * (sp["nsteps"] + 1) for sp in specs)
    out = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": 1,
           "steps": len(times), "warmup": args.warmup, "ms_per_step": ms / len(times),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded 2LPT initial conditions, BBKS P(k))",
           "config": {"workload": "batch: 32 x 128^3 particles, 384^3 meshes, L ~ U[250,400] "
                                  "Mpc/h, nsteps ~ U[5,20] (meta-seed 2024), one CUDA graph",
                      "realizations": nreal, "particle_steps_per_launch": psteps,
                      "graph_nodes": b.num_nodes(), "streams": args.batch_streams,
                      "deposit_variant": {"chosen": dep, "chosen_by": "cg_sim_tune_deposit"},
                      "l2": "inputs larger than L2 (0.23 GB per mesh, 32 realizations)"},
           "ms_per_launch": [round(t, 3) for t in times],
           "particle_force_evaluations_per_s": pforces * len(times) / (ms / 1e3),
           "note": "a step of this line is one graph launch running all 32 realizations"}
    print(json.dumps(out))
    b.close()
    lib.cg_host_free(hp_ptr)
    return 0


# coarse runs beside the conv net: (name, mesh, (gradient, laplacian,
# deconvolve), least-squares fitted transfer functions, P(k)-calibrated
# transfer functions, knots)
LEARNED_VARIANTS = (("deconv2_128", 128, (0, 0, 2), False, False, 0),
                    ("calibrated_128", 128, (0, 0, 2), False, True, 32),
                    ("filtered_192", 192, (0, 0, 0), True, True, 24),
                    ("filtered_256", 256, (0, 0, 0), True, False, 32))
HEADLINE_VARIANT = "calibrated_128"


def run_learned(args):
    """Learned coarse-mesh run vs the plain factor-3 run (128^3 particles,
    L = 300 Mpc/h, coarse 128^3 / fine 384^3 mesh, 10 steps from z = 49):
    P(k) error up to 0.5 k_Nyq and wall time per realization."""
    from cola_halo_b200 import _lib
    from cola_halo_b200.bbks import write_bbks_table
    from cola_halo_b200.learned import MF_EDGES, ConvNet, evaluate
    from cola_halo_b200.schedule import Schedule
    lib = _lib.load()
    _lib.check(lib.cg_set_device(0), "cg_set_device")
    nc, L = 128, 300.0
    sched = Schedule.linear(0.02, 1.0, 10)
    table = write_bbks_table(os.path.join(tempfile.mkdtemp(), "bbks.dat"))
    net = ConvNet(nc, seed=7)
    net2 = ConvNet(nc, seed=8)
    net3 = ConvNet(nc, seed=9)
    net4 = ConvNet(nc, seed=10)
    res = evaluate(nc, L, sched, net, list(range(1, args.train_seeds + 1)),
                   list(range(1001, 1001 + args.eval_seeds)), table, epochs=args.epochs,
                   filter_nk=16, net2=net2, variants=LEARNED_VARIANTS,
                   net_variants=((HEADLINE_VARIANT, net3),),
                   net_first=(("net_calibrated_128", 128, (0, 0, 2), 32, net4),),
                   log=lambda s: print(s, file=sys.stderr, flush=True))
    seeds = res["seeds"]
    fine_s = float(np.mean([r["fine_s"] for r in seeds]))
    learned_s = float(np.mean([r["learned_s"] for r in seeds]))
    coarse_s = float(np.mean([r["coarse_s"] for r in seeds]))
    err_l = float(np.mean([r["err_learned"] for r in seeds]))
    head = HEADLINE_VARIANT
    head_s = float(np.mean([r[head + "_s"] for r in seeds]))
    err_h = float(np.mean([r["err_" + head] for r in seeds]))
    out = {"metric": "wall time to 1% P(k) error, learned vs plain PM",
           "value": fine_s / head_s, "unit": "x (plain factor-3 time / learned time)",
           "learned_method": "128^3 mesh (factor 1) with the CIC window divided out twice and "
                             "a transfer function T(|n|) of the force (32 knots) calibrated "
                             "on the final P(k) of 4 training seeds against the factor-3 run",
           "pk_err": err_h,
           "pk_err_max": float(np.max([r["err_" + head] for r in seeds])),
           "reaches_1pct": bool(err_h <= 0.01),
           "timing": "device time of each realization's time loop (11 force evaluations) "
                     "from the library's CUDA-event profile; host wall times beside it",
           "plain_fine_wall_s": float(np.mean([r["fine_wall_s"] for r in seeds])),
           "learned_wall_s": float(np.mean([r[head + "_wall_s"] for r in seeds])),
           "plain_coarse_wall_s": float(np.mean([r["coarse_wall_s"] for r in seeds])),
           "higher_is_better": True, "n_gpus": 1, "dtype": "f32 PM, bf16 net (fp32 accum)",
           "data": "synthetic (seeded 2LPT initial conditions, BBKS P(k))",
           "config": {"workload": "128^3 particles, L=300 Mpc/h, coarse 128^3 (factor 1) "
                                  "vs plain 384^3 (factor 3), 10 steps z=49 -> 0",
                      "train_seeds": args.train_seeds, "eval_seeds": args.eval_seeds,
                      "epochs": args.epochs, "kmax": "0.5 k_Nyq = %.4f h/Mpc" % (0.5 * math.pi * nc / L)},
           "plain_fine_s": fine_s, "learned_s": head_s, "plain_coarse_s": coarse_s,
           "pk_err_coarse": float(np.mean([r["err_coarse"] for r in seeds])),
           "conv_net": {"what": "3-layer 3x3x3 conv net (2->16->16->3, bf16 tcgen05, fp32 "
                                "accumulate) on the 128^3 mesh, trained online on PM pairs",
                        "s": learned_s, "speedup_vs_plain_fine": fine_s / learned_s,
                        "pk_err": err_l,
                        "pk_err_max": float(np.max([r["err_learned"] for r in seeds]))},
           "mass_function": {"log10_nfof_edges": [round(float(e), 4) for e in MF_EDGES],
                             "fine": res.get("mf_fine"), "coarse": res.get("mf_coarse"),
                             "conv_net": res.get("mf_learned"),
                             "ratio_err_coarse": res.get("mf_err_coarse"),
                             "ratio_err_conv_net": res.get("mf_err_learned"),
                             "halo_finder": "GPU FoF (cg_fof), b = 0.2, >= 32 members, "
                                            "summed over the evaluation seeds"},
           "train_s": res["train_s"], "train_steps": res["train_steps"],
           "loss_first": res["loss_first"], "loss_last": res["loss_last"]}
    # the Fourier-space correction: per-step transfer functions T_s(|n|) of
    # the coarse force (16 knots, least squares on 4 training seeds), alone
    # and with a second net trained on the filtered force
    for name in (["filtered", "filtered_net"] + [v[0] for v in LEARNED_VARIANTS] +
                 [HEADLINE_VARIANT + "_net", "net_calibrated_128"]):
        if "err_" + name in seeds[0]:
            t = float(np.mean([r[name + "_s"] for r in seeds]))
            out[name] = {"s": t, "speedup_vs_plain_fine": fine_s / t,
                         "wall_s": float(np.mean([r[name + "_wall_s"] for r in seeds])),
                         "pk_err": float(np.mean([r["err_" + name] for r in seeds])),
                         "pk_err_max": float(np.max([r["err_" + name] for r in seeds])),
                         "mf_ratio_err": res.get("mf_err_" + name),
                         "mf": res.get("mf_" + name)}
    for name, ng, kernel, fit, cal, nk in LEARNED_VARIANTS:
        if name in out:
            out[name].update({"mesh": ng, "force_kernel": list(kernel), "lsq_fit": fit,
                              "pk_calibrated": cal, "knots": nk})
            if fit or cal:
                out[name]["fit_s"] = res["fit_s_" + name]
            if cal:
                out[name]["calibration_train_err"] = [round(h, 4) for h in
                                                      res["cal_hist_" + name]]
    if "filters" in res:
        out["filter"] = {"knots": 16, "fit_seeds": 4, "fit_s": res["filter_fit_s"],
                         "T_first_last_step": [[round(v, 4) for v in res["filters"][0]],
                                               [round(v, 4) for v in res["filters"][-1]]]}
    if "filters_" + head in res:
        out["headline_T_last_step"] = [round(v, 4) for v in res["filters_" + head][-1]]
    if "train2_s" in res:
        out["filtered_net"]["train_s"] = res["train2_s"]
        out["filtered_net"]["loss_last"] = res["loss2_last"]
    if "net_calibrated_128" in out:
        out["net_calibrated_128"].update({
            "what": "the conv net trained first on the window-corrected 128^3 force, then a "
                    "transfer function T(|n|) of 32 knots calibrated on the final P(k) of runs "
                    "with the net's correction in",
            "train_s": res["train_s_net_calibrated_128"],
            "loss_first": res["loss_first_net_calibrated_128"],
            "loss_last": res["loss_last_net_calibrated_128"],
            "fit_s": res["fit_s_net_calibrated_128"],
            "calibration_train_err": [round(h, 4) for h in res["cal_hist_net_calibrated_128"]]})
    hn = HEADLINE_VARIANT + "_net"
    if hn in out:
        out[hn].update({"what": "the headline correction plus the conv net trained on what it "
                                "leaves (fine force - corrected coarse force) over the training "
                                "seeds",
                        "train_s": res["train_s_" + hn], "loss_first": res["loss_first_" + hn],
                        "loss_last": res["loss_last_" + hn],
                        "net_gain_pk_err": out[HEADLINE_VARIANT]["pk_err"] - out[hn]["pk_err"]})
    print(json.dumps(out))
    net2.close()
    return 0


def run_learned_large(args):
    """The large configuration: 512^3 particles, L = 1200 Mpc/h, 20 steps
    from z = 49; the plain run on a 1024^3 mesh (factor 2) is the truth, the
    learned run a 512^3 mesh (factor 1) with the calibrated Fourier-space
    correction (calibrated on the training seeds' final P(k) against the
    factor-2 runs); the plain 512^3 run beside it."""
    from cola_halo_b200 import _lib
    from cola_halo_b200.bbks import write_bbks_table
    from cola_halo_b200.learned import evaluate_large
    from cola_halo_b200.schedule import Schedule
    lib = _lib.load()
    _lib.check(lib.cg_set_device(0), "cg_set_device")
    nc, L = 512, 1200.0
    sched = Schedule.linear(0.02, 1.0, 20)
    table = write_bbks_table(os.path.join(tempfile.mkdtemp(), "bbks.dat"))
    ntrain = min(args.train_seeds, 2)
    neval = min(args.eval_seeds, 2)
    res = evaluate_large(nc, L, sched, 512, 2, list(range(1, ntrain + 1)),
                         list(range(1001, 1001 + neval)), table,
                         log=lambda s: print(s, file=sys.stderr, flush=True))
    seeds = res["seeds"]
    mean = lambda key: float(np.mean([r[key] for r in seeds]))
    out = {"metric": "wall time to matched P(k) error, learned 512^3 vs plain factor-2 1024^3",
           "value": mean("fine_s") / mean("learned_s"),
           "unit": "x (plain factor-2 time / learned time)", "higher_is_better": True,
           "n_gpus": 1, "dtype": "f32", "data": "synthetic (seeded 2LPT initial conditions, "
           "BBKS P(k))",
           "config": {"workload": "512^3 particles, L=1200 Mpc/h, 20 COLA steps z=49 -> 0; "
                                  "learned 512^3 mesh vs plain 1024^3 mesh (factor 2)",
                      "train_seeds": ntrain, "eval_seeds": neval,
                      "kmax": "0.5 k_Nyq = %.4f h/Mpc" % (0.5 * math.pi * nc / L)},
           "learned_method": "512^3 mesh (factor 1), CIC window divided out twice, T(|n|) of "
                             "32 knots calibrated on the final P(k) of the training seeds "
                             "against the factor-2 runs",
           "plain_fine_s": mean("fine_s"), "learned_s": mean("learned_s"),
           "plain_coarse_s": mean("coarse_s"),
           "pk_err_learned": mean("err_learned"),
           "pk_err_learned_max": float(np.max([r["err_learned"] for r in seeds])),
           "pk_err_coarse": mean("err_coarse"),
           "timing": "device time of each realization's time loop (21 force evaluations) from "
                     "the library's CUDA-event profile",
           "calibration_s": res["calibration_s"],
           "calibration_train_err": [round(h, 4) for h in res["calibration_train_err"]],
           "seeds": seeds}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
