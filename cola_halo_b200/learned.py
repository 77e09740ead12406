"""Learned small-scale force correction on a coarse mesh (cg_net_* in
colagpu.h): training on PM-generated pairs and learned-correction runs."""
import ctypes

import numpy as np

from . import _lib
from .schedule import output_scale_factors, run_time_loop


class ConvNet:
    def __init__(self, ngrid, seed=1):
        self.lib = _lib.load()
        self.ngrid = ngrid
        h = ctypes.c_void_p()
        _lib.check(self.lib.cg_net_create(ctypes.byref(h), ngrid, seed), "cg_net_create")
        self.h = h
        self.nparams = self.lib.cg_net_num_params()

    def close(self):
        if self.h:
            self.lib.cg_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        _lib.check(self.lib.cg_net_get_params(self.h, p.ctypes.data), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(self.lib.cg_net_set_params(self.h, p.ctypes.data), "set_params")

    def set_scales(self, in_delta, in_phi, out_scale):
        _lib.check(self.lib.cg_net_set_scales(self.h, in_delta, in_phi, out_scale), "scales")

    def tensor_cores(self, on):
        _lib.check(self.lib.cg_net_set_tensor_cores(self.h, 1 if on else 0), "tensor cores")

    def forward_host(self, in2):
        n = self.ngrid
        a = np.ascontiguousarray(in2, dtype=np.float32)
        out = np.zeros((n, n, n, 3), dtype=np.float32)
        _lib.check(self.lib.cg_net_forward_host(self.h, a.ctypes.data, out.ctypes.data),
                   "forward_host")
        return out

    def backward_host(self, in2, grad3):
        a = np.ascontiguousarray(in2, dtype=np.float32)
        g = np.ascontiguousarray(grad3, dtype=np.float32)
        out = np.zeros(self.nparams, dtype=np.float32)
        _lib.check(self.lib.cg_net_backward_host(self.h, a.ctypes.data, g.ctypes.data,
                                                 out.ctypes.data), "backward_host")
        return out

    def train_step(self, coarse, fine, lr):
        loss = ctypes.c_double()
        _lib.check(self.lib.cg_net_train_step(self.h, coarse.h, fine.h, lr, ctypes.byref(loss)),
                   "cg_net_train_step")
        return loss.value

    def forces(self, coarse):
        _lib.check(self.lib.cg_net_forces(self.h, coarse.h), "cg_net_forces")

    def run(self, coarse, sched, zout=(0.0,)):
        """The reference time loop on the coarse realization with corrected
        forces; returns the snapshots."""
        snaps = []
        run_time_loop(sched, output_scale_factors(zout), move=coarse.move,
                      force=lambda: self.forces(coarse), kick=coarse.kick, drift=coarse.drift,
                      snapshot=lambda a, i: snaps.append((a, coarse.snapshot(a))),
                      kick_drift=coarse.kick_drift)
        return snaps


def copy_particles(dst, src):
    _lib.check(_lib.load().cg_sim_copy_particles(dst.h, src.h), "cg_sim_copy_particles")


def _lpt_particles(nc, boxsize, seed, omega_m, a_init, table):
    """2LPT particles of one seed from the GPU drop-in lpt_set_displacement."""
    from .types import HostParticles
    lib = _lib.load()
    lib.cg_dropin_set_abort(0)
    lib.power_init(table.encode(), a_init, 0.81, omega_m, 1 - omega_m)
    lib.lpt_init(nc, None, 0)
    hp = HostParticles(nc)
    rc = lib.lpt_set_displacement(a_init, omega_m, seed, boxsize, hp.ptr)
    if rc != 0:
        raise _lib.ColaGpuError(lib.cg_last_error().decode())
    return hp.local().copy()


def train_online(net, coarse, fine, sched, seeds, table, *, lr=2e-3, epochs=1,
                 steps_per_state=1, omega_m=0.273, log=None):
    """Train on PM-generated pairs along fine-mesh trajectories: for each
    seed and each time step, copy the fine run's particles to the coarse
    realization and take `steps_per_state` optimiser steps on
    (coarse features, fine - coarse force).  Returns the loss history."""
    hist = []
    for ep in range(epochs):
        for seed in seeds:
            p = _lpt_particles(fine.nc, fine.boxsize, seed, omega_m, sched.a_init, table)
            fine.set_particles(p, sched.a_init, sched.a_init)
            for i in range(1, sched.nloop):
                _, _, avel1, apos1 = sched.times(i)
                fine.move()
                copy_particles(coarse, fine)
                for _ in range(steps_per_state):
                    hist.append(net.train_step(coarse, fine, lr))
                # train_step left the fine forces of these positions in `fine`
                fine.kick(avel1)
                fine.drift(apos1)
            if log:
                log("epoch %d seed %d loss %.4g" % (ep, seed, hist[-1]))
    return hist


def power_spectrum_on(sim_pk, snap_x, a):
    """P(k) of snapshot positions measured with realization sim_pk's mesh
    (CIC window deconvolved, shot noise subtracted)."""
    from .types import PARTICLE_DTYPE
    p = np.zeros(len(snap_x), dtype=PARTICLE_DTYPE)
    p["x"] = snap_x
    p["id"] = np.arange(1, len(p) + 1)
    sim_pk.set_particles(p, a, a)
    sim_pk.move()
    return sim_pk.power_spectrum(deconvolve_cic=True, subtract_shot=True)


# log10(members) bin edges of the halo mass function: 32 members up, 0.25 dex
MF_EDGES = np.log10(32.0) + 0.25 * np.arange(13)


def halo_counts(snap, boxsize, nc, b=0.2):
    """FoF (b = 0.2 of the mean particle spacing, >= 32 members, fof.c) halo
    counts of a snapshot in the MF_EDGES log-mass bins (mass in particles)."""
    from .halos import fof
    ll = float(np.float32(b * boxsize / nc))
    h = fof(snap, boxsize, ll)
    return np.histogram(np.log10(h["nfof"].astype(np.float64)), bins=MF_EDGES)[0]


def mf_ratio_error(counts, counts_ref, min_ref=20):
    """max over bins with at least `min_ref` reference halos of
    |N / N_ref - 1|."""
    ok = counts_ref >= min_ref
    if not ok.any():
        return float("nan")
    return float(np.max(np.abs(counts[ok] / counts_ref[ok] - 1.0)))


def pk_error(k, p, p_ref, kmax):
    """max over bins with 0 < k <= kmax of |P/P_ref - 1|."""
    ok = (k > 0) & (k <= kmax) & (p_ref > 0)
    return float(np.max(np.abs(p[ok] / p_ref[ok] - 1.0)))


def evaluate(nc, boxsize, sched, net, train_seeds, eval_seeds, table, *, omega_m=0.273,
             epochs=1, lr=2e-3, log=None):
    """Train on PM pairs, then judge plain-coarse and learned-coarse runs
    against the plain factor-3 run on held-out seeds: P(k) error up to half
    the particle Nyquist wavenumber, and the device time of each run's time
    loop (with the host wall time beside it)."""
    import time

    from .sim import Simulation
    fine = Simulation(nc, 3 * nc, boxsize, omega_m)
    coarse = Simulation(nc, nc, boxsize, omega_m)
    t0 = time.perf_counter()
    hist = train_online(net, coarse, fine, sched, train_seeds, table, lr=lr, epochs=epochs,
                        omega_m=omega_m, log=log)
    train_s = time.perf_counter() - t0
    kmax = 0.5 * np.pi * nc / boxsize
    res = {"train_s": train_s, "train_steps": len(hist), "loss_first": float(np.mean(hist[:10])),
           "loss_last": float(np.mean(hist[-10:])), "seeds": []}

    lib = _lib.load()
    nst = _lib.NSTAGES

    def timed_run(sim, force):
        """The time loop up to the z = 0 output (its 11 force evaluations,
        kicks and drifts), timed on the device: the library's event profile
        spans the first launch to the last.  The snapshot itself (a download
        of the same size for every method) is taken after the timed region."""
        sim.sync()
        _lib.check(lib.cg_prof_begin(8192), "cg_prof_begin")
        t = time.perf_counter()
        run_time_loop(sched, output_scale_factors((0.0,)), move=sim.move, force=force,
                      kick=sim.kick, drift=sim.drift, snapshot=lambda a, i: None,
                      kick_drift=sim.kick_drift)
        ms = (ctypes.c_double * nst)()
        cnt = (ctypes.c_int * nst)()
        lib.cg_prof_end(ms, cnt, nst)
        wall = time.perf_counter() - t
        snap = sim.snapshot(output_scale_factors((0.0,))[0])
        return snap, sum(ms) / 1e3, wall

    for seed in eval_seeds:
        p = _lpt_particles(nc, boxsize, seed, omega_m, sched.a_init, table)
        fine.set_particles(p, sched.a_init, sched.a_init)
        s_f, t_f, w_f = timed_run(fine, fine.forces)
        coarse.set_particles(p, sched.a_init, sched.a_init)
        s_c, t_c, w_c = timed_run(coarse, coarse.forces)
        coarse.set_particles(p, sched.a_init, sched.a_init)
        s_l, t_l, w_l = timed_run(coarse, lambda: net.forces(coarse))
        k, pf, _ = power_spectrum_on(fine, s_f["x"], 1.0)
        _, pc, _ = power_spectrum_on(fine, s_c["x"], 1.0)
        _, pl, _ = power_spectrum_on(fine, s_l["x"], 1.0)
        mf_f, mf_c, mf_l = (halo_counts(s, boxsize, nc) for s in (s_f, s_c, s_l))
        res["mf_fine"] = res.get("mf_fine", 0) + mf_f
        res["mf_coarse"] = res.get("mf_coarse", 0) + mf_c
        res["mf_learned"] = res.get("mf_learned", 0) + mf_l
        r = {"seed": seed, "fine_s": t_f, "coarse_s": t_c, "learned_s": t_l,
             "fine_wall_s": w_f, "coarse_wall_s": w_c, "learned_wall_s": w_l,
             "err_coarse": pk_error(k, pc, pf, kmax), "err_learned": pk_error(k, pl, pf, kmax),
             "halos_fine": int(mf_f.sum()), "halos_coarse": int(mf_c.sum()),
             "halos_learned": int(mf_l.sum())}
        res["seeds"].append(r)
        if log:
            log(str(r))
    fine.close()
    coarse.close()
    if "mf_fine" in res:
        res["mf_err_coarse"] = mf_ratio_error(res["mf_coarse"], res["mf_fine"])
        res["mf_err_learned"] = mf_ratio_error(res["mf_learned"], res["mf_fine"])
        for key in ("mf_fine", "mf_coarse", "mf_learned"):
            res[key] = [int(c) for c in res[key]]
    return res
