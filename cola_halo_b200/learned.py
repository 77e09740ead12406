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
                 steps_per_state=1, omega_m=0.273, filters=None, log=None):
    """Train on PM-generated pairs along fine-mesh trajectories: for each
    seed and each time step, copy the fine run's particles to the coarse
    realization and take `steps_per_state` optimiser steps on
    (coarse features, fine - coarse force).  With `filters` (fitted by
    fit_force_filter) the coarse force is the filtered one of each step, so
    the net learns what the transfer function leaves.  Returns the loss
    history."""
    hist = []
    if filters is not None:
        coarse.set_force_filters(filters)
    for ep in range(epochs):
        for seed in seeds:
            p = _lpt_particles(fine.nc, fine.boxsize, seed, omega_m, sched.a_init, table)
            fine.set_particles(p, sched.a_init, sched.a_init)
            for i in range(1, sched.nloop):
                _, _, avel1, apos1 = sched.times(i)
                fine.move()
                copy_particles(coarse, fine)
                if filters is not None:
                    coarse.use_force_filter(min(i - 1, len(filters) - 1))
                for _ in range(steps_per_state):
                    hist.append(net.train_step(coarse, fine, lr))
                # train_step left the fine forces of these positions in `fine`
                fine.kick(avel1)
                fine.drift(apos1)
            if log:
                log("epoch %d seed %d loss %.4g" % (ep, seed, hist[-1]))
    return hist


def fit_force_filter(coarse, fine, sched, seeds, table, *, nk=16, sample=1 << 18,
                     ridge=1e-3, omega_m=0.273, log=None):
    """Fourier-space learned correction: per force evaluation s of the time
    loop, the isotropic transfer function T_s(|n|) of the coarse mesh's
    force that best reproduces the fine mesh's force on the same particles,
    by linear least squares along fine-mesh trajectories.

    The coarse force is linear in the knots (the Green step multiplies the
    spectrum by T, every later stage is linear), so with the hat basis e_j
    (one knot 1, the others 0) F(T) = sum_j T_j F(e_j), and T_s solves
    (A_s + lam I) T = b_s + lam 1 with A_jk = <F(e_j), F(e_k)>,
    b_j = <F(e_j), F_fine> summed over a fixed random sample of particles,
    their three components and the seeds; lam = ridge tr(A_s) / nk pulls
    poorly constrained knots toward T = 1 (the reference's force).
    Returns an (nloop - 1, nk) float32 array of knots; the coarse
    realization's filters are removed again."""
    nst = sched.nloop - 1
    A = np.zeros((nst, nk, nk))
    b = np.zeros((nst, nk))
    npart = fine.nc ** 3
    sub = np.sort(np.random.default_rng(0).choice(npart, size=min(sample, npart),
                                                  replace=False))
    coarse.set_force_filters(np.eye(nk, dtype=np.float32))
    G = np.empty((nk, 3 * len(sub)))
    for seed in seeds:
        p = _lpt_particles(fine.nc, fine.boxsize, seed, omega_m, sched.a_init, table)
        fine.set_particles(p, sched.a_init, sched.a_init)
        for i in range(1, sched.nloop):
            _, _, avel1, apos1 = sched.times(i)
            fine.move()
            copy_particles(coarse, fine)
            fine.forces()
            ff = fine.get_forces()[sub].astype(np.float64).ravel()
            for j in range(nk):
                coarse.use_force_filter(j)
                coarse.forces()
                G[j] = coarse.get_forces()[sub].ravel()
            A[i - 1] += G @ G.T
            b[i - 1] += G @ ff
            fine.kick(avel1)
            fine.drift(apos1)
        if log:
            log("filter fit: seed %d" % seed)
    coarse.set_force_filters(None)
    T = np.empty((nst, nk))
    for s in range(nst):
        lam = ridge * np.trace(A[s]) / nk
        T[s] = np.linalg.solve(A[s] + lam * np.eye(nk), b[s] + lam)
    return T.astype(np.float32)


def _final_positions(sim, sched, force):
    """Positions at a = 1 of the reference time loop on `sim`."""
    aout = output_scale_factors((0.0,))
    snaps = []
    run_time_loop(sched, aout, move=sim.move, force=force, kick=sim.kick, drift=sim.drift,
                  snapshot=lambda a, i: snaps.append(sim.snapshot(a)),
                  kick_drift=sim.kick_drift)
    return snaps[-1]["x"]


def calibrate_force_filter(sim, fine, sched, seeds, table, *, nk=16, base=None, iters=10,
                           gamma=0.5, kmax=None, omega_m=0.273, net=None, log=None):
    """Calibrate the transfer function of `sim`'s force on its final P(k):
    T_s(|n|) = base_s(|n|) C(|n|) with one C shared by all steps, updated
    multiplicatively from the ratio of the a = 1 power spectra of `sim` and
    of the fine realization on the training seeds,
        C <- C (P_sim / P_fine)^(-g),
    the ratio averaged over the seeds and read at each knot by linear
    interpolation in |n| over the bins up to `kmax` (h/Mpc; default the
    particle Nyquist wavenumber), held at its last value beyond.  An update
    that does not lower the training error (max over k <= kmax / 2 of
    |P/P_fine - 1|, mean over seeds) is discarded and retried with g
    halved (g starts at `gamma`).  With `net`, the runs add the conv net's
    correction to the filtered force (the net trained first, the transfer
    function calibrated on what the two give together).  Returns the best
    iterate as an (nsteps, nk) float32 array, with the error history of the
    `iters` evaluations."""
    nc, L, ng = fine.nc, fine.boxsize, sim.ngrid
    kmax = kmax or np.pi * nc / L
    if base is None:
        base = np.ones((sched.nloop - 1, nk), dtype=np.float32)
    nk = base.shape[1]
    knot_n = np.arange(nk) * (np.sqrt(3.0) * ng / 2) / (nk - 1)
    truth = []
    for seed in seeds:
        p = _lpt_particles(nc, L, seed, omega_m, sched.a_init, table)
        fine.set_particles(p, sched.a_init, sched.a_init)
        k, pf, _ = power_spectrum_on(fine, _final_positions(fine, sched, fine.forces), 1.0)
        truth.append((p, pf))
    n_of_k = k * L / (2 * np.pi)
    fit = (k > 0) & (k <= kmax)

    def trial(C):
        filt = (base * C[None, :]).astype(np.float32)
        ratios, errs = [], []
        for p, pf in truth:
            sim.set_particles(p, sched.a_init, sched.a_init)
            x = _final_positions(sim, sched, filtered_force(sim, filt, net))
            sim.set_force_filters(None)
            _, pc, _ = power_spectrum_on(fine, x, 1.0)
            ratios.append(pc / np.where(pf > 0, pf, 1.0))
            errs.append(pk_error(k, pc, pf, 0.5 * kmax))
        return float(np.mean(errs)), np.mean(ratios, axis=0), filt

    err, ratio, filt = trial(np.ones(nk))
    best = (err, ratio, np.ones(nk), filt)
    hist = [err]
    g = gamma
    for it in range(iters - 1):
        rk = np.interp(knot_n, n_of_k[fit], best[1][fit])
        C = best[2] * np.clip(rk, 0.5, 2.0) ** (-g)
        err, ratio, filt = trial(C)
        hist.append(err)
        if log:
            log("calibration %d (g %.3g): training P(k) error %.4f" % (it, g, err))
        if err < best[0]:
            best = (err, ratio, C, filt)
        else:
            g *= 0.5
    return best[3], hist


def filtered_force(sim, filters, net=None):
    """A force callback for run_time_loop that applies filters[s] at the
    s-th force evaluation (the last one beyond the table), plus the conv
    net's correction when `net` is given.  Loads the filters once."""
    sim.set_force_filters(filters)
    count = [0]

    def force():
        sim.use_force_filter(min(count[0], len(filters) - 1))
        count[0] += 1
        if net is None:
            sim.forces()
        else:
            net.forces(sim)
    return force


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
             epochs=1, lr=2e-3, filter_nk=16, filter_seeds=4, net2=None, variants=(),
             net_variants=(), net_first=(), log=None):
    """Train on PM pairs, then evaluate plain-coarse and learned-coarse runs
    against the plain factor-3 run on held-out seeds: P(k) error up to half
    the particle Nyquist wavenumber, and the device time of each run's time
    loop (with the host wall time beside it).

    filter_nk > 0 also fits per-step force transfer functions of filter_nk
    knots on the first `filter_seeds` training seeds (fit_force_filter) and
    evaluates the filtered coarse run; `net2`, when given, is trained on the
    filtered coarse force and evaluated as filter + net.  Each
    (name, ngrid, kernel, fit, calibrate, nk) in `variants` adds a run on an
    ngrid mesh with the Green-step options `kernel` = (gradient, laplacian,
    deconvolve), with transfer functions of nk knots: least-squares fitted
    on forces when `fit` (fit_force_filter), then calibrated on the final
    P(k) when `calibrate` (calibrate_force_filter), both on the first
    `filter_seeds` training seeds: the error-versus-time curve between the
    coarse and the fine mesh.  Each (variant name, net) in `net_variants`
    trains that net on the named variant's corrected force (its kernel and
    transfer functions) over all training seeds, and evaluates the variant
    with the net's correction added as "<name>_net".  Each (name, ngrid,
    kernel, nk, net) in `net_first` trains the net on that mesh's force
    with the Green-step options `kernel`, then calibrates transfer functions
    of nk knots on the final P(k) of the coarse runs with the net's
    correction in (calibrate_force_filter with net), and evaluates the two
    together as `name`."""
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
    filters = None
    if filter_nk > 0:
        t0 = time.perf_counter()
        filters = fit_force_filter(coarse, fine, sched, train_seeds[:filter_seeds], table,
                                   nk=filter_nk, omega_m=omega_m, log=log)
        res["filter_fit_s"] = time.perf_counter() - t0
        res["filters"] = filters.tolist()
        if net2 is not None:
            t0 = time.perf_counter()
            h2 = train_online(net2, coarse, fine, sched, train_seeds, table, lr=lr,
                              epochs=epochs, omega_m=omega_m, filters=filters, log=log)
            res["train2_s"] = time.perf_counter() - t0
            res["loss2_last"] = float(np.mean(h2[-10:]))
            coarse.set_force_filters(None)
    extra = []                 # (name, realization, filters or None)
    for name, ng, kernel, fit, calibrate, nk in variants:
        sim = Simulation(nc, ng, boxsize, omega_m)
        sim.set_force_kernel(*kernel)
        fl = None
        t0 = time.perf_counter()
        if fit:
            fl = fit_force_filter(sim, fine, sched, train_seeds[:filter_seeds], table, nk=nk,
                                  omega_m=omega_m, log=log)
        if calibrate:
            fl, hist = calibrate_force_filter(sim, fine, sched, train_seeds[:filter_seeds], table,
                                              nk=nk, base=fl, omega_m=omega_m, log=log)
            res["cal_hist_" + name] = hist
        if fit or calibrate:
            res["fit_s_" + name] = time.perf_counter() - t0
            res["filters_" + name] = fl.tolist()
        extra.append((name, sim, fl))
    nets_on = []               # (name, realization, filters, net)
    extra_sims = []
    for name, ng, kernel, nk, nt in net_first:
        sim = Simulation(nc, ng, boxsize, omega_m)
        sim.set_force_kernel(*kernel)
        t0 = time.perf_counter()
        h4 = train_online(nt, sim, fine, sched, train_seeds, table, lr=lr, epochs=epochs,
                          omega_m=omega_m, log=log)
        res["train_s_" + name] = time.perf_counter() - t0
        res["loss_first_" + name] = float(np.mean(h4[:10]))
        res["loss_last_" + name] = float(np.mean(h4[-10:]))
        t0 = time.perf_counter()
        fl, hist = calibrate_force_filter(sim, fine, sched, train_seeds[:filter_seeds], table,
                                          nk=nk, omega_m=omega_m, net=nt, log=log)
        res["fit_s_" + name] = time.perf_counter() - t0
        res["cal_hist_" + name] = hist
        res["filters_" + name] = fl.tolist()
        nets_on.append((name, sim, fl, nt))
        extra_sims.append(sim)
    for base, nt in net_variants:
        _, sim, fl = next(e for e in extra if e[0] == base)
        t0 = time.perf_counter()
        h3 = train_online(nt, sim, fine, sched, train_seeds, table, lr=lr, epochs=epochs,
                          omega_m=omega_m, filters=fl, log=log)
        sim.set_force_filters(None)
        res["train_s_" + base + "_net"] = time.perf_counter() - t0
        res["loss_first_" + base + "_net"] = float(np.mean(h3[:10]))
        res["loss_last_" + base + "_net"] = float(np.mean(h3[-10:]))
        nets_on.append((base + "_net", sim, fl, nt))

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
        runs = []
        if filters is not None:
            runs.append(("filtered", coarse, filters, None))
            if net2 is not None:
                runs.append(("filtered_net", coarse, filters, net2))
        runs += [(name, sim, fl, None) for name, sim, fl in extra]
        runs += nets_on
        for name, sim, fl, nt in runs:
            sim.set_particles(p, sched.a_init, sched.a_init)
            s_x, t_x, w_x = timed_run(sim, sim.forces if fl is None and nt is None else
                                      (lambda s=sim, n=nt: n.forces(s)) if fl is None else
                                      filtered_force(sim, fl, nt))
            sim.set_force_filters(None)
            _, px, _ = power_spectrum_on(fine, s_x["x"], 1.0)
            mf_x = halo_counts(s_x, boxsize, nc)
            res["mf_" + name] = res.get("mf_" + name, 0) + mf_x
            r.update({name + "_s": t_x, name + "_wall_s": w_x,
                      "err_" + name: pk_error(k, px, pf, kmax), "halos_" + name: int(mf_x.sum())})
        res["seeds"].append(r)
        if log:
            log(str(r))
    fine.close()
    coarse.close()
    for _, sim, _ in extra:
        sim.close()
    for sim in extra_sims:
        sim.close()
    if "mf_fine" in res:
        for name in (["coarse", "learned", "filtered", "filtered_net"] + [e[0] for e in extra] +
                     [e[0] for e in nets_on]):
            if "mf_" + name in res:
                res["mf_err_" + name] = mf_ratio_error(res["mf_" + name], res["mf_fine"])
        for key in [k for k in res if k.startswith("mf_") and not k.startswith("mf_err")]:
            res[key] = [int(c) for c in res[key]]
    return res


def evaluate_large(nc, boxsize, sched, coarse_ngrid, fine_factor, train_seeds, eval_seeds, table,
                   *, nk=32, kernel=(0, 0, 2), iters=8, omega_m=0.273, log=None):
    """The large-run comparison: a coarse mesh with the calibrated Fourier
    correction (the CIC window divided out `kernel`[2] times and T(|n|) of
    nk knots calibrated on the final P(k) of the training seeds) against
    the plain run on the fine_factor mesh, which is the truth here, with
    the plain coarse run beside it.  Per held-out seed: the device time of
    each realization's time loop and the P(k) error up to half the particle
    Nyquist wavenumber.  Returns a dict of per-seed rows and the fit."""
    import time

    from .sim import Simulation
    fine = Simulation(nc, fine_factor * nc, boxsize, omega_m)
    sim = Simulation(nc, coarse_ngrid, boxsize, omega_m)
    sim.set_force_kernel(*kernel)
    t0 = time.perf_counter()
    fl, hist = calibrate_force_filter(sim, fine, sched, train_seeds, table, nk=nk, iters=iters,
                                      omega_m=omega_m, log=log)
    res = {"calibration_s": time.perf_counter() - t0, "calibration_train_err": hist,
           "filters_last_step": fl[-1].tolist(), "seeds": []}
    plain = Simulation(nc, coarse_ngrid, boxsize, omega_m)
    lib = _lib.load()
    nst = _lib.NSTAGES
    kmax = 0.5 * np.pi * nc / boxsize
    aout = output_scale_factors((0.0,))

    def timed(s, force):
        s.sync()
        _lib.check(lib.cg_prof_begin(64 * sched.nloop), "cg_prof_begin")
        run_time_loop(sched, aout, move=s.move, force=force, kick=s.kick, drift=s.drift,
                      snapshot=lambda a, i: None, kick_drift=s.kick_drift)
        ms = (ctypes.c_double * nst)()
        cnt = (ctypes.c_int * nst)()
        lib.cg_prof_end(ms, cnt, nst)
        return s.snapshot(aout[0]), sum(ms) / 1e3

    for seed in eval_seeds:
        p = _lpt_particles(nc, boxsize, seed, omega_m, sched.a_init, table)
        fine.set_particles(p, sched.a_init, sched.a_init)
        s_f, t_f = timed(fine, fine.forces)
        plain.set_particles(p, sched.a_init, sched.a_init)
        s_c, t_c = timed(plain, plain.forces)
        sim.set_particles(p, sched.a_init, sched.a_init)
        s_l, t_l = timed(sim, filtered_force(sim, fl))
        sim.set_force_filters(None)
        k, pf, _ = power_spectrum_on(fine, s_f["x"], 1.0)
        _, pc, _ = power_spectrum_on(fine, s_c["x"], 1.0)
        _, pl, _ = power_spectrum_on(fine, s_l["x"], 1.0)
        row = {"seed": seed, "fine_s": t_f, "coarse_s": t_c, "learned_s": t_l,
               "err_coarse": pk_error(k, pc, pf, kmax), "err_learned": pk_error(k, pl, pf, kmax)}
        res["seeds"].append(row)
        if log:
            log(str(row))
    for s in (fine, sim, plain):
        s.close()
    return res
