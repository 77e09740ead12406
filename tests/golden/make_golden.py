"""Regenerate the golden fixtures in this directory from the reference's own
C code (oracle/_ref/libcolaref.so, built from the reference sources against
the project's shims by oracle/Makefile).

    python tests/golden/make_golden.py

Writes
  ranlxd1.txt       first draws of gsl_rng_ranlxd1 (shim) for a few seeds
  bbks_table.dat    the BBKS input spectrum the fixtures were made with
  ref_nc16.npz      nc=16, 48^3 mesh, L=100 Mpc/h, seed 100, Omega_m=0.273,
                    reference schedule (10 steps): 2LPT particles, the
                    forces of the first step, and the z=0 snapshot
  ref_coarse_grid.npz  the reference's coarse_grid2 file contents (nc = 16)
                    of that z=0 snapshot

    python tests/golden/make_golden.py coarse    # only ref_coarse_grid.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cola_halo_b200.bbks import write_bbks_table  # noqa: E402
from cola_halo_b200.schedule import Schedule, output_scale_factors, run_time_loop  # noqa: E402
from cola_halo_b200.types import HostParticles, HostSnapshot  # noqa: E402
from oracle import ref as R  # noqa: E402

OM = 0.273


def main():
    lib = R.load()
    with open(os.path.join(HERE, "ranlxd1.txt"), "w") as f:
        f.write("# seed  first 24 draws of gsl_rng_ranlxd1 (oracle shim), repr of float64\n")
        for seed in (1, 100, 12345, 2147483647):
            f.write("%d %s\n" % (seed, " ".join(repr(v) for v in R.ranlxd1_stream(seed, 24))))
    table = write_bbks_table(os.path.join(HERE, "bbks_table.dat"))
    nc, factor, L, seed = 16, 3, 100.0, 100
    sched = Schedule.reference(10)
    lib.power_init(table.encode(), sched.a_init, 0.81, OM, 1 - OM)
    lib.comm_init(nc * factor, nc, L)
    lib.lpt_init(nc, None, 0)
    parts = HostParticles(nc)
    lib.lpt_set_displacement(sched.a_init, OM, seed, L, parts.ptr)
    ics = parts.local().copy()
    lib.pm_init(nc * factor, factor, L, 1.25, None, 0, None, 0)
    snap = HostSnapshot(nc, parts.struct.np_allocated, L, OM)
    parts.struct.a_v = sched.a_init
    forces = []

    def force():
        lib.pm_calculate_forces(parts.ptr)
        if not forces:
            forces.append(parts.force[: nc ** 3].copy())
    run_time_loop(sched, output_scale_factors([0.0]),
                  move=lambda: lib.move_particles2(parts.ptr, L, None, 0), force=force,
                  kick=lambda a: lib.cola_kick(parts.ptr, OM, a),
                  drift=lambda a: lib.cola_drift(parts.ptr, OM, a),
                  snapshot=lambda a, i: lib.cola_set_snapshot(a, parts.ptr, snap.ptr))
    s = snap.local()
    np.savez_compressed(os.path.join(HERE, "ref_nc16.npz"),
                        x0=ics["x"], dx1=ics["dx1"], dx2=ics["dx2"], id=ics["id"],
                        f0=forces[0], snap_x=s["x"], snap_v=s["v"], snap_id=s["id"],
                        meta=np.array([nc, factor, L, seed, OM, sched.a_init]))
    coarse_grid()


def coarse_grid():
    import tempfile
    g = np.load(os.path.join(HERE, "ref_nc16.npz"))
    L = float(g["meta"][2])
    snap = np.zeros(len(g["snap_x"]), dtype=R_pmin_dtype())
    snap["x"], snap["v"], snap["id"] = g["snap_x"], g["snap_v"], g["snap_id"]
    with tempfile.TemporaryDirectory() as d:
        Lf, delta = R.coarse_grid_file(snap, L, 16, os.path.join(d, "grid.bin"))
    np.savez_compressed(os.path.join(HERE, "ref_coarse_grid.npz"), delta=delta,
                        meta=np.array([16, Lf, len(snap)]))


def R_pmin_dtype():
    from cola_halo_b200.types import PARTICLE_MIN_DTYPE
    return PARTICLE_MIN_DTYPE


if __name__ == "__main__":
    if sys.argv[1:] == ["coarse"]:
        coarse_grid()
    else:
        main()
