"""GPU GADGET-1 writer (cg_write_gadget, cg_sim_write_gadget and the
drop-in write_snapshot) against the numpy restatement, which is pinned byte
for byte to the reference's own write.c (test_oracle_gadget.py).  The files
must be identical byte for byte.  Also the drop-in snapshot residency:
fof_find_halos, write_snapshot and coarse_grid2 read the device copy that
cola_set_snapshot leaves, and the host copy stays in step with it."""
import ctypes
import os

import numpy as np
import pytest

from oracle import restate as R
from tests.test_oracle_gadget import snapshot_particles
from cola_halo_b200.types import PARTICLE_MIN_DTYPE

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
OM = 0.273


def expected(p, a, L, om, h, long_id=False, np_total=None):
    return R.gadget_bytes(p["x"], p["v"], p["id"], a, L, om, h, use_long_id=long_id,
                          np_total=np_total)


@pytest.mark.parametrize("n", [0, 1, 1000, (1 << 20), (1 << 20) + 1, 2500000])
def test_write_gadget_host_input_matches_restatement(gpu_lib, tmp_path, n):
    """Chunk edges: one particle, exactly one chunk, one past it, and three
    chunks with a ragged end."""
    from cola_halo_b200.gadget import write_gadget
    L, a, h = 300.0, 0.61, 0.705
    p = snapshot_particles(n, L, seed=n % 97)
    for long_id in (False, True):
        path = str(tmp_path / "snap.0")
        write_gadget(path, p, a, L, OM, h, use_long_id=long_id)
        assert open(path, "rb").read() == expected(p, a, L, OM, h, long_id)


def test_write_gadget_device_input_and_np_total(gpu_lib, tmp_path):
    import torch
    from cola_halo_b200.gadget import read_gadget, write_gadget
    L, a, h = 150.0, 0.25, 0.7
    p = snapshot_particles(1500000, L, seed=11)
    p["id"][:4] = [2 ** 32 + 1, 2 ** 33 + 7, 2 ** 62, 0]
    d = torch.from_numpy(p.view(np.uint8).copy()).cuda()
    torch.cuda.synchronize()
    for long_id in (False, True):
        path = str(tmp_path / "dev.0")
        write_gadget(path, d.data_ptr(), a, L, OM, h, use_long_id=long_id, np_count=len(p),
                     np_total=8 * len(p), num_files=8)
        want = R.gadget_bytes(p["x"], p["v"], p["id"], a, L, OM, h, use_long_id=long_id,
                              np_total=8 * len(p), num_files=8)
        assert open(path, "rb").read() == want
    hdr, pos, vel, ids = read_gadget(path)
    assert hdr["np_total"][1] == 8 * len(p) and hdr["num_files"] == 8
    np.testing.assert_array_equal(ids, p["id"].astype(np.uint64))


def test_sim_write_gadget_matches_snapshot(gpu_lib, bbks_table, tmp_path):
    from cola_halo_b200 import Simulation
    from cola_halo_b200.schedule import Schedule
    from tests.helpers import lattice_particles
    nc, L, h = 32, 100.0, 0.68
    sim = Simulation(nc, 3 * nc, L, OM)
    sim.set_particles(lattice_particles(nc, L, 5, OM, 0.05, bbks_table), 0.05, 0.05)
    snap = sim.run(Schedule.linear(0.05, 1.0, 6))[-1][1]
    path = str(tmp_path / "sim.0")
    sim.write_gadget(path, 1.0, h=h, use_long_id=True)
    assert open(path, "rb").read() == expected(snap, 1.0, L, OM, h, True)
    sim.close()


def test_dropin_output_sequence_reads_the_device_snapshot(gpu_lib, bbks_table, tmp_path):
    """main.c's output step (main.c:346-382): cola_set_snapshot, then
    fof_find_halos (wraps positions), write_snapshot and coarse_grid2, all
    through the drop-in entry points."""
    from cola_halo_b200.coarse import read_grid_file
    from cola_halo_b200.schedule import Schedule, output_scale_factors, run_time_loop
    from cola_halo_b200.types import HostParticles, HostSnapshot
    from tests.helpers import lattice_particles
    from tests.test_gpu_coarse_grid import assert_grid_close
    lib = gpu_lib
    nc, factor, L = 32, 3, 64.0
    # an output between steps (z = 1, a = 0.5): the snapshot drifts the
    # particles from the last wrap to aout, carrying some across the faces,
    # so the wrap has work to do (at a z = 0 output on a step boundary it
    # has none)
    sched = Schedule.linear(0.05, 1.0, 3)
    lib.cg_dropin_set_abort(0)
    lib.pm_init(nc * factor, factor, L, 1.25, None, 0, None, 0)
    parts = HostParticles(nc)
    parts.p[: nc ** 3] = lattice_particles(nc, L, 21, OM, 0.05, bbks_table)
    parts.struct.np_local = nc ** 3
    parts.struct.a_x = parts.struct.a_v = 0.05
    snap = HostSnapshot(nc, parts.struct.np_allocated, L, OM)
    seen = {}

    def output(a, i):
        lib.cola_set_snapshot(a, parts.ptr, snap.ptr)
        raw = snap.local().copy()
        lib.fof_find_halos(snap.ptr, np.float32(0.2 * L / nc))
        wrapped = snap.local().copy()
        base = str(tmp_path / "snp")
        lib.write_snapshot(base.encode(), snap.ptr, 0)
        grid = str(tmp_path / "grid.b")
        lib.coarse_grid2(grid.encode(), snap.ptr, 16, None, 0)
        seen.update(raw=raw, wrapped=wrapped, base=base, grid=grid, a=snap.struct.a)
    run_time_loop(sched, output_scale_factors([1.0]),
                  move=lambda: lib.move_particles2(parts.ptr, L, None, 0),
                  force=lambda: lib.pm_calculate_forces(parts.ptr),
                  kick=lambda a: lib.cola_kick(parts.ptr, OM, a),
                  drift=lambda a: lib.cola_drift(parts.ptr, OM, a), snapshot=output)
    assert seen, lib.cg_last_error()
    raw, wrapped = seen["raw"], seen["wrapped"]
    # the host copy was wrapped as move_particles2_min wraps (move.c:33-41)
    x = raw["x"].copy()
    L32 = np.float32(L)
    x = np.where(x < 0, x + L32, np.where(x >= L32, x - L32, x)).astype(np.float32)
    assert (raw["x"] != x).any(), "no particle left the box: the wrap went untested"
    np.testing.assert_array_equal(wrapped["x"], x)
    np.testing.assert_array_equal(wrapped["v"], raw["v"])
    # write_snapshot and coarse_grid2 read the (wrapped) device copy: the
    # same bytes as the host copy gives
    got = open(seen["base"] + ".0", "rb").read()
    assert got == expected(wrapped, seen["a"], L, OM, snap.struct.h)
    _, delta = read_grid_file(seen["grid"])
    assert_grid_close(delta, R.coarse_grid(wrapped["x"], L, 16)[0])
    # a host edit after cg_snapshot_invalidate reaches the next write
    snap.p["v"][:10] *= 2
    lib.cg_snapshot_invalidate()
    lib.write_snapshot(seen["base"].encode(), snap.ptr, 1)
    assert open(seen["base"] + ".0", "rb").read() == expected(snap.local(), seen["a"], L, OM,
                                                                snap.struct.h, True)
    lib.cg_dropin_finalize()


def test_write_gadget_errors(gpu_lib, tmp_path):
    from cola_halo_b200.types import HostSnapshot
    p = snapshot_particles(10, 10.0)
    bad = str(tmp_path / "no_such_dir" / "x.0").encode()
    assert gpu_lib.cg_write_gadget(bad, p.ctypes.data, 10, 10, 1, 1.0, 10.0, 0.3, 0.7, 0) == -7
    assert gpu_lib.cg_write_gadget(bad, None, 10, 10, 1, 1.0, 10.0, 0.3, 0.7, 0) == -1
    assert gpu_lib.cg_write_gadget(b"/dev/null", p.ctypes.data, 10, 10, 1, 0.0, 10.0, 0.3, 0.7,
                                   0) == -1
    snap = HostSnapshot(4, 10, 10.0, 0.3)
    snap.p[:] = p
    snap.struct.np_local = 10
    snap.struct.a = 1.0
    gpu_lib.cg_dropin_set_abort(0)
    gpu_lib.cg_snapshot_invalidate()
    gpu_lib.write_snapshot(str(tmp_path / "no_such_dir" / "s").encode(), snap.ptr, 0)
    assert b"Unable to write to file" in gpu_lib.cg_last_error()
