"""GPU coarse density grid (cg_coarse_grid and the drop-in coarse_grid2)
against the reference's own coarse_grid.c output (committed fixture and,
where the shim build is present, the reference run here) and the numpy
restatement.  The GPU adds the CIC weights with float atomics in any order
and the reference in particle order, so a cell's density differs by float
rounding of its sum: |delta_gpu - delta_ref| <= 1e-5 (1 + |delta_ref|)."""
import ctypes
import os

import numpy as np
import pytest

from oracle import restate as R
from tests.test_oracle_coarse_grid import face_particles, pmin_of
from cola_halo_b200.types import PARTICLE_MIN_DTYPE

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
OM = 0.273
RTOL = 1e-5


def assert_grid_close(got, want):
    assert got.shape == want.shape and got.dtype == np.float32
    err = np.abs(got.astype(np.float64) - want) / (1.0 + np.abs(want.astype(np.float64)))
    assert err.max(initial=0) <= RTOL, err.max()


def test_coarse_grid_matches_golden_fixture(gpu_lib):
    from cola_halo_b200.coarse import coarse_grid
    g = np.load(os.path.join(HERE, "golden", "ref_coarse_grid.npz"))
    s = np.load(os.path.join(HERE, "golden", "ref_nc16.npz"))
    nc, L, n = int(g["meta"][0]), float(g["meta"][1]), int(g["meta"][2])
    p = np.zeros(n, dtype=PARTICLE_MIN_DTYPE)
    p["x"], p["v"], p["id"] = s["snap_x"], s["snap_v"], s["snap_id"]
    delta, total = coarse_grid(p, L, nc)
    assert_grid_close(delta, g["delta"])
    assert abs(total - n) < 1e-3 * n


@pytest.mark.parametrize("nc", [7, 16, 25, 26, 64, 128])
def test_coarse_grid_matches_restatement_uniform(gpu_lib, nc):
    from cola_halo_b200.coarse import coarse_grid
    L = 250.0
    x = np.random.default_rng(nc).uniform(0, L, (200000, 3)).astype(np.float32)
    delta, total = coarse_grid(pmin_of(x), L, nc)
    want, want_total = R.coarse_grid(x, L, nc)
    assert_grid_close(delta, want)
    assert abs(total - want_total) <= 1e-5 * len(x)


def test_coarse_grid_single_cell(gpu_lib):
    """nc = 1: one cell holds all 8 n weights.  The reference's running
    float sum of 1.6e6 terms drifts by ~8e-4 (199846 instead of 200000);
    the GPU sums per CTA first, so it is checked against the float64 sum of
    the same float weights instead."""
    from cola_halo_b200.coarse import coarse_grid
    L = 250.0
    x = np.random.default_rng(1).uniform(0, L, (200000, 3)).astype(np.float32)
    delta, total = coarse_grid(pmin_of(x), L, 1)
    s = x * (np.float32(1) / np.float32(L))
    w = np.float32(1) - (s - np.floor(s))
    u = np.float32(1) - w
    exact = 0.0
    for a in (w, u):
        for b in (w, u):
            for c in (w, u):
                exact += float(np.sum((a[:, 0] * b[:, 1]) * c[:, 2], dtype=np.float64))
    assert abs(total - exact) <= 1e-5 * exact
    want = np.float32(1.0 / len(x)) * np.float32(exact) - np.float32(1)
    assert abs(float(delta[0, 0, 0]) - float(want)) <= 1e-5


def test_coarse_grid_faces_and_np_total(gpu_lib):
    from cola_halo_b200.coarse import coarse_grid
    L = 64.0
    x = face_particles(L, 8)
    delta, _ = coarse_grid(pmin_of(x), L, 8)
    assert_grid_close(delta, R.coarse_grid(x, L, 8)[0])
    delta, _ = coarse_grid(pmin_of(x), L, 8, np_total=len(x) + 123)
    assert_grid_close(delta, R.coarse_grid(x, L, 8, np_total=len(x) + 123)[0])
    # far outside the box (the reference's index is undefined there): the
    # grid stays in bounds and keeps every particle's mass
    far = np.array([[-3.5 * L, 0.5, 0.5], [7.25 * L, 1.0, 2.0], [1.0, -1e6, 1e6]], np.float32)
    delta, total = coarse_grid(pmin_of(far), L, 8)
    assert abs(total - 3.0) < 1e-5


def test_coarse_grid_matches_reference_and_device_input(gpu_lib, ref, bbks_table, tmp_path):
    import torch
    from oracle import ref as REF
    from cola_halo_b200 import Simulation
    from cola_halo_b200.coarse import coarse_grid
    from cola_halo_b200.schedule import Schedule
    from tests.helpers import lattice_particles
    nc, L = 64, 64.0
    sim = Simulation(nc, 3 * nc, L, OM)
    sim.set_particles(lattice_particles(nc, L, 11, OM, 0.05, bbks_table), 0.05, 0.05)
    snap = sim.run(Schedule.linear(0.05, 1.0, 10))[-1][1]
    sim.close()
    for ncg in (16, 32, 64):
        _, want = REF.coarse_grid_file(snap, L, ncg, str(tmp_path / "g.bin"))
        got, _ = coarse_grid(snap, L, ncg)
        assert_grid_close(got, want)
    # device particles in, device grid out
    d = torch.from_numpy(snap.view(np.uint8).copy()).cuda()
    out = torch.empty(32 ** 3, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    res, total = coarse_grid(d.data_ptr(), L, 32, np_count=len(snap), out=out.data_ptr())
    assert res is None
    got = out.cpu().numpy().reshape(32, 32, 32)
    assert_grid_close(got, coarse_grid(snap, L, 32)[0])
    assert abs(total - len(snap)) < 1e-3 * len(snap)


def test_dropin_coarse_grid2_writes_the_reference_file(gpu_lib, tmp_path):
    from cola_halo_b200.coarse import read_grid_file
    from cola_halo_b200.types import HostSnapshot
    g = np.load(os.path.join(HERE, "golden", "ref_coarse_grid.npz"))
    s = np.load(os.path.join(HERE, "golden", "ref_nc16.npz"))
    nc, L, n = int(g["meta"][0]), float(g["meta"][1]), int(g["meta"][2])
    snap = HostSnapshot(16, n, L, OM)
    snap.p["x"], snap.p["v"], snap.p["id"] = s["snap_x"], s["snap_v"], s["snap_id"]
    snap.struct.np_local = n
    gpu_lib.cg_dropin_set_abort(0)
    path = str(tmp_path / "grid_gpu.bin")
    size = 4 * nc * nc * (nc + 16)
    gpu_lib.coarse_grid2(path.encode(), snap.ptr, nc, None, size)
    assert os.path.getsize(path) == 12 + 4 * nc ** 3
    Lf, delta = read_grid_file(path)
    assert Lf == np.float32(L)
    assert_grid_close(delta, g["delta"])
    # unwritable file: the reference's code 10021 path, as a return
    gpu_lib.coarse_grid2(str(tmp_path / "no_such_dir" / "g.bin").encode(), snap.ptr, nc, None,
                         size)
    assert b"Unable to write grid" in gpu_lib.cg_last_error()


def test_coarse_grid_bad_arguments(gpu_lib):
    total = ctypes.c_double()
    out = np.zeros(8, np.float32)
    p = pmin_of(np.ones((4, 3), np.float32))
    assert gpu_lib.cg_coarse_grid(None, 4, 4, 10.0, 2, out.ctypes.data, ctypes.byref(total)) != 0
    assert gpu_lib.cg_coarse_grid(p.ctypes.data, 4, 0, 10.0, 2, out.ctypes.data, None) != 0
    assert gpu_lib.cg_coarse_grid(p.ctypes.data, 4, 4, 0.0, 2, out.ctypes.data, None) != 0
    assert gpu_lib.cg_coarse_grid(p.ctypes.data, 4, 4, 10.0, 0, out.ctypes.data, None) != 0
    # no particles: an empty box, delta = -1 everywhere
    assert gpu_lib.cg_coarse_grid(None, 0, 4, 10.0, 2, out.ctypes.data, ctypes.byref(total)) == 0
    np.testing.assert_array_equal(out, -np.ones(8, np.float32))
    assert total.value == 0.0
