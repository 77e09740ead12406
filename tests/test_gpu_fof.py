"""GPU friends-of-friends (cg_fof and the drop-in fof_find_halos /
fof_write_halos) against the reference's own fof.c (shim build) and the
numpy restatement: clumps across the periodic faces, the golden 16^3
snapshot, and the z = 0 snapshot of a 64^3 COLA run."""
import ctypes
import os

import numpy as np
import pytest

from oracle import restate as R
from tests.test_oracle_fof import assert_catalogs_match, clumps
from cola_halo_b200.types import PARTICLE_MIN_DTYPE

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
OM = 0.273


def rows(h):
    return np.column_stack([h["nfof"], h["x"], h["v"]]).astype(np.float64)


def many_clumps(L=100.0, nc=32, n_clumps=60, seed=4):
    """Clumps of 10 .. 400 particles, several across the faces of the box."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, L, (n_clumps, 3))
    centres[:6, 0] = rng.choice([0.05, L - 0.05], 6)
    centres[6:10, 1:] = 0.02
    sizes = rng.integers(10, 400, n_clumps)
    pts = [rng.uniform(0, L, (nc ** 3 - sizes.sum(), 3))]
    for c, m in zip(centres, sizes):
        pts.append((c + rng.normal(0, 0.15, (m, 3))) % L)
    x = np.concatenate(pts).astype(np.float32)
    p = np.zeros(len(x), dtype=PARTICLE_MIN_DTYPE)
    p["x"] = x
    p["v"] = rng.normal(0, 300, (len(x), 3))
    p["id"] = np.arange(1, len(x) + 1)
    return p


def test_fof_matches_reference_on_clumps(gpu_lib, ref, tmp_path):
    from oracle import ref as REF
    from cola_halo_b200.halos import fof
    for p, L, nc in [(clumps(100.0, 16), 100.0, 16), (many_clumps(), 100.0, 32)]:
        ll = np.float32(0.2 * L / nc)
        got = fof(p, L, ll)
        want = REF.fof_catalog(p, L, nc, ll, str(tmp_path))
        assert len(want) >= 3
        assert_catalogs_match(rows(got), want, L)
        assert_catalogs_match(rows(got), R.fof_halos(p["x"], p["v"], L, ll), L)
        # fixed order: by each group's smallest particle index, so repeatable
        again = fof(p, L, ll)
        np.testing.assert_array_equal(got["nfof"], again["nfof"])


def test_fof_matches_reference_on_golden_snapshot(gpu_lib, ref, tmp_path):
    from oracle import ref as REF
    from cola_halo_b200.halos import fof
    g = np.load(os.path.join(HERE, "golden", "ref_nc16.npz"))
    p = np.zeros(len(g["snap_x"]), dtype=PARTICLE_MIN_DTYPE)
    p["x"], p["v"], p["id"] = g["snap_x"], g["snap_v"], g["snap_id"]
    for b in (0.2, 0.35):
        ll = np.float32(b * 100.0 / 16)
        want = REF.fof_catalog(p, 100.0, 16, ll, str(tmp_path))
        assert_catalogs_match(rows(fof(p, 100.0, ll)), want, 100.0)


def test_fof_on_cola_snapshot_and_device_input(gpu_lib, ref, bbks_table, tmp_path):
    import torch
    from oracle import ref as REF
    from cola_halo_b200 import Simulation
    from cola_halo_b200.halos import fof
    from cola_halo_b200.schedule import Schedule
    from tests.helpers import lattice_particles
    nc, L = 64, 64.0
    sim = Simulation(nc, 3 * nc, L, OM)
    sim.set_particles(lattice_particles(nc, L, 7, OM, 0.05, bbks_table), 0.05, 0.05)
    snap = sim.run(Schedule.linear(0.05, 1.0, 10))[-1][1]
    sim.close()
    ll = np.float32(0.2 * L / nc)
    got = fof(snap, L, ll)
    want = REF.fof_catalog(snap, L, nc, ll, str(tmp_path))
    assert len(want) > 20
    assert_catalogs_match(rows(got), want, L)
    # the same particles from device memory
    d = torch.from_numpy(snap.view(np.uint8).copy()).cuda()
    torch.cuda.synchronize()
    dev = fof(d.data_ptr(), L, ll, np_count=len(snap))
    np.testing.assert_array_equal(dev["nfof"], got["nfof"])
    np.testing.assert_allclose(dev["x"], got["x"], atol=1e-5 * L)


def test_dropin_fof_writes_the_reference_catalogue(gpu_lib, ref, tmp_path):
    from oracle import ref as REF
    from cola_halo_b200.types import HostSnapshot
    L, nc = 100.0, 32
    p = many_clumps(L, nc, seed=9)
    # some positions just outside the box, wrapped in place as the reference does
    p["x"][:50, 0] -= np.float32(L)
    ll = np.float32(0.2 * L / nc)
    want = REF.fof_catalog(p, L, nc, ll, str(tmp_path))
    snap = HostSnapshot(nc, len(p), L, OM)
    snap.p[:] = p
    snap.struct.np_local = len(p)
    gpu_lib.cg_dropin_set_abort(0)
    gpu_lib.fof_init(len(p), nc, None, gpu_lib.fof_calc_memory(len(p), nc))
    gpu_lib.fof_find_halos(snap.ptr, ll)
    assert (snap.p["x"][:50, 0] >= 0).all()
    path = str(tmp_path / "fof_gpu.txt")
    gpu_lib.fof_write_halos(path.encode())
    got = np.loadtxt(path, ndmin=2)
    assert_catalogs_match(got, want, L)


def test_fof_edge_cases(gpu_lib):
    from cola_halo_b200.halos import fof
    L, ll = np.float32(10.0), np.float32(0.5)
    chain = np.zeros(32 + 31, dtype=PARTICLE_MIN_DTYPE)
    chain["x"][:32, 0] = (np.arange(32) * 0.4 - 6.0) % 10.0
    chain["x"][:32, 1:] = 5.0
    chain["x"][32:, 1] = np.arange(31) * 0.3 % 10.0
    chain["x"][32:, 0], chain["x"][32:, 2] = 2.0, 8.0
    h = fof(chain, L, ll)
    assert len(h) == 1 and h["nfof"][0] == 32
    assert 0 <= h["x"][0, 0] < L
    pair = np.zeros(2, dtype=PARTICLE_MIN_DTYPE)
    pair["x"] = [[1.0, 1.0, 1.0], [1.5, 1.0, 1.0]]      # exactly ll apart: not linked
    assert len(fof(pair, L, ll, nfof_min=2)) == 0
    assert len(fof(np.zeros(0, dtype=PARTICLE_MIN_DTYPE), L, ll)) == 0
    blob = np.zeros(5000, dtype=PARTICLE_MIN_DTYPE)      # one group of everything
    blob["x"] = np.random.default_rng(0).uniform(4.9, 5.1, (5000, 3))
    h = fof(blob, L, ll)
    assert len(h) == 1 and h["nfof"][0] == 5000
    n = ctypes.c_longlong()
    assert gpu_lib.cg_fof(None, 10, 10.0, 0.5, 32, None, 0, ctypes.byref(n)) != 0
    assert gpu_lib.cg_fof(blob.ctypes.data, 5000, -1.0, 0.5, 32, None, 0, ctypes.byref(n)) != 0
