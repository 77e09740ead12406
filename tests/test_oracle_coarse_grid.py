"""The numpy coarse-grid restatement against the reference's own
coarse_grid.c (shim build): uniform particles, particles on and past the
box faces, a one-cell grid and the z = 0 snapshot of the 16^3 golden
realization.  Both add in particle order in float32, so they agree bit for
bit."""
import os

import numpy as np

from oracle import restate as R
from cola_halo_b200.types import PARTICLE_MIN_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))


def pmin_of(x):
    p = np.zeros(len(x), dtype=PARTICLE_MIN_DTYPE)
    p["x"] = x
    p["id"] = np.arange(1, len(x) + 1)
    return p


def face_particles(L, nc):
    """Uniform particles plus ones exactly on the faces and cell edges, just
    below L, at L, and up to one cell outside the box on either side."""
    rng = np.random.default_rng(5)
    dx = L / nc
    special = np.array([0.0, L, np.nextafter(np.float32(L), np.float32(0)), -0.5 * dx,
                        -dx, L + 0.5 * dx, 3 * dx, 1e-7, -1e-7], dtype=np.float32)
    pts = [rng.uniform(0, L, (4000, 3))]
    for a in special:
        q = rng.uniform(0, L, (3, 3))
        q[:, 0], q[1, 1], q[2, 2] = a, a, a
        pts.append(q)
    return np.concatenate(pts).astype(np.float32)


def test_coarse_grid_restatement_matches_reference_uniform(ref, tmp_path):
    from oracle import ref as REF
    L = 100.0
    x = np.random.default_rng(2).uniform(0, L, (20000, 3)).astype(np.float32)
    for nc in (1, 4, 16, 24):
        Lf, want = REF.coarse_grid_file(pmin_of(x), L, nc, str(tmp_path / "g.bin"))
        got, total = R.coarse_grid(x, L, nc)
        assert Lf == np.float32(L) and want.shape == (nc, nc, nc)
        np.testing.assert_array_equal(got, want)
        assert abs(total - len(x)) < 1e-3 * len(x)


def test_coarse_grid_restatement_matches_reference_on_faces(ref, tmp_path):
    from oracle import ref as REF
    L = 64.0
    x = face_particles(L, 8)
    Lf, want = REF.coarse_grid_file(pmin_of(x), L, 8, str(tmp_path / "g.bin"))
    got, _ = R.coarse_grid(x, L, 8)
    np.testing.assert_array_equal(got, want)


def test_coarse_grid_restatement_matches_reference_np_total(ref, tmp_path):
    """nbar_inv comes from np_total, not the local count (coarse_grid.c:51)."""
    from oracle import ref as REF
    L = 50.0
    x = np.random.default_rng(3).uniform(0, L, (3000, 3)).astype(np.float32)
    Lf, want = REF.coarse_grid_file(pmin_of(x), L, 6, str(tmp_path / "g.bin"), np_total=2900)
    got, _ = R.coarse_grid(x, L, 6, np_total=2900)
    np.testing.assert_array_equal(got, want)


def test_coarse_grid_restatement_matches_reference_on_golden_snapshot(ref, tmp_path):
    from oracle import ref as REF
    g = np.load(os.path.join(HERE, "golden", "ref_nc16.npz"))
    L = 100.0
    x = g["snap_x"].astype(np.float32)
    for nc in (8, 16, 32):
        Lf, want = REF.coarse_grid_file(pmin_of(x), L, nc, str(tmp_path / "g.bin"))
        got, _ = R.coarse_grid(x, L, nc)
        np.testing.assert_array_equal(got, want)


def test_coarse_grid_restatement_properties():
    """Mass conservation and the uniform lattice: particles on cell corners
    give delta = 0 exactly."""
    L, nc = 32.0, 8
    g = (np.arange(nc, dtype=np.float32) * np.float32(L / nc))
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    d, total = R.coarse_grid(x, L, nc)
    assert total == nc ** 3
    np.testing.assert_array_equal(d, np.zeros_like(d))
    # each particle carries unit mass: the contrast averages to 0
    x = np.random.default_rng(4).uniform(-L, 2 * L, (5000, 3)).astype(np.float32)
    d, total = R.coarse_grid(x, L, nc)
    assert abs(total - 5000) < 1e-2
    assert abs(float(d.astype(np.float64).mean())) < 1e-5


def test_coarse_grid_restatement_matches_golden_fixture():
    """The committed reference output (tests/golden/make_golden.py coarse)."""
    g = np.load(os.path.join(HERE, "golden", "ref_coarse_grid.npz"))
    s = np.load(os.path.join(HERE, "golden", "ref_nc16.npz"))
    nc, L, n = int(g["meta"][0]), float(g["meta"][1]), int(g["meta"][2])
    got, total = R.coarse_grid(s["snap_x"], L, nc)
    np.testing.assert_array_equal(got, g["delta"])
    assert abs(total - n) < 1e-3 * n


def test_grid_file_reader_reads_the_reference_file(ref, tmp_path):
    """cola_halo_b200.coarse.read_grid_file on a file the reference's own
    coarse_grid2 wrote, and its rejection of a truncated file."""
    from oracle import ref as REF
    from cola_halo_b200.coarse import read_grid_file
    L = 80.0
    x = np.random.default_rng(9).uniform(0, L, (5000, 3)).astype(np.float32)
    path = str(tmp_path / "g.bin")
    _, want = REF.coarse_grid_file(pmin_of(x), L, 12, path)
    Lf, got = read_grid_file(path)
    assert Lf == np.float32(L)
    np.testing.assert_array_equal(got, want)
    raw = open(path, "rb").read()
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(raw[:-4])
    import pytest
    with pytest.raises(ValueError):
        read_grid_file(bad)
