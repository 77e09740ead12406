"""The numpy friends-of-friends restatement against the reference's own
fof.c (shim build): compact clumps, halos across the periodic faces, and
the z = 0 snapshot of the 16^3 golden realization."""
import os

import numpy as np
import pytest

from oracle import restate as R
from cola_halo_b200.types import PARTICLE_MIN_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))


def clumps(L, nc, seed=1, centres=((50, 50, 50), (0.2, 99.9, 30), (99.8, 10, 0.1)), m=200,
           sigma=0.3):
    rng = np.random.default_rng(seed)
    pts = [rng.uniform(0, L, (nc ** 3 - m * len(centres), 3))]
    for c in centres:
        pts.append((np.array(c) + rng.normal(0, sigma, (m, 3))) % L)
    x = np.concatenate(pts).astype(np.float32)
    p = np.zeros(len(x), dtype=PARTICLE_MIN_DTYPE)
    p["x"] = x
    p["v"] = rng.normal(0, 100, (len(x), 3))
    p["id"] = np.arange(1, len(x) + 1)
    return p


def sort_rows(rows):
    rows = np.asarray(rows, dtype=np.float64).reshape(-1, 7)
    return rows[np.lexsort((rows[:, 3], rows[:, 2], rows[:, 1], rows[:, 0]))]


def assert_catalogs_match(got, want, L, pos_tol=1e-4, vel_tol=1e-4):
    got, want = sort_rows(got), sort_rows(want)
    assert len(got) == len(want)
    np.testing.assert_array_equal(got[:, 0], want[:, 0])
    d = np.abs(got[:, 1:4] - want[:, 1:4])
    d = np.minimum(d, L - d)                 # a centre may sit on either face
    assert d.max(initial=0) <= pos_tol * L
    vs = np.abs(want[:, 4:7]).max(initial=1.0)
    assert np.abs(got[:, 4:7] - want[:, 4:7]).max(initial=0) <= vel_tol * vs


def test_fof_restatement_matches_reference_on_clumps(ref, tmp_path):
    from oracle import ref as REF
    L, nc = 100.0, 16
    p = clumps(L, nc)
    ll = np.float32(0.2 * L / nc)
    want = REF.fof_catalog(p, L, nc, ll, str(tmp_path))
    got = R.fof_halos(p["x"], p["v"], L, ll)
    assert len(got) == 3
    assert_catalogs_match(got, want, L)


def test_fof_restatement_matches_reference_on_golden_snapshot(ref, tmp_path):
    from oracle import ref as REF
    g = np.load(os.path.join(HERE, "golden", "ref_nc16.npz"))
    nc, L = 16, 100.0
    p = np.zeros(len(g["snap_x"]), dtype=PARTICLE_MIN_DTYPE)
    p["x"], p["v"], p["id"] = g["snap_x"], g["snap_v"], g["snap_id"]
    for b in (0.2, 0.35):
        ll = np.float32(b * L / nc)
        want = REF.fof_catalog(p, L, nc, ll, str(tmp_path))
        got = R.fof_halos(p["x"], p["v"], L, ll)
        assert_catalogs_match(got, want, L)


def test_fof_restatement_edge_cases():
    L = np.float32(10.0)
    ll = np.float32(0.5)
    # exactly nfof_min along a chain through the x = 0 face, and one short of it
    chain = np.zeros((32, 3), dtype=np.float32)
    chain[:, 0] = (np.arange(32) * 0.4 - 6.0) % 10.0
    chain[:, 1:] = 5.0
    short = np.zeros((31, 3), dtype=np.float32)
    short[:, 1] = np.arange(31) * 0.3 % 10.0
    short[:, 0], short[:, 2] = 2.0, 8.0
    x = np.concatenate([chain, short])
    rows = R.fof_halos(x, np.zeros_like(x), L, ll)
    assert len(rows) == 1 and rows[0, 0] == 32
    # spacing exactly ll is not linked (strict inequality)
    pair = np.array([[1.0, 1.0, 1.0], [1.5, 1.0, 1.0]], dtype=np.float32)
    assert len(R.fof_halos(pair, np.zeros_like(pair), L, ll, nfof_min=2)) == 0
    assert len(R.fof_halos(np.zeros((0, 3), np.float32), np.zeros((0, 3)), L, ll)) == 0
