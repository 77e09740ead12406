"""The numpy GADGET-1 restatement against the reference's own write.c
(shim build): 4- and 8-byte ids, ids above 2^32, an empty snapshot, and the
z = 0 snapshot of the 16^3 golden realization -- byte for byte."""
import os

import numpy as np

from oracle import restate as R
from cola_halo_b200.types import PARTICLE_MIN_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))


def snapshot_particles(n, L, seed=3):
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=PARTICLE_MIN_DTYPE)
    p["x"] = rng.uniform(0, L, (n, 3))
    p["v"] = rng.normal(0, 400, (n, 3))
    p["id"] = rng.permutation(n) + 1
    return p


def test_gadget_restatement_matches_reference(ref, tmp_path):
    from oracle import ref as REF
    L, om, h, a = 250.0, 0.273, 0.705, 0.37
    p = snapshot_particles(5000, L)
    p["id"][:3] = [2 ** 32 + 5, 2 ** 40, -1]          # truncated to 4 bytes, or kept
    for long_id in (0, 1):
        want = REF.gadget_file(p, L, om, h, a, str(tmp_path / ("r%d" % long_id)), long_id)
        got = R.gadget_bytes(p["x"], p["v"], p["id"], a, L, om, h, use_long_id=long_id)
        assert got == want
        assert len(got) == 4 * 8 + 256 + 5000 * (24 + (8 if long_id else 4))


def test_gadget_restatement_matches_reference_empty_and_golden(ref, tmp_path):
    from oracle import ref as REF
    p = np.zeros(0, dtype=PARTICLE_MIN_DTYPE)
    want = REF.gadget_file(p, 100.0, 0.3, 0.7, 1.0, str(tmp_path / "e"), 0)
    assert R.gadget_bytes(p["x"], p["v"], p["id"], 1.0, 100.0, 0.3, 0.7) == want
    g = np.load(os.path.join(HERE, "golden", "ref_nc16.npz"))
    q = np.zeros(len(g["snap_x"]), dtype=PARTICLE_MIN_DTYPE)
    q["x"], q["v"], q["id"] = g["snap_x"], g["snap_v"], g["snap_id"]
    want = REF.gadget_file(q, 100.0, 0.273, 0.705, 1.0, str(tmp_path / "g"), 0)
    assert R.gadget_bytes(q["x"], q["v"], q["id"], 1.0, 100.0, 0.273, 0.705) == want


def test_gadget_reader_round_trip(tmp_path):
    from cola_halo_b200.gadget import read_gadget
    L, a = 64.0, 0.5
    p = snapshot_particles(1000, L)
    path = tmp_path / "s.0"
    path.write_bytes(R.gadget_bytes(p["x"], p["v"], p["id"], a, L, 0.3, 0.7, use_long_id=True))
    hdr, pos, vel, ids = read_gadget(str(path))
    assert hdr["np"][1] == 1000 and hdr["np_total"][1] == 1000 and hdr["num_files"] == 1
    assert hdr["time"] == np.float32(a) and hdr["boxsize"] == L
    np.testing.assert_array_equal(pos, p["x"])
    np.testing.assert_array_equal(vel, np.float32(1 / np.sqrt(np.float32(a))) * p["v"])
    np.testing.assert_array_equal(ids, p["id"].astype(np.uint64))
