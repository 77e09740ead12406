"""The reference's own driver (main.c) on this library: the drop-in boundary
end to end.

oracle/Makefile (`make -C oracle drivers`) builds main.c and the files
around it twice from the reference sources: cola_halo_cpu with the
reference's hot path (the whole program on the host), and cola_halo_gpu
with pm.o, cola.o, lpt.o, power.o, move.o, fof.o, coarse_grid.o and
write_snapshot taken from libcolagpu.so.  Both run the same parameter file
(2LPT initial condition file, 10 COLA steps, outputs at z = 1 and 0 with
FoF catalogues, GADGET snapshots and coarse grids); their files are compared
here.  The GPU forces differ from the host's by float rounding, so particle
positions agree to about 1e-5 of the box and the catalogues to the halos
whose membership hangs on a pair at the linking length."""
import os
import subprocess

import numpy as np
import pytest

from cola_halo_b200.coarse import read_grid_file
from cola_halo_b200.gadget import read_gadget

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
L, NC, SEED = 64.0, 32, 100

PARAM = """nc = {nc}
boxsize = {L}
random_seed= {seed}
nrealization= {nreal}
ntimestep= 10
a_final= 1.0
output_redshifts= {{1.0, 0.0}}
omega_m = 0.273
h       = 0.705
sigma8  = 0.81
pm_nc_factor= 3
np_alloc_factor= 1.25
loglevel= 2
powerspectrum= "{table}"
fof= "fof"
linking_factor= 0.2
snapshot= "snp"
coarse_grid= "grid"
coarse_grid_nc= 16
initial= "init"
write_longid= {longid}
"""


def run_driver(exe, workdir, longid="false", nreal=1):
    os.makedirs(workdir, exist_ok=True)
    param = os.path.join(workdir, "param.txt")
    with open(param, "w") as f:
        f.write(PARAM.format(nc=NC, L=L, seed=SEED, longid=longid, nreal=nreal,
                             table=os.path.join(HERE, "golden", "bbks_table.dat")))
    r = subprocess.run([exe, param], cwd=workdir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, "%s failed (%d):\n%s\n%s" % (exe, r.returncode, r.stdout[-2000:],
                                                           r.stderr[-2000:])
    return r.stdout


@pytest.fixture(scope="module")
def outputs(tmp_path_factory):
    cpu = os.path.join(REF_DIR, "cola_halo_cpu")
    gpu = os.path.join(REF_DIR, "cola_halo_gpu")
    if not (os.path.exists(cpu) and os.path.exists(gpu)):
        pytest.skip("reference drivers not built (make -C oracle drivers)")
    base = tmp_path_factory.mktemp("driver")
    run_driver(cpu, str(base / "cpu"))
    log = run_driver(gpu, str(base / "gpu"))
    return str(base / "cpu"), str(base / "gpu"), log


def periodic_absdiff(a, b):
    d = np.abs(a.astype(np.float64) - b)
    return np.minimum(d, L - d)


def test_driver_writes_the_same_files(gpu_lib, outputs):
    cpu, gpu, log = outputs
    names = sorted(os.listdir(cpu))
    assert names == sorted(os.listdir(gpu))
    for n in ("init_%05d.0" % SEED, "snp%05da.0" % SEED, "snp%05db.0" % SEED,
              "fof%05da.txt" % SEED, "fof%05db.txt" % SEED, "grid%05da.b" % SEED,
              "grid%05db.b" % SEED):
        assert n in names
        assert os.path.getsize(os.path.join(gpu, n)) > 0
    assert "Total" in log          # the reference's timer_print ran to the end


def test_driver_snapshots_match(gpu_lib, outputs):
    cpu, gpu, _ = outputs
    for name, xtol in (("init_%05d.0", 1e-6), ("snp%05da.0", 1e-5), ("snp%05db.0", 1e-5)):
        hc, pc, vc, ic = read_gadget(os.path.join(cpu, name % SEED))
        hg, pg, vg, ig = read_gadget(os.path.join(gpu, name % SEED))
        # the header is computed from the same float fields: identical
        assert hc.tobytes() == hg.tobytes(), name
        # the reference's fof_find_halos leaves the snapshot in its k-d tree
        # order, the GPU finder in the particles' own order: compare by id
        oc, og = np.argsort(ic, kind="stable"), np.argsort(ig, kind="stable")
        np.testing.assert_array_equal(ig[og], ic[oc])
        pc, vc, pg, vg = pc[oc], vc[oc], pg[og], vg[og]
        assert periodic_absdiff(pg, pc).max() <= xtol * L, name
        # velocities carry the last kick's force difference; in the densest
        # halo it reaches ~2e-4 of the largest speed
        vs = np.abs(vc).max()
        dv = np.abs(vg.astype(np.float64) - vc)
        assert dv.max() <= 1e-3 * vs, name
        assert np.sqrt(np.mean(dv ** 2)) <= 1e-5 * vs, name


def test_driver_coarse_grids_match(gpu_lib, outputs):
    cpu, gpu, _ = outputs
    for s in "ab":
        Lc, dc = read_grid_file(os.path.join(cpu, "grid%05d%s.b" % (SEED, s)))
        Lg, dg = read_grid_file(os.path.join(gpu, "grid%05d%s.b" % (SEED, s)))
        assert Lc == Lg
        err = np.abs(dg.astype(np.float64) - dc) / (1.0 + np.abs(dc))
        assert err.max() <= 1e-3, err.max()


def test_driver_halo_catalogues_match(gpu_lib, outputs):
    cpu, gpu, _ = outputs
    for s in "ab":
        rc = np.loadtxt(os.path.join(cpu, "fof%05d%s.txt" % (SEED, s)), ndmin=2)
        rg = np.loadtxt(os.path.join(gpu, "fof%05d%s.txt" % (SEED, s)), ndmin=2)
        assert len(rc) > 0
        # membership of a few pairs at the linking length may flip
        assert abs(len(rg) - len(rc)) <= max(2, len(rc) // 50)
        assert abs(rg[:, 0].sum() - rc[:, 0].sum()) <= max(64, rc[:, 0].sum() // 50)
        # every catalogue halo has a partner of nearly the same mass at the
        # same place
        for h in rc[np.argsort(-rc[:, 0])][:20]:
            d = periodic_absdiff(rg[:, 1:4], h[1:4]).max(axis=1)
            j = int(np.argmin(d))
            assert d[j] <= 2e-3 * L
            assert abs(rg[j, 0] - h[0]) <= max(2, 0.02 * h[0])


def test_driver_two_realizations_with_long_ids(gpu_lib, outputs, tmp_path):
    """Two realizations in one process (seeds 100 and 101: the drop-in
    state is reused, the particles re-uploaded and the snapshot residency
    renewed) and 8-byte GADGET ids."""
    cpu = os.path.join(REF_DIR, "cola_halo_cpu")
    gpu = os.path.join(REF_DIR, "cola_halo_gpu")
    run_driver(cpu, str(tmp_path / "cpu"), longid="true", nreal=2)
    run_driver(gpu, str(tmp_path / "gpu"), longid="true", nreal=2)
    for seed in (SEED, SEED + 1):
        name = "snp%05db.0" % seed
        hc, pc, vc, ic = read_gadget(str(tmp_path / "cpu" / name))
        hg, pg, vg, ig = read_gadget(str(tmp_path / "gpu" / name))
        assert hc.tobytes() == hg.tobytes()
        assert ic.dtype == np.uint64 and ig.dtype == np.uint64
        oc, og = np.argsort(ic, kind="stable"), np.argsort(ig, kind="stable")
        np.testing.assert_array_equal(ig[og], ic[oc])
        assert periodic_absdiff(pg[og], pc[oc]).max() <= 1e-5 * L
        rc = np.loadtxt(str(tmp_path / "cpu" / ("fof%05db.txt" % seed)), ndmin=2)
        rg = np.loadtxt(str(tmp_path / "gpu" / ("fof%05db.txt" % seed)), ndmin=2)
        assert abs(len(rg) - len(rc)) <= max(2, len(rc) // 50)
    # the two seeds differ
    _, p0, _, i0 = read_gadget(str(tmp_path / "gpu" / ("snp%05db.0" % SEED)))
    _, p1, _, i1 = read_gadget(str(tmp_path / "gpu" / ("snp%05db.0" % (SEED + 1))))
    assert not np.array_equal(p0[np.argsort(i0)], p1[np.argsort(i1)])
