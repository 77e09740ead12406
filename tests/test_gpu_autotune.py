"""FFT schedule variants and the autotuner: every compiled variant of the
strided x pass and of the fused Green pass gives the same force meshes as
the default schedule (to float rounding), the default matches the oracle,
and cg_autotune times, installs and caches a choice."""
import ctypes
import os

import numpy as np
import pytest

from oracle import restate as R
from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu
OM = 0.273


def _variants(lib, n):
    g, f = ctypes.c_int(), ctypes.c_int()
    assert lib.cg_schedule_variants(n, ctypes.byref(g), ctypes.byref(f)) == 0
    return g.value, f.value


def _schedule(lib, n):
    g, f = ctypes.c_int(), ctypes.c_int()
    assert lib.cg_get_schedule(n, ctypes.byref(g), ctypes.byref(f)) == 0
    return g.value, f.value


def test_schedule_variants_match_default_and_oracle(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation
    nc, factor, L = 64, 4, 256.0
    N = nc * factor
    ng, nf = _variants(gpu_lib, N)
    assert ng == 7 and nf == 3
    p = lattice_particles(nc, L, 31, OM, 0.5, bbks_table)
    sim = Simulation(nc, N, L, OM)

    def meshes():
        sim.set_particles(p, 0.5, 0.5)
        sim.move()
        sim.forces()
        return [sim.get_mesh(1 + a).astype(np.float64) for a in range(3)], sim.get_forces()

    try:
        assert gpu_lib.cg_set_schedule(N, 0, 0) == 0
        base, fbase = meshes()
        x = R.wrap(p["x"], L)
        _, _, want = R.pm_force_meshes(x, N, L, factor)
        for a in range(3):
            assert np.abs(base[a] - want[a]).max() < 2e-5 * np.abs(want[a]).max()
        for g, f in [(1, 0), (2, 0), (3, 0), (4, 0), (5, 0), (6, 0), (0, 1), (0, 2), (2, 2),
                     (6, 2)]:
            assert gpu_lib.cg_set_schedule(N, g, f) == 0
            got, fgot = meshes()
            for a in range(3):
                scale = np.abs(base[a]).max()
                assert np.abs(got[a] - base[a]).max() < 1e-5 * scale, (g, f, a)
            assert np.abs(fgot - fbase).max() < 1e-5 * np.abs(fbase).max()
    finally:
        gpu_lib.cg_set_schedule(N, 0, 0)
        sim.close()


def test_schedule_arguments_checked(gpu_lib):
    assert _variants(gpu_lib, 128) == (1, 1)
    assert gpu_lib.cg_set_schedule(128, 1, 0) != 0
    assert gpu_lib.cg_set_schedule(256, 7, 0) != 0
    assert gpu_lib.cg_set_schedule(256, 0, -1) != 0
    assert gpu_lib.cg_set_schedule(100, 0, 0) != 0
    assert _variants(gpu_lib, 1024)[0] == 1      # 8-line Green variants stop at 768


def test_autotune_times_installs_and_caches(gpu_lib, tmp_path):
    import torch
    cache = tmp_path / "schedules.txt"
    old = os.environ.get("COLAGPU_TUNE_CACHE")
    os.environ["COLAGPU_TUNE_CACHE"] = str(cache)
    try:
        ng, nf = _variants(gpu_lib, 384)
        mg = (ctypes.c_float * ng)()
        mf = (ctypes.c_float * nf)()
        assert gpu_lib.cg_autotune(384, 1, mg, mf) == 0, gpu_lib.cg_last_error()
        g, f = _schedule(gpu_lib, 384)
        assert all(t > 0 for t in mg) and all(t > 0 for t in mf)
        assert g == int(np.argmin(list(mg))) and f == int(np.argmin(list(mf)))
        line = cache.read_text().strip().splitlines()[-1].split("\t")
        assert line[1:] == ["384", str(g), str(f)]
        # a cached entry is installed without timing
        dev = torch.cuda.get_device_name(0)
        with open(cache, "a") as fh:
            fh.write("%s\t512\t1\t2\n" % dev)
        assert gpu_lib.cg_autotune(512, 0, None, None) == 0
        assert _schedule(gpu_lib, 512) == (1, 2)
    finally:
        if old is None:
            os.environ.pop("COLAGPU_TUNE_CACHE", None)
        else:
            os.environ["COLAGPU_TUNE_CACHE"] = old
        gpu_lib.cg_set_schedule(384, 0, 0)
        gpu_lib.cg_set_schedule(512, 0, 0)
