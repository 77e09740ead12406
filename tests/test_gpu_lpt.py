"""2LPT initial conditions on the GPU (drop-in lpt_set_displacement) vs the
shim-built reference lpt.c with the same RANLUX seeds."""
import numpy as np
import pytest

from cola_halo_b200.types import HostParticles
from tests.helpers import periodic_diff

pytestmark = pytest.mark.gpu

OM = 0.273


@pytest.mark.parametrize("nc,L,seed", [(16, 100.0, 100), (32, 200.0, 1), (64, 200.0, 100)])
def test_lpt_matches_reference(gpu_lib, ref, bbks_table, nc, L, seed):
    a0 = 0.1
    ref.power_init(bbks_table.encode(), a0, 0.81, OM, 1 - OM)
    ref.lpt_init(nc, None, 0)
    pr = HostParticles(nc)
    ref.lpt_set_displacement(a0, OM, seed, L, pr.ptr)
    want = pr.local()

    lib = gpu_lib
    lib.cg_dropin_set_abort(0)
    lib.power_init(bbks_table.encode(), a0, 0.81, OM, 1 - OM)
    lib.lpt_init(nc, None, 0)
    pg = HostParticles(nc)
    assert lib.lpt_set_displacement(a0, OM, seed, L, pg.ptr) == 0, lib.cg_last_error()
    got = pg.local()
    assert pg.struct.np_local == nc ** 3
    assert abs(pg.struct.a_x - a0) < 1e-7 and pg.struct.a_v == 0.0
    np.testing.assert_array_equal(got["id"], want["id"])
    for k in ("dx1", "dx2"):
        scale = np.abs(want[k]).max()
        assert np.abs(got[k] - want[k]).max() < 2e-5 * scale, k
    assert periodic_diff(got["x"], want["x"], L).max() < 2e-6 * L
    assert np.all(got["v"] == 0)
    # PowerSpec / GrowthFactor of the drop-in power.c replacement
    for k in (0.01, 0.1, 1.0, 3.0):
        assert abs(lib.PowerSpec(k) / ref.PowerSpec(k) - 1) < 1e-12
    assert abs(lib.GrowthFactor(a0, 1.0) / ref.GrowthFactor(a0, 1.0) - 1) < 1e-7
