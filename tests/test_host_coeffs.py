"""The library's double-precision host coefficients (no GPU needed) vs the
restatement of cola.c:156-292 and power.c."""
import numpy as np
import pytest

from oracle import restate as R

OM = 0.273


@pytest.fixture(scope="module")
def lib():
    from cola_halo_b200 import _lib
    return _lib.load()


def test_growth(lib):
    ct = R.ColaTime(OM)
    for a in np.concatenate([np.linspace(0.02, 1.0, 40), [0.2, 0.2000001, 0.7174]]):
        assert lib.cg_growth_D1(OM, a) == pytest.approx(ct.D1(a), rel=1e-12)
        assert lib.cg_growth_D2(OM, a) == pytest.approx(ct.D2(a), rel=1e-12)


def test_sq_sphi(lib):
    ct = R.ColaTime(OM)
    for ai, af, ar in ((0.1, 0.2, 0.15), (0.02, 0.118, 0.069), (0.9, 1.0, 0.95)):
        assert lib.cg_cola_Sq(OM, ai, af, ar) == pytest.approx(ct.Sq(ai, af, ar), rel=1e-11)
        assert lib.cg_cola_Sphi(OM, ai, af, ar) == pytest.approx(ct.Sphi(ai, af, ar), rel=1e-14)


def test_kick_drift_coeffs(lib):
    from cola_halo_b200.sim import drift_coeffs, kick_coeffs
    ct = R.ColaTime(OM)
    for a_v, a_x, a1 in [(0.1, 0.1, 0.15), (0.15, 0.2, 0.25), (0.85, 0.9, 0.95)]:
        np.testing.assert_allclose(kick_coeffs(OM, a_v, a_x, a1), ct.kick_coeffs(a_v, a_x, a1),
                                   rtol=1.5e-7)
        np.testing.assert_allclose(drift_coeffs(OM, a_x, a_v, a1), ct.drift_coeffs(a_x, a_v, a1),
                                   rtol=1.5e-7)


def test_power_table_dropin(lib, bbks_table):
    lib.cg_dropin_set_abort(0)
    lib.power_init(bbks_table.encode(), 0.1, 0.81, OM, 1 - OM)
    pw = R.PowerTable(bbks_table)
    for k in (1e-3, 0.01, 0.2, 1.7, 50.0):
        assert lib.PowerSpec(k) == pytest.approx(float(pw(k)), rel=1e-12)
    assert lib.GrowthFactor(0.1, 1.0) == pytest.approx(R.growth_factor(0.1, 1.0, OM), rel=1e-10)


def test_power_init_sigma8_check(lib, bbks_table):
    """power.c:111-113: abort code 3010 when sigma_8 is >5% off (returns
    with an error message when aborts are disabled)."""
    lib.cg_dropin_set_abort(0)
    lib.power_init(bbks_table.encode(), 0.1, 0.9, OM, 1 - OM)
    assert b"sigma8" in lib.cg_last_error()
