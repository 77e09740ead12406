import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def bbks_table(tmp_path_factory):
    from cola_halo_b200.bbks import write_bbks_table
    p = tmp_path_factory.mktemp("tables") / "bbks.dat"
    return str(write_bbks_table(str(p)))


@pytest.fixture(scope="session")
def ref():
    """The reference's own C code built against the oracle shims."""
    from oracle import ref as R
    if not os.path.exists(R.LIB_PATH):
        try:
            R.build()
        except Exception as e:  # pragma: no cover
            pytest.skip("reference build unavailable: %s" % e)
    if not os.path.exists(R.LIB_PATH):
        pytest.skip("oracle/_ref/libcolaref.so not built (needs the reference sources)")
    return R.load()


@pytest.fixture(scope="session")
def gpu_lib():
    from cola_halo_b200 import _lib
    lib = _lib.load()
    if lib.cg_device_count() < 1:
        pytest.skip("no CUDA device")
    return lib
