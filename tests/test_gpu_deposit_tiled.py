"""The cell-sorted deposit (COLAGPU_DEPOSIT=tiled, deposit_tiled.cu) through
the same PM parity tests as the default atomic deposit.  The selection is
read once per process, so the PM tests run again in a child process."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pm_parity_with_tiled_deposit(gpu_lib):
    env = dict(os.environ, COLAGPU_DEPOSIT="tiled")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p",
                        "no:cacheprovider", "tests/test_gpu_pm.py", "tests/test_gpu_pk.py"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
