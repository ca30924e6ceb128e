"""Parity with denser global key tables.  The library reads DFC_TABLE_FACTOR
(global-table slots per estimated group; 16 while the table fits 4 GiB, else
8) once per process, so each setting runs a selection of the parity tests in
a child process: 2 and 4 slots per group give probe chains several times
longer than the defaults, and the results must not change."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("factor", ["2", "4"])
def test_dense_key_tables(factor):
    env = dict(os.environ, DFC_TABLE_FACTOR=factor)
    cmd = [
        sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
        str(ROOT / "tests" / "test_gpu_parity.py"),
        "-k", "test_fixture or config2_reduced or aggregate_table_generator or regrow",
    ]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
