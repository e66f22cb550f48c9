"""The bounds-checking build (libgdock_check.so: the kernel source compiled
with -DGD_CHECK, every instrumented shared- and global-memory index compared
with its array's length) on small cases against the FP64 oracle, at several
tile shapes; a child process loads it (tests/check_worker.py).  No index may
leave its array, results must stay within the parity tolerance, and replica
groupings of one tile shape must give identical bytes."""

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_bounds_checked_small_cases(lib):
    from geauxdock_b200 import build

    assert build.CHECK_LIB.exists()
    env = dict(os.environ, GDOCK_LIB=str(build.CHECK_LIB))
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "check_worker.py")], capture_output=True, text=True,
                       timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    assert d["cases"] >= 50
    assert d["violations"] == [], d["violations"][:5]
    assert d["raced"] == [], d["raced"][:5]
    assert d["max_scaled_error"] <= 1.0, d["max_scaled_error"]


def test_product_library_is_not_the_checking_build(lib):
    import ctypes as C

    from geauxdock_b200._lib import GD_E_STATE

    out = (C.c_int * 4)()
    assert lib.gd_check_report(out, 0) == GD_E_STATE
