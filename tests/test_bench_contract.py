"""bench.py's reference arm -- the reference's own CPU Monte Carlo, built from
its sources, on the headline workload; it needs no GPU: one JSON line with the
keys the bench contract names, the reference's identity and a zero-copy e2e."""

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e")


def test_reference_arm_json_line(oracle_lib):
    if not oracle_lib.have_ref():
        oracle_lib.build()
    if not oracle_lib.have_ref():
        pytest.skip("reference build unavailable")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=900, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert all(k in d for k in KEYS), [k for k in KEYS if k not in d]
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "pose-evals/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 1
    assert "replica ensemble" in d["config"]["workload"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # the reference arm runs the reference alone: none of this package's libraries is mapped
    assert "oracle/_ref/libgdref.so" in d["libraries_loaded"]
    assert not [f for f in d["libraries_loaded"] if f.startswith("geauxdock_b200/")], d["libraries_loaded"]
