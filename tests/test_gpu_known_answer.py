"""The reference's known-answer line through the CUDA kernels.

doc/instructions.txt:186-187 (printed by src/common/kernel_print.C:11) gives
the ten initial energies of replica 0 of ligand 1a07C1 against protein
1a07C-1, rounded to four decimals (src/common/util_print.C:96-101).  The
Complex of that job, built by this repository's loader from the reference's
input files (byte-identical to the reference frontend's, tests/test_loaders.py),
is committed as tests/golden/known_answer_1a07.npz together with the expected
line (tests/golden/make_known_answer.py), so this runs without the reference
tree.  Dock (steps_total = steps_per_dump = 200) records the initial state as
entry 0 of replica 0's Record, the entry the reference prints."""

import zlib
from pathlib import Path

import numpy as np
import pytest

from geauxdock_b200 import dock, layout as Lo
from geauxdock_b200._lib import GD_PREC_FP32, GD_PREC_FP32_KAHAN, GD_PREC_FP64, check
from oracle import tolerance as TOL

pytestmark = pytest.mark.gpu
FIXTURE = Path(__file__).resolve().parent / "golden" / "known_answer_1a07.npz"


def _fixture():
    f = np.load(FIXTURE)
    raw = zlib.decompress(f["complex"].tobytes())
    assert len(raw) == Lo.COMPLEX.itemsize == int(f["complex_bytes"][0])
    cx = Lo.aligned_zeros(Lo.COMPLEX)
    cx.view(np.uint8)[:] = np.frombuffer(raw, np.uint8)
    return cx, f["expected"], f["oracle64"]


@pytest.mark.parametrize("kernel", [0, 1], ids=["batched", "plain"])
def test_known_answer_through_dock(lib, kernel):
    cx, want, e64 = _fixture()
    assert int(cx[0]["size"]["n_rep"]) == 51 and int(cx[0]["size"]["lig_natom"]) == 34
    check(lib.gd_set_option(b"kernel", kernel))
    try:
        with dock.DockSession(1, seed=1) as s:
            rec = s.dock(cx)
    finally:
        check(lib.gd_set_option(b"kernel", 0))
    first = rec[0]["replica"][0]
    assert int(first["step"]) == 0 and int(rec[0]["next_entry"]) >= 1
    got = np.asarray(first["energy"], np.float64)
    TOL.check(got, e64, "initial energies vs FP64 oracle")
    assert [round(float(v), 4) for v in got] == pytest.approx(list(want), abs=1e-12), (got, want)


@pytest.mark.parametrize("prec", [GD_PREC_FP32, GD_PREC_FP32_KAHAN, GD_PREC_FP64])
def test_known_answer_pose_eval(lib, prec):
    """The same pose (replica 0's stored movematrix, ligand and protein
    conformation 0) through the pose-evaluation path in every precision."""
    cx, want, e64 = _fixture()
    out, _, _ = dock.eval_poses(cx, np.zeros((1, 2), np.int32), np.zeros((1, 6), np.float32), prec)
    TOL.check(out[0], e64, f"precision {prec}")
    assert [round(float(v), 4) for v in out[0]] == pytest.approx(list(want), abs=1e-12)
