"""Regenerate tests/golden/known_answer_1a07.npz: the reference's one pinned
result as a fixture that travels without the reference tree.

The reference's known-answer line (doc/instructions.txt:186-187, printed by
src/common/kernel_print.C:11) is the ten initial energies of replica 0 of
ligand 1a07C1 (data/astex/ligands/1a07C1.sdf, 1a07C1-0.8.ff) against protein
1a07C-1 (data/astex/proteins/1a07C-1.pdb), one temperature, rounded to four
decimals (src/common/util_print.C:96-101).  This script builds that Complex
with this repository's loader (gd_load_complex, the reference frontend's
path; tests/test_loaders.py checks it byte for byte against the reference's
own frontend) and stores:

  complex   the Complex record's bytes, zlib-compressed (6.58 MB, mostly zero)
  expected  the ten numbers of the known-answer line, read from the doc
  oracle64  the FP64 oracle's ten energies of the same pose (the 4-decimal
            rounding margin of each term is checked here, so that an FP32
            evaluation within 1e-5 rounds to the same line)

Run where the reference sources are present (GD_REFERENCE, oracle/refpath.py)
and libgdock.so and oracle/liboracle.so are built.
"""

import sys
import zlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from geauxdock_b200 import layout as Lo, loaders, params  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle.refpath import reference_path  # noqa: E402

REF = Path(sys.argv[1]) if len(sys.argv) > 1 else reference_path()
OUT = HERE / "known_answer_1a07.npz"


def known_answer_line() -> list[float]:
    for ln in (REF / "doc/instructions.txt").read_text().splitlines():
        t = ln.split()
        if len(t) == 12 and t[0] == "0" and t[1] == "0":
            return [float(x) for x in t[2:]]
    raise RuntimeError("known-answer line not found in doc/instructions.txt")


def main() -> None:
    d = REF / "data"
    e0 = params.parse_enepara0(*[d / "parameters" / n for n in ("paras", "08ff_opt", "08_nor_a", "08_nor_b")])
    lig = d / "astex" / "ligands"
    cx = loaders.load_complex(lig / "1a07C1.sdf", lig / "1a07C1-0.8.ff", d / "astex" / "proteins" / "1a07C-1.pdb",
                              "1a07C1", e0, num_temp=1, steps_total=200, steps_per_dump=200)
    want = np.array(known_answer_line())
    e64, _ = O.energy(cx, 0, 0, np.zeros(6, np.float32))
    assert np.array_equal(np.round(e64, 4), want), (e64, want)
    # distance of each FP64 term to the nearest 4-decimal rounding boundary
    margin = np.abs(np.abs(e64 * 1e4 - np.floor(e64 * 1e4)) - 0.5) * 1e-4
    blob = zlib.compress(cx.tobytes(), 9)
    np.savez(OUT, complex=np.frombuffer(blob, np.uint8), expected=want, oracle64=e64,
             complex_bytes=np.array([Lo.COMPLEX.itemsize]))
    print(OUT, OUT.stat().st_size, "bytes; n_rep", int(cx[0]["size"]["n_rep"]),
          "; smallest rounding margin", float(margin.min()))


if __name__ == "__main__":
    main()
