"""Regenerate ff08_enepara0.npy: the reference's parameter files
(data/parameters/paras, 08ff_opt, 08_nor_a, 08_nor_b) parsed by
geauxdock_b200.params.parse_enepara0 into one EnePara0 record.

Usage: python geauxdock_b200/data/make_params.py [reference root; default: GD_REFERENCE, see oracle/refpath.py]
"""

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from geauxdock_b200 import params  # noqa: E402

from oracle.refpath import reference_path  # noqa: E402

ref = Path(sys.argv[1]) if len(sys.argv) > 1 else reference_path()
d = ref / "data" / "parameters"
e = params.parse_enepara0(d / "paras", d / "08ff_opt", d / "08_nor_a", d / "08_nor_b")
np.save(params.DEFAULT_PARAMS, np.frombuffer(e.tobytes(), dtype=np.uint8))
print(params.DEFAULT_PARAMS, params.DEFAULT_PARAMS.stat().st_size, "bytes")
