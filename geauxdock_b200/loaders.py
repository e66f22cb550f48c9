"""Input files -> reference-layout Complex (gd_load_complex).

The frontend path of the reference for one docking job: the ligand .sdf with
its conformer ensemble, the .ff file (KDE points, pocket-specific potential,
MCS rows of the ligand) and the protein .pdb models, with the force field from
the parameter files (params.parse_enepara0 + params.optimize_enepara).
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import layout as Lo, params
from ._lib import LoadArgs, check, load


def load_complex(sdf: str | Path, ff: str | Path, pdb: str | Path, ligand_id: str,
                 enepara0: np.ndarray, enepara: np.ndarray | None = None, *, num_temp: int = 1,
                 floor_temp: float = 0.044, ceiling_temp: float = 0.036, translation_step: float = 0.02,
                 rotation_step: float = 0.08, steps_total: int = 200, steps_per_dump: int = 200,
                 steps_per_exchange: int = 0, molid: str = "MOLID") -> np.ndarray:
    """One Complex record (numpy, 64-byte aligned) for the job described by the files."""
    if enepara is None:
        enepara = params.optimize_enepara(enepara0)
    e0 = np.array([enepara0], dtype=Lo.ENEPARA0) if np.ndim(enepara0) == 0 else np.asarray(enepara0, Lo.ENEPARA0)
    e1 = np.array([enepara], dtype=Lo.ENEPARA) if np.ndim(enepara) == 0 else np.asarray(enepara, Lo.ENEPARA)
    a = LoadArgs()
    a.lig_sdf, a.lhm_ff, a.prt_pdb = str(sdf).encode(), str(ff).encode(), str(pdb).encode()
    a.ligand_id, a.molid = ligand_id.encode(), molid.encode()
    a.enepara0, a.enepara = e0.ctypes.data, e1.ctypes.data
    a.num_temp, a.floor_temp, a.ceiling_temp = num_temp, floor_temp, ceiling_temp
    a.translation_step, a.rotation_step = translation_step, rotation_step
    a.steps_total, a.steps_per_dump, a.steps_per_exchange = steps_total, steps_per_dump, steps_per_exchange
    cx = Lo.aligned_zeros(Lo.COMPLEX)
    check(load().gd_load_complex(C.byref(a), C.c_void_p(cx.ctypes.data)))
    return cx
