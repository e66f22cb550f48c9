"""Force-field parameters: type-code tables, the parameter-file parser, and the
bundled default parameter set.

The type codes are the reference's interface (src/frontend/data.C):
  ligand atom types   getLigCode  (data.C:532-587), 24 SYBYL types
  protein point types getPntCode  (data.C:391-454), 30 effective points
  residue codes       getResCode / getResCodeOne (data.C:239-337)
and the per-residue side-chain points of the coarse-grained protein
(src/frontend/load.C:548-616).

parse_enepara0() reads the four parameter files with the semantics of
loadEnePara, loadWeight and loadNorPara (src/frontend/load.C:1189-1441):
whitespace-separated records keyed by their first three characters, values
parsed as decimals and stored as float, hydrophobicity rescaled to [-1, 1].
The precomputation OptimizeEnepara (src/frontend/util_optimize_soa.C:489-540)
runs in libgdock (gd_optimize_enepara) so that its float arithmetic is the C
library's.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import layout

LIG_TYPES = ["Br", "C.1", "C.2", "C.3", "C.ar", "C.cat", "Cl", "F", "I", "N.1", "N.2", "N.3", "N.4", "N.am",
             "N.ar", "N.pl3", "O.2", "O.3", "O.co2", "P.3", "S.2", "S.3", "S.O", "S.O2"]
POINT_TYPES = ["CA", "PP", "A1", "C1", "D1", "E1", "E2", "F1", "F2", "H1", "H2", "I1", "K1", "K2", "L1", "M1",
               "M2", "N1", "P1", "Q1", "Q2", "R1", "R2", "S1", "T1", "V1", "W1", "W2", "Y1", "Y2"]
RES_ONE = "ARCPLIEHWTMDGFKQSNYV"          # getResCodeOne: A=0 ... V=19
RES_THREE = ["ALA", "ARG", "CYS", "PRO", "LEU", "ILE", "GLU", "HIS", "TRP", "THR", "MET", "ASP", "GLY", "PHE",
             "LYS", "GLN", "SER", "ASN", "TYR", "VAL"]
GLY = 12
BADKDE = 50                                # getLigCode for an unknown name

# side-chain points per residue code: [(point type, class), ...] (load.C:548-616)
SIDE_CHAIN = {
    0: [(2, 2)], 1: [(21, 2), (22, 3)], 2: [(3, 2)], 3: [(18, 2)], 4: [(14, 2)], 5: [(11, 2)],
    6: [(5, 2), (6, 3)], 7: [(9, 2), (10, 3)], 8: [(26, 2), (27, 3)], 9: [(24, 2)], 10: [(15, 2), (16, 3)],
    11: [(4, 2)], 12: [], 13: [(7, 2), (8, 3)], 14: [(12, 2), (13, 3)], 15: [(19, 2), (20, 3)], 16: [(23, 2)],
    17: [(17, 2)], 18: [(28, 2), (29, 3)], 19: [(25, 2)],
}

DATA_DIR = Path(__file__).resolve().parent / "data"
DEFAULT_PARAMS = DATA_DIR / "ff08_enepara0.npy"

_LIG = {n: i for i, n in enumerate(LIG_TYPES)}
_PNT = {n: i for i, n in enumerate(POINT_TYPES)}


def lig_code(name: str) -> int:
    return _LIG.get(name, BADKDE)


def pnt_code(name: str) -> int:
    if name not in _PNT:
        raise ValueError(f"unknown effective point {name!r}")
    return _PNT[name]


def res_code_one(name: str) -> int:
    i = RES_ONE.find(name)
    if len(name) != 1 or i < 0:
        raise ValueError(f"unknown residue {name!r}")
    return i


def _f32(s: str) -> np.float32:
    return np.float32(float(s))


def parse_enepara0(paras: str | Path, weight: str | Path, nor_a: str | Path, nor_b: str | Path) -> np.ndarray:
    """Parameter files -> one EnePara0 record (raw force-field parameters)."""
    e = np.zeros(1, dtype=layout.ENEPARA0)[0]
    for line in Path(paras).read_text().splitlines():
        if len(line) <= 3:
            continue
        key, tok = line[:3], line.split()
        if key == "VDW":
            p, l = pnt_code(tok[1]), lig_code(tok[2])
            e["vdw"][p, l] = (_f32(tok[3]), _f32(tok[4]))
        elif key == "PLJ":
            e["lj"][:] = [_f32(t) for t in tok[1:4]]
        elif key == "ELE":
            if tok[1][1:2] != "C":
                e["ele"][pnt_code(tok[1])] = _f32(tok[2])
            else:
                e["ele"][res_code_one(tok[1][0]) + 30] = _f32(tok[2])
        elif key == "PEL":
            e["el"][:] = [_f32(t) for t in tok[1:3]]
        elif key == "PMF":
            p, l = pnt_code(tok[1]), lig_code(tok[2])
            e["pmf"][p, l] = (_f32(tok[3]), _f32(tok[4]))
        elif key == "HPP":
            e["hpp"][res_code_one(tok[1])] = _f32(tok[2])
        elif key == "HPL":
            e["hpl"][lig_code(tok[1])] = (_f32(tok[2]), _f32(tok[3]))
        elif key == "HDB":
            p, l = pnt_code(tok[1]), lig_code(tok[2])
            e["hdb"][p, l] = (_f32(tok[3]), _f32(tok[4]))
        elif key == "WEI":
            vals = tok[1:]
            for i in range(min(len(vals), layout.MAXWEI)):
                e["w"][i] = _f32(vals[i])
        elif key == "KDE":
            e["kde"] = _f32(tok[1])
    # hydrophobicity rescaled to [-1, 1] (load.C:1351-1374); the arithmetic is
    # float except the final "* 2.0 - 1.0", which the C code does in double
    hpp = e["hpp"].astype(np.float32)
    lo, hi = np.float32(1e6), np.float32(-1e6)
    for v in hpp:
        lo = v if v < lo else lo
        hi = v if v > hi else hi
    for i, v in enumerate(hpp):
        t = np.float32(np.float32(v - lo) / np.float32(hi - lo))
        x = np.float32(float(t) * 2.0 - 1.0)
        e["hpp"][i] = min(max(x, np.float32(-1.0)), np.float32(1.0))
    # one value per line, first 30 characters (load.C:1378-1441, 1476-1507)
    for path, field in ((weight, "w"), (nor_a, "a_para"), (nor_b, "b_para")):
        lines = Path(path).read_text().splitlines()
        for i, ln in enumerate(lines[: layout.MAXWEI]):
            s = ln[:30].split()
            e[field][i] = _f32(s[0]) if s else np.float32(0.0)
    return e


def default_enepara0() -> np.ndarray:
    """The bundled parameter set (the reference's data/parameters, parsed)."""
    if not DEFAULT_PARAMS.exists():
        raise FileNotFoundError(f"{DEFAULT_PARAMS} missing (geauxdock_b200/data/make_params.py)")
    raw = np.load(DEFAULT_PARAMS)
    return np.frombuffer(raw.tobytes(), dtype=layout.ENEPARA0)[0].copy()


def optimize_enepara(ep0: np.ndarray) -> np.ndarray:
    """EnePara0 -> EnePara with OptimizeEnepara's arithmetic (in libgdock)."""
    from ._lib import check, load

    src = np.array([ep0], dtype=layout.ENEPARA0)
    dst = np.zeros(1, dtype=layout.ENEPARA)
    check(load().gd_optimize_enepara(C.c_void_p(src.ctypes.data), C.c_void_p(dst.ctypes.data)))
    return dst[0]
