"""numpy mirrors of the boundary structs of include/gdock_types.h.

Each dtype carries the explicit offsets and item size of the C struct (the
reference's layout, src/common/geauxdock.h and geauxdock_soa.h), so a numpy
record and the C struct are the same bytes.  tests/test_layout.py checks every
size and offset here against the compiled library.
"""

from __future__ import annotations

import numpy as np

MAXPRO, MAXLIG, MAX_CONF_PRT, MAX_CONF_LIG = 2048, 64, 20, 64
MAX_TMP, MAX_REP, MAXTP1, MAXTP2, MAXTP3, MAXTP4 = 1024, 16384, 31, 24, 50, 20
MAXWEI, MAXKDE, MAX_MCS_ROW, MAX_MCS_COL = 10, 10240, 512, 64
STEPS_PER_DUMP = 200
MCS_INVALID_COORD = np.float32(0.01234)


def _dt(fields, itemsize):
    names, formats, offsets = [], [], []
    for name, fmt, off in fields:
        names.append(name)
        formats.append(fmt)
        offsets.append(off)
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": itemsize})


def _seq(spec, itemsize, start=0):
    """Fields laid out back to back from `start` (all 4-byte aligned here)."""
    out, off = [], start
    for name, fmt in spec:
        out.append((name, fmt, off))
        off += np.dtype(fmt).itemsize
    return out, off


f4, i4 = np.float32, np.int32
L = MAXLIG

_lig, _end = _seq([(n, (f4 if n[0] != "t" else i4, L)) for n in
                   ["x1", "y1", "z1", "t1", "c1", "x2", "y2", "z2", "t2", "c2", "x3", "y3", "z3", "t3", "c3"]]
                  + [("kde_begin_idx", (i4, L)), ("kde_end_idx", (i4, L)), ("center", (f4, 3)),
                     ("lig_natom", i4)], 4416)
LIGAND = _dt(_lig, 4416)

_prt, _ = _seq([("t", (i4, MAXPRO)), ("x", (f4, MAXPRO)), ("y", (f4, MAXPRO)), ("z", (f4, MAXPRO)),
                ("cdc", (i4, MAXPRO)), ("hpp", (f4, MAXPRO)), ("ele", (f4, MAXPRO)), ("c", (i4, MAXPRO)),
                ("seq3r", (i4, MAXPRO)), ("pocket_center", (f4, 3)), ("prt_npoint", i4)], 73792)
PROTEIN = _dt(_prt, 73792)

PSP = _dt([("psp", (f4, (MAXLIG, MAXPRO)), 0)], 524288)

_kde, _ = _seq([("t", (i4, MAXKDE)), ("x", (f4, MAXKDE)), ("y", (f4, MAXKDE)), ("z", (f4, MAXKDE)),
                ("kde_npoint", i4)], 163904)
KDE = _dt(_kde, 163904)

_mcs, _ = _seq([("x", (f4, L)), ("y", (f4, L)), ("z", (f4, L)), ("ncol", i4), ("tcc", f4)], 832)
MCS = _dt(_mcs, 832)

T2 = (MAXTP2, MAXTP1)
_ep, _ = _seq([("p1a", (f4, T2)), ("p2a", (f4, T2)), ("lj0", f4), ("lj1", f4), ("el1", f4), ("el0", f4),
               ("a1", f4), ("b1", f4), ("pmf0", (f4, T2)), ("pmf1", (f4, T2)), ("hdb0", (f4, T2)),
               ("hdb1", (f4, T2)), ("hpp", (f4, MAXTP4)), ("hpl0", (f4, MAXTP2)), ("hpl1", (f4, MAXTP2)),
               ("hpl2", (f4, MAXTP2)), ("kde2", f4), ("kde3", f4), ("a_para", (f4, MAXWEI)),
               ("b_para", (f4, MAXWEI)), ("w", (f4, MAXWEI))], 18432)
ENEPARA = _dt(_ep, 18432)

T3 = (MAXTP1, MAXTP2, 2)
_ep0, _ = _seq([("vdw", (f4, T3)), ("ele", (f4, MAXTP3)), ("pmf", (f4, T3)), ("hpp", (f4, MAXTP4)),
                ("hpl", (f4, (MAXTP2, 2))), ("hdb", (f4, T3)), ("lj", (f4, 3)), ("el", (f4, 2)), ("kde", f4),
                ("w", (f4, MAXWEI)), ("a_para", (f4, MAXWEI)), ("b_para", (f4, MAXWEI))], 18472)
ENEPARA0 = _dt(_ep0, 18472)

TEMP = _dt([("t", f4, 0), ("minus_beta", f4, 4), ("order", i4, 8)], 12)

REPLICA = _dt([("idx_rep", i4, 0), ("idx_lig", i4, 4), ("idx_prt", i4, 8), ("idx_tmp", i4, 12),
               ("movematrix", (f4, 6), 16), ("energy", (f4, MAXWEI), 40), ("step", i4, 80),
               ("is_accept", i4, 84)], 128)

MCPARA = _dt([("steps_total", i4, 0), ("steps_per_dump", i4, 4), ("steps_per_exchange", i4, 8),
              ("move_scale", (f4, 6), 12), ("outputdir", "S128", 36), ("outputfile", "S128", 164)], 292)

RECORD = _dt([("replica", (REPLICA, STEPS_PER_DUMP), 0), ("next_entry", i4, 25600)], 25664)

SIZE = _dt([(n, i4, 4 * k) for k, n in enumerate(
    ["n_lig", "n_prt", "n_tmp", "n_rep", "lig_natom", "prt_npoint", "kde_npoint", "mcs_nrow"])], 32)

PARAT = _dt([("rep_begin", i4, 0), ("rep_end", i4, 4), ("n_rep", i4, 8), ("record_sz", i4, 12)], 16)

COMPLEX = _dt([
    ("lig", (LIGAND, MAX_CONF_LIG), 0), ("prt", (PROTEIN, MAX_CONF_PRT), 282624), ("psp", PSP, 1758464),
    ("kde", KDE, 2282752), ("mcs", (MCS, MAX_MCS_ROW), 2446656), ("mcs_r", "V395264", 2872640),
    ("mcs_ell", "V528384", 3267904), ("mcs_csr", "V657472", 3796288), ("enepara", ENEPARA, 4453760),
    ("temp", (TEMP, MAX_TMP), 4472192), ("replica", (REPLICA, MAX_REP), 4484480), ("size", SIZE, 6581632),
    ("mcpara", MCPARA, 6581664), ("lig_file", "S256", 6581956), ("prt_file", "S256", 6582212),
    ("lhm_file", "S256", 6582468), ("enepara_file", "S256", 6582724), ("weight_file", "S256", 6582980),
    ("rep_begin", i4, 6583236), ("rep_end", i4, 6583240), ("signal", i4, 6583244)], 6583296)


def aligned_zeros(dtype, n: int = 1, align: int = 64) -> np.ndarray:
    """Zeroed array of n records whose first byte is `align`-aligned."""
    dt = np.dtype(dtype)
    raw = np.zeros(n * dt.itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off: off + n * dt.itemsize].view(dt)
