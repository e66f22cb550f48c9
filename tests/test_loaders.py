"""The molecule loaders (gd_load_complex) against the reference frontend built
from its sources (oracle/_ref: loadLigand, loadLHM, loadProtein, Optimize*,
SetTemperature, SetReplica), on the reference's own input files: every field
of the Complex, except copy 1 of the ligand, which the reference's CPU build
sorts by type and the GPU frontend this loader follows keeps in input order.
Runs where the reference's files are present (they are not copied here)."""

import ctypes as C

import numpy as np
import pytest

from conftest import REFERENCE, have_reference_sources

pytestmark = pytest.mark.skipif(not have_reference_sources(), reason="reference sources and data absent")

DATA = REFERENCE / "data"
PARAMS = [DATA / "parameters" / n for n in ("paras", "08ff_opt", "08_nor_a", "08_nor_b")]
LIG_FIELDS = ["x2", "y2", "z2", "t2", "c2", "x3", "y3", "z3", "t3", "c3", "kde_begin_idx", "kde_end_idx",
              "center", "lig_natom"]


def _ref(O, lig_id, sdf, ff, pdb, num_temp=3, floor=0.044, ceil=0.036, ts=0.02, rs=0.08, total=100, dump=100):
    from geauxdock_b200 import layout as Lo

    cx = Lo.aligned_zeros(Lo.COMPLEX)
    args = [lig_id.encode()] + [str(p).encode() for p in (sdf, ff, pdb, *PARAMS)]
    n = O.ref().gdref_load_complex(*args, num_temp, C.c_float(floor), C.c_float(ceil), C.c_float(ts),
                                   C.c_float(rs), total, dump, cx.ctypes.data)
    assert n == int(cx[0]["size"]["n_rep"])
    return cx


def _ours(lig_id, sdf, ff, pdb, num_temp=3, floor=0.044, ceil=0.036, ts=0.02, rs=0.08, total=100, dump=100):
    from geauxdock_b200 import loaders, params

    e0 = params.parse_enepara0(*PARAMS)
    return loaders.load_complex(sdf, ff, pdb, lig_id, e0, num_temp=num_temp, floor_temp=floor,
                                ceiling_temp=ceil, translation_step=ts, rotation_step=rs, steps_total=total,
                                steps_per_dump=dump)


def _same(a, b, what):
    assert a.tobytes() == b.tobytes(), what


def _compare(got, want, ligand_only=False):
    g, w = got[0], want[0]
    sz = w["size"]
    for f in ("n_lig", "lig_natom", "kde_npoint", "mcs_nrow") + (() if ligand_only else ("n_prt", "prt_npoint",
                                                                                          "n_tmp", "n_rep")):
        assert g["size"][f] == sz[f], f
    for j in range(int(sz["n_lig"])):
        for f in LIG_FIELDS:
            _same(g["lig"][j][f], w["lig"][j][f], f"lig[{j}].{f}")
    _same(g["kde"], w["kde"], "kde")
    _same(g["psp"], w["psp"], "psp")
    nrow = int(sz["mcs_nrow"])
    _same(g["mcs"][:nrow], w["mcs"][:nrow], "mcs")
    _same(g["mcs_ell"], w["mcs_ell"], "mcs_ell")
    _same(g["mcs_csr"], w["mcs_csr"], "mcs_csr")
    if ligand_only:
        return
    for j in range(int(sz["n_prt"])):
        _same(g["prt"][j], w["prt"][j], f"prt[{j}]")
    _same(g["enepara"], w["enepara"], "enepara")
    _same(g["temp"][:int(sz["n_tmp"])], w["temp"][:int(sz["n_tmp"])], "temp")
    n = int(sz["n_rep"])
    for f in g["replica"].dtype.names:
        _same(g["replica"][:n][f], w["replica"][:n][f], f"replica.{f}")
    for f in ("steps_total", "steps_per_dump", "move_scale"):
        _same(g["mcpara"][f], w["mcpara"][f], f"mcpara.{f}")
    assert g["rep_begin"] == w["rep_begin"] and g["rep_end"] == w["rep_end"]


@pytest.mark.parametrize("pdb", ["1a07C.pdb", "1a07C-1.pdb", "1a07C-3.pdb"])
def test_1a07_complex_matches_reference(oracle_lib, pdb):
    O = oracle_lib
    if not O.have_ref():
        O.build()
    lig = DATA / "astex" / "ligands"
    files = ("1a07C1", lig / "1a07C1.sdf", lig / "1a07C1-0.8.ff", DATA / "astex" / "proteins" / pdb)
    want = _ref(O, *files)
    got = _ours(*files)
    _compare(got, want)
    # the GPU frontend keeps ligand copy 1 in input order
    for j in range(int(got[0]["size"]["n_lig"])):
        _same(got[0]["lig"][j]["x1"], got[0]["lig"][j]["x2"], "x1 == x2")


def test_every_ligand_parses_like_reference(oracle_lib):
    """All ligands of the reference's data set (with one protein file, which only
    the protein fields depend on): conformer ensembles with the near-duplicate
    filter, KDE points, psp, MCS rows.  Runs in a child process (see
    loader_parity_worker.py for why)."""
    import subprocess
    import sys
    from pathlib import Path

    O = oracle_lib
    if not O.have_ref():
        O.build()
    worker = Path(__file__).resolve().parent / "loader_parity_worker.py"
    r = subprocess.run([sys.executable, str(worker)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-4000:])
    n = int(r.stdout.strip().split()[-1])
    assert n > 100


def test_loader_errors_are_status_codes(lib, tmp_path):
    from geauxdock_b200 import loaders, params
    from geauxdock_b200._lib import GD_E_INVALID, GdockError

    e0 = params.parse_enepara0(*PARAMS)
    lig = DATA / "astex" / "ligands"
    with pytest.raises(GdockError) as ei:
        loaders.load_complex(tmp_path / "missing.sdf", lig / "1a07C1-0.8.ff",
                             DATA / "astex" / "proteins" / "1a07C.pdb", "1a07C1", e0)
    assert ei.value.code == GD_E_INVALID
    bad = tmp_path / "bad.pdb"
    bad.write_text("ATOM      1  CA  XXX A   1      1.000   2.000   3.000  1.00  0.00           C\nENDMDL\n")
    with pytest.raises(GdockError) as ei:
        loaders.load_complex(lig / "1a07C1.sdf", lig / "1a07C1-0.8.ff", bad, "1a07C1", e0)
    assert ei.value.code == GD_E_INVALID


def test_known_answer_through_loader(oracle_lib):
    """The reference's known-answer line (doc/instructions.txt:186-187) from a
    Complex built by this loader: initial energies of replica 0 of 1a07C1 x
    1a07C-1, FP64 oracle rounded as the reference prints them."""
    from test_oracle import _known_answer_line

    lig = DATA / "astex" / "ligands"
    cx = _ours("1a07C1", lig / "1a07C1.sdf", lig / "1a07C1-0.8.ff", DATA / "astex" / "proteins" / "1a07C-1.pdb",
               num_temp=1)
    e, _ = oracle_lib.energy(cx, 0, 0, np.zeros(6, np.float32))
    assert [round(float(v), 4) for v in e] == pytest.approx(_known_answer_line(), abs=1e-12)
