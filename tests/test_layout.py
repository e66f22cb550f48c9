"""libgdock.so loads without a GPU, exports every function include/*.h
declares, and its struct layouts agree with the numpy mirrors."""

import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, re.M):
            if m.group(1) not in ("if", "while", "for", "return", "sizeof", "GD_STATIC_ASSERT"):
                names.add(m.group(1))
    return names


def test_exports_every_declared_symbol(lib):
    declared = _declared_functions()
    assert {"Dock", "SetDevice", "DeviceAlloc", "DeviceFree", "SetParaT", "CopyH2D", "InitCurand"} <= declared
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    from geauxdock_b200._lib import EXPORTED

    assert declared == set(EXPORTED) - {"gd_layout"}


@pytest.mark.parametrize("name,dtype", [("Complex", "COMPLEX"), ("Record", "RECORD"), ("ReplicaMC", "REPLICA"),
                                        ("EnePara", "ENEPARA"), ("EnePara0", "ENEPARA0"), ("Ligand", "LIGAND"),
                                        ("Protein", "PROTEIN"), ("Kde", "KDE"), ("Mcs", "MCS"), ("ParaT", "PARAT")])
def test_sizes(lib, name, dtype):
    from geauxdock_b200 import layout as Lo
    from geauxdock_b200._lib import layout

    assert getattr(Lo, dtype).itemsize == layout("sizeof." + name)


def test_reference_sizes(lib):
    """Sizes measured from the reference headers (src/common/geauxdock.h)."""
    from geauxdock_b200._lib import layout

    assert layout("sizeof.Complex") == 6583296
    assert layout("sizeof.Record") == 25664
    assert layout("sizeof.ReplicaMC") == 128
    assert layout("sizeof.EnePara") == 18432


def test_offsets(lib):
    from geauxdock_b200 import layout as Lo
    from geauxdock_b200._lib import layout

    for f in ["lig", "prt", "psp", "kde", "mcs", "enepara", "temp", "replica", "size", "mcpara", "lig_file",
              "rep_begin", "rep_end", "signal"]:
        assert Lo.COMPLEX.fields[f][1] == layout("Complex." + f), f
    for f in ["w", "hpl0", "kde2"]:
        assert Lo.ENEPARA.fields[f][1] == layout("EnePara." + f), f
    assert Lo.RECORD.fields["next_entry"][1] == layout("Record.next_entry")


def test_reference_layout_matches(oracle_lib):
    O = oracle_lib
    if not O.have_ref():
        pytest.skip("reference library not built")
    from geauxdock_b200 import layout as Lo

    r = O.ref()
    assert r.gdref_sizeof(b"Complex") == Lo.COMPLEX.itemsize
    assert r.gdref_sizeof(b"Record") == Lo.RECORD.itemsize
    assert r.gdref_sizeof(b"EnePara0") == Lo.ENEPARA0.itemsize


def test_ctypes_mirrors_of_api_structs(lib):
    """The ctypes structures of the serving and descriptor API match the C layout."""
    import ctypes as C

    from geauxdock_b200._lib import (Cluster, JobDesc, LoadArgs, PocketDesc, Request, Result, ServerConfig,
                                     ServerStats, layout)

    for name, cls in (("gd_job_desc_t", JobDesc), ("gd_pocket_desc_t", PocketDesc), ("gd_load_args_t", LoadArgs), ("gd_cluster_t", Cluster),
                      ("gd_server_config_t", ServerConfig), ("gd_request_t", Request),
                      ("gd_result_t", Result), ("gd_server_stats_t", ServerStats)):
        assert layout(f"sizeof.{name}") == C.sizeof(cls), name
    assert layout("gd_server_stats_t.warps_per_cta") == ServerStats.warps_per_cta.offset
    assert layout("gd_result_t.t_done") == Result.t_done.offset
