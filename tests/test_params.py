"""Parameter-file parsing and OptimizeEnepara, byte-identical to the reference."""

import numpy as np
import pytest

from conftest import REFERENCE, have_reference_sources


def _ref_enepara(O):
    from geauxdock_b200 import layout as Lo

    d = REFERENCE / "data/parameters"
    e0 = Lo.aligned_zeros(Lo.ENEPARA0)
    e = Lo.aligned_zeros(Lo.ENEPARA)
    O.ref().gdref_load_enepara(*(str(d / f).encode() for f in ("paras", "08ff_opt", "08_nor_a", "08_nor_b")),
                               e0.ctypes.data, e.ctypes.data)
    return e0[0], e[0]


@pytest.mark.skipif(not have_reference_sources(), reason="reference sources absent")
def test_parser_matches_reference_loader(oracle_lib):
    from geauxdock_b200 import params

    O = oracle_lib
    if not O.have_ref():
        O.build()
    d = REFERENCE / "data/parameters"
    mine = params.parse_enepara0(d / "paras", d / "08ff_opt", d / "08_nor_a", d / "08_nor_b")
    ref0, _ = _ref_enepara(O)
    for f in ref0.dtype.names:
        a, b = np.asarray(mine[f]), np.asarray(ref0[f])
        if f == "w":   # w[9] is read past the end of a token array in the reference (load.C:1320-1331)
            a, b = a[:9], b[:9]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f


def test_bundled_parameters_roundtrip():
    from geauxdock_b200 import params

    if not have_reference_sources():
        pytest.skip("reference sources absent")
    d = REFERENCE / "data/parameters"
    mine = params.parse_enepara0(d / "paras", d / "08ff_opt", d / "08_nor_a", d / "08_nor_b")
    assert mine.tobytes() == params.default_enepara0().tobytes()


@pytest.mark.skipif(not have_reference_sources(), reason="reference sources absent")
def test_optimize_enepara_bit_identical(oracle_lib, lib):
    from geauxdock_b200 import params

    O = oracle_lib
    if not O.have_ref():
        O.build()
    _, ref = _ref_enepara(O)
    mine = params.optimize_enepara(params.default_enepara0())
    for f in ref.dtype.names:
        a, b = np.asarray(mine[f]), np.asarray(ref[f])
        if f == "w":
            a, b = a[:9], b[:9]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f


def test_optimize_enepara_formulas(lib):
    """Spot values of OptimizeEnepara's formulas (util_optimize_soa.C:489-540)."""
    from geauxdock_b200 import params

    e0 = params.default_enepara0()
    e = params.optimize_enepara(e0)
    i, j = 3, 0   # ligand type C.3, point type CA
    tmp = np.float32(e0["vdw"][j, i, 0] * e0["lj"][2])
    assert e["p1a"][i, j] == pytest.approx(2.0 * e0["vdw"][j, i, 1] * float(tmp) ** 9, rel=1e-6)
    assert e["a1"] == np.float32(4.0) - np.float32(3.0) * e0["el"][0]
    assert e["kde2"] == np.float32(-0.5) / (e0["kde"] * e0["kde"])
    assert np.all(np.isinf(e["hdb1"][e0["hdb"][:, :, 1].T == 0]))   # 1/0 where no HDB line exists


def test_type_tables():
    from geauxdock_b200 import params

    assert len(params.LIG_TYPES) == 24 and len(params.POINT_TYPES) == 30
    assert params.lig_code("Br") == 0 and params.lig_code("S.O2") == 23 and params.lig_code("H") == params.BADKDE
    assert params.pnt_code("CA") == 0 and params.pnt_code("Y2") == 29
    assert params.res_code_one("G") == params.GLY == 12
    assert sum(len(v) for v in params.SIDE_CHAIN.values()) == 28
