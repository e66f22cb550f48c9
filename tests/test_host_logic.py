"""Host-side logic of the C ABI that needs no GPU: replica partitioning
(SetParaT), option validation, and input validation before any device work."""

import ctypes as C

import numpy as np
import pytest

from geauxdock_b200 import layout as Lo, synth
from geauxdock_b200._lib import GD_E_INVALID, GdockError, check


def _parat(lib, cx, ngpu):
    from geauxdock_b200.dock import ParaT

    lib.gd_set_ngpu(ngpu)
    pts = (ParaT * ngpu)()
    arr = (C.POINTER(ParaT) * ngpu)(*[C.pointer(pts[g]) for g in range(ngpu)])
    rc = lib.SetParaT(C.c_void_p(cx.ctypes.data), arr)
    lib.gd_set_ngpu(1)
    return rc, [(p.rep_begin, p.rep_end, p.n_rep, p.record_sz) for p in pts]


def _ref_split(n_rep, ngpu):
    """prepair.C:366-392, maximising balance."""
    per = int(np.ceil(n_rep / ngpu))
    out = []
    for g in range(ngpu):
        b = per * g
        e = min(b + per, n_rep) - 1
        out.append((b, e, e - b + 1, Lo.RECORD.itemsize * (e - b + 1)))
    return out


@pytest.mark.parametrize("ngpu", [1, 2, 3, 8])
def test_setparat_matches_reference_split(lib, enepara, ngpu):
    pk, job = synth.config2(1)
    cx = synth.to_complex(job, pk, enepara)
    rc, got = _parat(lib, cx, ngpu)
    assert rc == 0
    assert got == _ref_split(3520, ngpu)


def test_setparat_exchange_cuts_at_protein_blocks(lib, enepara):
    pk, job = synth.config2(1)
    cx = synth.to_complex(job, pk, enepara, steps_per_exchange=50)
    rc, got = _parat(lib, cx, 4)
    assert rc == 0
    block = 16 * 20
    for b, e, n, _ in got:
        assert b % block == 0 and (e + 1) % block == 0 or e == 3519
    assert got[-1][1] == 3519 and sum(g[2] for g in got) == 3520


def test_setparat_too_many_gpus(lib, enepara):
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    rc, _ = _parat(lib, cx, 2)     # 1 replica cannot keep 2 GPUs busy (prepair.C:371-374)
    assert rc == GD_E_INVALID


def test_options_validated(lib):
    with pytest.raises(GdockError):
        check(lib.gd_set_option(b"kernel", 7))
    with pytest.raises(GdockError):
        check(lib.gd_set_option(b"nonsense", 1))
    assert lib.gd_get_option(b"kpl") == 0          # default pair-tile shape: the library's choice
    check(lib.gd_set_option(b"kpl", 4))
    assert lib.gd_get_option(b"kpl") == 4
    check(lib.gd_set_option(b"kpl", 0))
    assert lib.gd_get_option(b"graph") == 1
    assert lib.gd_get_option(b"stage") == -1
    assert lib.gd_get_option(b"dock_cache") == 1
    assert lib.gd_get_option(b"device_base") == 0
    with pytest.raises(GdockError):
        check(lib.gd_set_option(b"device_base", -1))
    assert lib.gd_get_option(b"stall_test") == 0 and lib.gd_get_option(b"wait_limit") == 0
    with pytest.raises(GdockError):
        check(lib.gd_set_option(b"stall_test", 3))
    with pytest.raises(GdockError):
        check(lib.gd_set_option(b"stage", 2))
    with pytest.raises(GdockError):
        check(lib.gd_set_option(b"graph", 2))
    # the allocation-failure test hook counts down and is off by default
    assert lib.gd_get_option(b"fail_alloc") == 0
    check(lib.gd_set_option(b"fail_alloc", 2))
    assert lib.gd_get_option(b"fail_alloc") == 2
    check(lib.gd_set_option(b"fail_alloc", 0))
    with pytest.raises(GdockError):
        check(lib.gd_set_option(b"fail_alloc", -1))


def test_eval_rejects_bad_conformation_before_device_work(lib, enepara):
    from geauxdock_b200 import dock

    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    with pytest.raises(GdockError) as ei:
        dock.eval_poses(cx, np.array([[0, 3]]), np.zeros((1, 6)))
    assert ei.value.code == GD_E_INVALID


def test_server_defaults_and_validation(lib, enepara):
    """Server configuration defaults; a bad configuration or a missing GPU is an
    error status before any device work."""
    import ctypes as C

    from geauxdock_b200._lib import GD_E_INVALID, GD_E_NODEVICE, PocketDesc, ServerConfig

    cfg = ServerConfig()
    lib.gd_server_config_default(C.byref(cfg))
    assert cfg.hbm_budget_bytes == 100 * 10**9 and cfg.steps_per_round == 50 and cfg.max_jobs == 256
    keep: list = []
    pk = synth.make_pocket(np.random.default_rng(3), 300, 2)
    parr = (PocketDesc * 1)(synth.pocket_desc(pk, keep))
    ep = np.array([enepara], dtype=Lo.ENEPARA)
    h = C.c_void_p()
    bad = ServerConfig()
    lib.gd_server_config_default(C.byref(bad))
    bad.steps_per_round = 0
    assert lib.gd_server_create(parr, 1, C.c_void_p(ep.ctypes.data), C.byref(bad), C.byref(h)) == GD_E_INVALID
    rc = lib.gd_server_create(parr, 1, C.c_void_p(ep.ctypes.data), C.byref(cfg), C.byref(h))
    import torch

    if not torch.cuda.is_available():
        assert rc == GD_E_NODEVICE
    else:
        assert rc == 0
        lib.gd_server_destroy(h)
