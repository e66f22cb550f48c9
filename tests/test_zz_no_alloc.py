"""gd_eval_poses_noalloc: pose energies for callers that cannot allocate
device memory around a docking call (a process whose device memory belongs to
another allocator, or a serving loop that cannot afford cudaFree's device-wide
synchronisation).  The caller passes device buffers it already owns -- here
torch tensors stand in for such memory -- and the library uses only its fixed
scratch array.  Its output must match the allocating entry point
gd_eval_poses, and the FP64 oracle, within the energy tolerance of the other
GPU tests (oracle/tolerance.py), on two different complexes evaluated one
after the other (so the second call also shows that nothing stale from the
first call's scratch contents leaks in).  Malformed inputs are refused with a
status, and the next valid call still matches.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""

import ctypes as C

import numpy as np
import pytest

from geauxdock_b200 import dock, layout as Lo, synth
from geauxdock_b200._lib import GD_E_CAPACITY, GD_E_INVALID, GD_PREC_FP32, GD_PREC_FP64, GdockError, check
from oracle import tolerance as TOL

pytestmark = pytest.mark.gpu


def _device_copy(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()


def _noalloc(lib, torch, d_cx, conf, mm, precision=GD_PREC_FP32, stream=True):
    n = len(conf)
    d_conf = torch.from_numpy(np.ascontiguousarray(conf, np.int32)).cuda()
    d_mm = torch.from_numpy(np.ascontiguousarray(mm, np.float32)).cuda()
    d_out = torch.full((n, 10), float("nan"), dtype=torch.float32, device="cuda")
    d_raw = torch.full((n, 9), float("nan"), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream if stream else None
    torch.cuda.synchronize()
    check(lib.gd_eval_poses_noalloc(C.c_void_p(d_cx.data_ptr()), n, C.c_void_p(d_conf.data_ptr()),
                                    C.c_void_p(d_mm.data_ptr()), precision, C.c_void_p(d_out.data_ptr()),
                                    C.c_void_p(d_raw.data_ptr()), C.c_void_p(st)))
    return d_out.cpu().numpy(), d_raw.cpu().numpy()


def _oracle(O, cx, conf, mm):
    return np.array([O.energy(cx, int(c[0]), int(c[1]), m)[0] for c, m in zip(conf, mm)])


def test_noalloc_matches_eval_poses_two_calls(lib, enepara, oracle_lib):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(17)
    # call 1: the replica-ensemble complex, poses over every conformation pair
    pk2, job2 = synth.config2(1)
    cx2 = synth.to_complex(job2, pk2, enepara)
    conf2 = np.stack([rng.integers(0, 20, 300), rng.integers(0, 11, 300)], axis=1).astype(np.int32)
    mm2 = synth.config4_poses(5, 300, radius=6.0)
    # call 2: a different, smaller complex
    pk1, job1 = synth.config1(1)
    cx1 = synth.to_complex(job1, pk1, enepara)
    conf1 = np.zeros((64, 2), np.int32)
    mm1 = synth.config4_poses(6, 64, radius=4.0)
    for k, (cx, conf, mm) in enumerate(((cx2, conf2, mm2), (cx1, conf1, mm1))):
        want, want_raw, _ = dock.eval_poses(cx, conf, mm, GD_PREC_FP32)
        got, got_raw = _noalloc(lib, torch, _device_copy(torch, cx), conf, mm, stream=(k == 0))
        assert np.isfinite(got).all() and np.isfinite(got_raw).all()
        TOL.check(got, want.astype(np.float64), f"call {k + 1} vs gd_eval_poses")
        TOL.check(got, _oracle(oracle_lib, cx, conf, mm), f"call {k + 1} vs FP64 oracle")


def test_noalloc_fp64_matches_oracle(lib, enepara, oracle_lib):
    torch = pytest.importorskip("torch")
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    mm = synth.config4_poses(8, 32, radius=5.0)
    conf = np.zeros((32, 2), np.int32)
    got, _ = _noalloc(lib, torch, _device_copy(torch, cx), conf, mm, GD_PREC_FP64)
    # the outputs are float32: the FP64 kernel's values rounded once
    err = TOL.relative_error(got, _oracle(oracle_lib, cx, conf, mm))
    assert err.max() <= 2e-7, float(err.max())


def test_noalloc_rejects_sizes_beyond_scratch(lib, enepara):
    torch = pytest.importorskip("torch")
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    cx[0]["size"]["n_lig"] = Lo.MAX_CONF_LIG + 1
    with pytest.raises(GdockError) as ei:
        _noalloc(lib, torch, _device_copy(torch, cx), np.zeros((4, 2), np.int32), np.zeros((4, 6), np.float32))
    assert ei.value.code == GD_E_CAPACITY
    assert "exceeds the fixed scratch" in str(ei.value)


def test_noalloc_refuses_invalid_then_recovers(lib, enepara, oracle_lib):
    """A point type out of range, a class-2 point's seq3r outside the psp
    table, and a pose naming a conformation the Complex does not have are each
    refused with GD_E_INVALID; the next valid call still matches the oracle."""
    torch = pytest.importorskip("torch")
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    mm = synth.config4_poses(9, 16, radius=4.0)
    conf = np.zeros((16, 2), np.int32)
    bad_type = cx.copy()
    bad_type[0]["prt"][0]["t"][3] = 99
    cls2 = int(np.nonzero(cx[0]["prt"][0]["c"][:int(cx[0]["size"]["prt_npoint"])] == 2)[0][0])
    bad_seq = cx.copy()
    bad_seq[0]["prt"][0]["seq3r"][cls2] = Lo.MAXPRO + 5
    for bad, what in ((bad_type, "protein point type"), (bad_seq, "seq3r")):
        with pytest.raises(GdockError) as ei:
            _noalloc(lib, torch, _device_copy(torch, bad), conf, mm)
        assert ei.value.code == GD_E_INVALID, what
    bad_conf = conf.copy()
    bad_conf[5, 1] = 7                           # one protein conformation only
    with pytest.raises(GdockError) as ei:
        _noalloc(lib, torch, _device_copy(torch, cx), bad_conf, mm)
    assert ei.value.code == GD_E_INVALID and "out of range" in str(ei.value)
    got, _ = _noalloc(lib, torch, _device_copy(torch, cx), conf, mm)
    TOL.check(got, _oracle(oracle_lib, cx, conf, mm), "valid call after refusals")
