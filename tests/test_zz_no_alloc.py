"""gd_eval_poses_noalloc: pose energies for callers that cannot allocate
device memory around a docking call (a process whose device memory belongs to
another allocator, or a serving loop that cannot afford cudaFree's device-wide
synchronisation).  The caller passes device buffers it already owns -- here
torch tensors stand in for such memory -- and the library uses only its fixed
scratch array.  Its output must match the allocating entry point
gd_eval_poses within the energy tolerance of the other GPU tests, on two
different complexes evaluated one after the other (so the second call also
shows that nothing stale from the first call's scratch contents leaks in).

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""

import ctypes as C

import numpy as np
import pytest

from geauxdock_b200 import dock, layout as Lo, synth
from geauxdock_b200._lib import GD_E_CAPACITY, GD_PREC_FP32, GdockError, check

pytestmark = pytest.mark.gpu
TOL32 = 1e-5


def _device_copy(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()


def _noalloc(lib, torch, d_cx, conf, mm):
    n = len(conf)
    d_conf = torch.from_numpy(np.ascontiguousarray(conf, np.int32)).cuda()
    d_mm = torch.from_numpy(np.ascontiguousarray(mm, np.float32)).cuda()
    d_out = torch.full((n, 10), float("nan"), dtype=torch.float32, device="cuda")
    d_raw = torch.full((n, 9), float("nan"), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    check(lib.gd_eval_poses_noalloc(C.c_void_p(d_cx.data_ptr()), n, C.c_void_p(d_conf.data_ptr()),
                                    C.c_void_p(d_mm.data_ptr()), GD_PREC_FP32, C.c_void_p(d_out.data_ptr()),
                                    C.c_void_p(d_raw.data_ptr()), C.c_void_p(stream)))
    return d_out.cpu().numpy(), d_raw.cpu().numpy()


def _close(a, b):
    scale = np.maximum(np.abs(b.astype(np.float64)), 1.0)
    err = np.abs(a.astype(np.float64) - b) / scale
    assert np.isfinite(a).all()
    assert err.max() <= TOL32, float(err.max())


def test_noalloc_matches_eval_poses_two_calls(lib, enepara):
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
    for cx, conf, mm in ((cx2, conf2, mm2), (cx1, conf1, mm1)):
        want, want_raw, _ = dock.eval_poses(cx, conf, mm, GD_PREC_FP32)
        got, got_raw = _noalloc(lib, torch, _device_copy(torch, cx), conf, mm)
        _close(got, want)


def test_noalloc_rejects_sizes_beyond_scratch(lib, enepara):
    torch = pytest.importorskip("torch")
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    cx[0]["size"]["n_lig"] = Lo.MAX_CONF_LIG + 1
    with pytest.raises(GdockError) as ei:
        _noalloc(lib, torch, _device_copy(torch, cx), np.zeros((4, 2), np.int32), np.zeros((4, 6), np.float32))
    assert ei.value.code == GD_E_CAPACITY
    assert "exceeds the fixed scratch" in str(ei.value)
