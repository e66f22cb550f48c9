"""ctypes access to the checkers (TEST INFRASTRUCTURE ONLY).

liboracle.so  -- the FP64 C restatement (gd_oracle.c).
_ref/libgdref.so -- the reference's own CPU code built from its sources.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
these; the product never does.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libgdref.so"

_ora = None
_ref = None


def build(reference: str | None = None) -> None:
    """make the FP64 oracle (always) and the reference library (when the sources are present)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    from oracle.refpath import reference_sources

    ref = reference or reference_sources()
    if ref is not None and Path(ref, "src").is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={ref}"], check=True)


def oracle() -> C.CDLL:
    global _ora
    if _ora is None:
        lib = C.CDLL(str(ORACLE_SO))
        vp = C.c_void_p
        lib.gdo_energy.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp]
        lib.gdo_montecarlo.argtypes = [vp, vp, C.c_int, C.c_int, C.c_uint64, C.c_int]
        lib.gdo_exchange.argtypes = [vp, C.c_int, C.c_uint64]
        lib.gdo_philox4x32_10.argtypes = [vp, vp, vp]
        lib.gdo_u01.argtypes = [C.c_uint32]
        lib.gdo_u01.restype = C.c_float
        lib.gdo_energy_desc_batch.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, vp]
        _ora = lib
    return _ora


def have_ref() -> bool:
    return REF_SO.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_SO))
        vp = C.c_void_p
        lib.gdref_dock.argtypes = [vp, vp]
        lib.gdref_montecarlo.argtypes = [vp, vp, C.c_int, C.c_int]
        lib.gdref_set_threads.argtypes = [C.c_int]
        lib.gdref_max_threads.restype = C.c_int
        lib.gdref_sizeof.argtypes = [C.c_char_p]
        lib.gdref_sizeof.restype = C.c_size_t
        lib.gdref_load_enepara.argtypes = [C.c_char_p] * 4 + [vp, vp]
        lib.gdref_optimize_enepara.argtypes = [vp, vp]
        lib.gdref_load_complex.argtypes = [C.c_char_p] * 8 + [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                                               C.c_int, C.c_int, vp]
        _ref = lib
    return _ref


def ref_optimize_enepara(ep0: np.ndarray) -> np.ndarray:
    """The reference's own OptimizeEnepara (util_optimize_soa.C:489-540) on a raw
    EnePara0 record: an EnePara record, built without libgdock.so."""
    from geauxdock_b200 import layout as Lo

    src = np.array([ep0], dtype=Lo.ENEPARA0)
    out = np.zeros(1, dtype=Lo.ENEPARA)
    ref().gdref_optimize_enepara(src.ctypes.data, out.ctypes.data)
    return out[0]


def mapped_libraries(root: Path) -> list[str]:
    """Shared objects under `root` that this process has mapped (/proc/self/maps)."""
    out = set()
    try:
        for ln in Path("/proc/self/maps").read_text().splitlines():
            f = ln.split()[-1] if ln.split() else ""
            if f.endswith(".so") and f.startswith(str(root)):
                out.add(str(Path(f).relative_to(root)))
    except OSError:
        pass
    return sorted(out)


def energy(cx: np.ndarray, il: int, ip: int, mm) -> tuple[np.ndarray, np.ndarray]:
    """FP64 oracle energy of one pose: (e[10], raw[9])."""
    m = np.ascontiguousarray(mm, dtype=np.float32)
    e = np.zeros(10)
    raw = np.zeros(9)
    oracle().gdo_energy(cx.ctypes.data, il, ip, m.ctypes.data, e.ctypes.data, raw.ctypes.data)
    return e, raw


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    oracle().gdo_philox4x32_10(c.ctypes.data, k.ctypes.data, o.ctypes.data)
    return o


def montecarlo(cx: np.ndarray, record, s1: int, s2max: int, seed: int, steps_per_exchange: int = 0) -> None:
    oracle().gdo_montecarlo(cx.ctypes.data, None if record is None else record.ctypes.data, s1, s2max, seed,
                            steps_per_exchange)


def ref_energies(cx: np.ndarray, reps: np.ndarray | None = None) -> np.ndarray:
    """The reference's own FP32 energy of every replica's stored pose: MonteCarlo_d with
    s2max == 1 (no move, forced accept; kernel_cpp_montecarlo_soa.C:248, :384).  Returns
    energy[n_rep, 10]; cx is not modified."""
    from geauxdock_b200 import layout as Lo

    work = cx.copy()
    if reps is not None:
        work[0]["replica"][: len(reps)] = reps
    n = int(work[0]["size"]["n_rep"])
    work[0]["rep_begin"], work[0]["rep_end"] = 0, n - 1
    for r in range(n):
        work[0]["replica"][r]["is_accept"] = 0
    rec = Lo.aligned_zeros(Lo.RECORD, n)
    ref().gdref_montecarlo(work.ctypes.data, rec.ctypes.data, 0, 1)
    return np.array(work[0]["replica"]["energy"][:n])


def energy_desc(pocket, job, enepara: np.ndarray, conf: np.ndarray, mm: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """FP64 energies of n poses of a cap-free job (synth.Pocket / synth.Job): (e [n,10], raw [n,9])."""
    from geauxdock_b200 import layout as Lo, synth

    keep: list = []
    pd = synth.pocket_desc(pocket, keep)
    jd = synth.job_desc(job, keep)
    ep = np.array([enepara], dtype=Lo.ENEPARA)
    conf = np.ascontiguousarray(conf, dtype=np.int32)
    mm = np.ascontiguousarray(mm, dtype=np.float32)
    n = len(mm)
    e = np.zeros((n, 10), np.float64)
    raw = np.zeros((n, 9), np.float64)
    oracle().gdo_energy_desc_batch(C.byref(pd), C.byref(jd), ep.ctypes.data, n, conf.ctypes.data, mm.ctypes.data,
                                   e.ctypes.data, raw.ctypes.data)
    return e, raw
