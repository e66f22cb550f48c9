"""Python mirror of the reference's GPU driver (src/main_gpu/geauxdock.C:285-339)
over the drop-in C ABI: SetDevice, DeviceAlloc, InitCurand, then per complex
SetParaT, CopyH2D, Dock; DeviceFree at the end.  Also thin wrappers of the
additive entry points (pose evaluation, resident ensembles)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import layout as Lo
from ._lib import GD_PREC_FP32, check, load


class ParaT(C.Structure):
    _fields_ = [("rep_begin", C.c_int), ("rep_end", C.c_int), ("n_rep", C.c_int), ("record_sz", C.c_int)]


class DockSession:
    """Device buffers and RNG handles for `ngpu` GPUs, reused across complexes."""

    def __init__(self, ngpu: int = 1, seed: int | None = None):
        self.lib = load()
        self.n = ngpu
        check(self.lib.gd_set_ngpu(ngpu))
        self.cd = (C.c_void_p * ngpu)()
        self.rd = (C.c_void_p * ngpu)()
        self.rng = (C.c_void_p * ngpu)()
        self.parat = (ParaT * ngpu)()
        self.pt = (C.POINTER(ParaT) * ngpu)(*[C.pointer(self.parat[g]) for g in range(ngpu)])
        check(self.lib.SetDevice())
        check(self.lib.DeviceAlloc(self.cd, self.rd, self.rng))
        if seed is not None:
            for g in range(ngpu):
                check(self.lib.gd_rng_seed(self.rng[g], seed + g))
        check(self.lib.InitCurand(self.rng))

    def seed(self, seed: int) -> None:
        for g in range(self.n):
            check(self.lib.gd_rng_seed(self.rng[g], seed + g))

    def reuse(self, g: int = 0) -> tuple[int, int]:
        """(Dock calls, calls that refilled the kept device state) of GPU g's handle."""
        calls, reused = C.c_uint64(), C.c_uint64()
        check(self.lib.gd_rng_dock_reuse(self.rng[g], C.byref(calls), C.byref(reused)))
        return calls.value, reused.value

    def dock(self, cx: np.ndarray, record: np.ndarray | None = None) -> np.ndarray:
        """Dock one Complex record in place; returns the Record array (last dump chunk)."""
        assert cx.dtype == Lo.COMPLEX
        nrep = int(cx[0]["size"]["n_rep"])
        if record is None:
            record = Lo.aligned_zeros(Lo.RECORD, nrep)
        ch = C.c_void_p(cx.ctypes.data)
        check(self.lib.SetParaT(ch, self.pt))
        check(self.lib.CopyH2D(ch, self.cd, self.pt))
        check(self.lib.Dock(ch, C.c_void_p(record.ctypes.data), self.cd, self.rd, self.pt, self.rng))
        return record

    def close(self) -> None:
        if self.cd is not None:
            check(self.lib.DeviceFree(self.cd, self.rd, self.rng))
            self.cd = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def eval_poses(cx: np.ndarray, conf: np.ndarray, mm: np.ndarray, precision: int = GD_PREC_FP32,
               want64: bool = False):
    """Energies of poses on the GPU: returns (out[n,10] float32, raw[n,9] float32, out64 or None)."""
    lib = load()
    conf = np.ascontiguousarray(conf, dtype=np.int32).reshape(-1, 2)
    mm = np.ascontiguousarray(mm, dtype=np.float32).reshape(-1, 6)
    n = len(conf)
    out = np.zeros((n, 10), dtype=np.float32)
    raw = np.zeros((n, 9), dtype=np.float32)
    out64 = np.zeros((n, 10), dtype=np.float64) if want64 else None
    check(lib.gd_eval_poses(C.c_void_p(cx.ctypes.data), n, C.c_void_p(conf.ctypes.data),
                            C.c_void_p(mm.ctypes.data), precision, C.c_void_p(out.ctypes.data),
                            C.c_void_p(out64.ctypes.data) if want64 else None, C.c_void_p(raw.ctypes.data)))
    return out, raw, out64


class Ensemble:
    """A resident ensemble (gd_ensemble_*)."""

    def __init__(self, handle: C.c_void_p, njob: int, keep=None):
        self.lib = load()
        self.h = handle
        self.njob = njob
        self._keep = keep

    @classmethod
    def from_complexes(cls, cxs, seeds, device: int = 0) -> "Ensemble":
        lib = load()
        arr = (C.c_void_p * len(cxs))(*[c.ctypes.data for c in cxs])
        sd = (C.c_uint64 * len(cxs))(*seeds)
        h = C.c_void_p()
        check(lib.gd_ensemble_create_complex(arr, len(cxs), sd, device, C.byref(h)))
        return cls(h, len(cxs))

    @classmethod
    def from_jobs(cls, pockets, jobs, enepara: np.ndarray, device: int = 0) -> "Ensemble":
        from . import synth

        lib = load()
        keep: list = []
        from ._lib import JobDesc, PocketDesc

        parr = (PocketDesc * len(pockets))(*[synth.pocket_desc(p, keep) for p in pockets])
        jarr = (JobDesc * len(jobs))(*[synth.job_desc(j, keep) for j in jobs])
        ep = np.array([enepara], dtype=Lo.ENEPARA)
        keep.append(ep)
        h = C.c_void_p()
        check(lib.gd_ensemble_create(parr, len(pockets), jarr, len(jobs), C.c_void_p(ep.ctypes.data), device,
                                     C.byref(h)))
        return cls(h, len(jobs), keep)

    def init(self) -> None:
        check(self.lib.gd_ensemble_init(self.h))

    def run(self, nsteps: int, steps_per_exchange: int = 0) -> None:
        check(self.lib.gd_ensemble_run(self.h, nsteps, steps_per_exchange))

    def sync(self, all_launches: bool = False):
        """Wait; returns (Monte Carlo kernel ms, Monte Carlo launches[, all kernel launches])."""
        ms = C.c_double()
        nl = C.c_int()
        na = C.c_int()
        check(self.lib.gd_ensemble_sync(self.h, C.byref(ms), C.byref(nl), C.byref(na)))
        return (ms.value, nl.value, na.value) if all_launches else (ms.value, nl.value)

    def replicas(self, job: int = 0) -> np.ndarray:
        n = check(self.lib.gd_ensemble_num_replicas(self.h, job))
        out = Lo.aligned_zeros(Lo.REPLICA, n)
        check(self.lib.gd_ensemble_replicas(self.h, job, C.c_void_p(out.ctypes.data)))
        return out

    def stats(self, job: int = 0) -> np.ndarray:
        n = check(self.lib.gd_ensemble_num_replicas(self.h, job))
        out = np.zeros((n, 8), dtype=np.float64)
        check(self.lib.gd_ensemble_stats(self.h, job, C.c_void_p(out.ctypes.data)))
        return out

    def eval_poses(self, job: int, conf: np.ndarray, mm: np.ndarray, precision: int = GD_PREC_FP32,
                   want64: bool = False, want_raw: bool = False):
        """Energies of arbitrary poses of one job: (out [n,10] float32, raw [n,9] or None, out64 or None)."""
        conf = np.ascontiguousarray(conf, dtype=np.int32).reshape(-1, 2)
        mm = np.ascontiguousarray(mm, dtype=np.float32).reshape(-1, 6)
        n = len(mm)
        out = np.zeros((n, 10), np.float32)
        raw = np.zeros((n, 9), np.float32) if want_raw else None
        out64 = np.zeros((n, 10), np.float64) if want64 else None
        check(self.lib.gd_ensemble_eval_poses(self.h, job, n, conf.ctypes.data, mm.ctypes.data, precision,
                                              out.ctypes.data, None if out64 is None else out64.ctypes.data,
                                              None if raw is None else raw.ctypes.data))
        return out, raw, out64

    def best_poses(self, job: int = 0):
        """Each replica's best pose: (movematrix [nrep, 6] float32, total energy [nrep] float64)."""
        n = check(self.lib.gd_ensemble_num_replicas(self.h, job))
        mm = np.zeros((n, 6), np.float32)
        e = np.zeros(n, np.float64)
        check(self.lib.gd_ensemble_best_poses(self.h, job, mm.ctypes.data, e.ctypes.data))
        return mm, e

    def cluster(self, job: int = 0, rmsd_cut: float = 2.0, ref_lig: int = 0, ref_mm=None, max_clusters: int = 4096):
        """Best pose per replica, RMSD to the reference pose (default: the native pose) and leader
        clustering in energy order: (list of cluster dicts, cluster_of [nrep], rmsd_to_ref [nrep])."""
        from ._lib import Cluster

        n = check(self.lib.gd_ensemble_num_replicas(self.h, job))
        out = (Cluster * max_clusters)()
        ncl = C.c_int()
        cof = np.zeros(n, np.int32)
        rmsd = np.zeros(n, np.float32)
        mm = None if ref_mm is None else np.ascontiguousarray(ref_mm, np.float32)
        check(self.lib.gd_ensemble_cluster(self.h, job, ref_lig, None if mm is None else mm.ctypes.data, rmsd_cut,
                                           out, max_clusters, C.byref(ncl), cof.ctypes.data, rmsd.ctypes.data))
        cl = [{k: getattr(c, k) for k, _ in Cluster._fields_ if k != "pad_"} for c in out[:min(ncl.value, max_clusters)]]
        return cl, cof, rmsd

    def snapshot(self) -> bytes:
        """Checkpoint of the resident state (gd_ensemble_snapshot): replicas, accept
        flags, FP64 statistics and the step counter."""
        n = self.lib.gd_ensemble_snapshot_bytes(self.h)
        buf = C.create_string_buffer(n)
        check(self.lib.gd_ensemble_snapshot(self.h, buf, n))
        return buf.raw

    def restore(self, snap: bytes) -> None:
        """Resume from a checkpoint of an ensemble of the same jobs and seeds."""
        check(self.lib.gd_ensemble_restore(self.h, snap, len(snap)))

    def autotune(self, steps: int = 4) -> str:
        buf = C.create_string_buffer(8192)
        check(self.lib.gd_ensemble_autotune(self.h, steps, buf, len(buf)))
        return buf.value.decode()

    def close(self) -> None:
        if self.h:
            self.lib.gd_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Server:
    """A request loop on one GPU (gd_server_*): resident pockets, requests
    admitted by an HBM budget into running rounds (continuous batching)."""

    def __init__(self, pockets, enepara: np.ndarray, device: int = 0, **config):
        from . import synth
        from ._lib import PocketDesc, ServerConfig

        self.lib = load()
        self.h = None
        self._keep: list = []
        cfg = ServerConfig()
        self.lib.gd_server_config_default(C.byref(cfg))
        for k, v in config.items():
            if not hasattr(cfg, k):
                raise TypeError(f"unknown server option {k!r}")
            setattr(cfg, k, v)
        cfg.device = device
        parr = (PocketDesc * len(pockets))(*[synth.pocket_desc(p, self._keep) for p in pockets])
        ep = np.array([enepara], dtype=Lo.ENEPARA)
        self._keep.append(ep)
        h = C.c_void_p()
        check(self.lib.gd_server_create(parr, len(pockets), C.c_void_p(ep.ctypes.data), C.byref(cfg), C.byref(h)))
        self.h = h
        self._pocket_nconf = [p.nconf for p in pockets]
        self._live: dict = {}   # ticket -> (arrays kept alive, replicas, stats)

    def submit(self, job, steps: int, steps_per_exchange: int = 0, results: bool = True) -> int:
        """Queue a docking request (synth.Job-like; job.pocket indexes the pockets); returns its ticket."""
        from . import synth
        from ._lib import Request

        keep: list = []
        jd = synth.job_desc(job, keep)
        keep.append(jd)
        nrep = job.nlig * job.ntmp * self._nconf(job.pocket)
        rep = Lo.aligned_zeros(Lo.REPLICA, nrep) if results else None
        st = np.zeros((nrep, 8), np.float64) if results else None
        req = Request()
        req.job = C.addressof(jd)
        req.steps = steps
        req.steps_per_exchange = steps_per_exchange
        req.replicas_out = rep.ctypes.data if results else None
        req.stats_out = st.ctypes.data if results else None
        t = C.c_longlong()
        check(self.lib.gd_server_submit(self.h, C.byref(req), C.byref(t)))
        self._live[t.value] = (keep, rep, st)
        return t.value

    def _nconf(self, pocket: int) -> int:
        # an out-of-range index is refused by gd_server_submit
        return self._pocket_nconf[pocket] if 0 <= pocket < len(self._pocket_nconf) else 0

    def poll(self, max_results: int = 64, timeout_ms: int = -1) -> list:
        """Finished requests: dicts with ticket, status, times and (if kept) replicas / stats."""
        from ._lib import Result

        buf = (Result * max_results)()
        n = check(self.lib.gd_server_poll(self.h, buf, max_results, timeout_ms))
        out = []
        for r in buf[:n]:
            keep, rep, st = self._live.pop(r.ticket, (None, None, None))
            out.append({"ticket": r.ticket, "status": r.status, "nrep": r.nrep, "steps": r.steps,
                        "t_submit": r.t_submit, "t_admit": r.t_admit, "t_done": r.t_done,
                        "replicas": rep, "stats": st})
        return out

    def drain(self, timeout_ms: int = -1) -> None:
        check(self.lib.gd_server_drain(self.h, timeout_ms))

    def cancel(self, ticket: int) -> None:
        """Cancel a queued or running request (its result reports GD_E_CANCELLED)."""
        check(self.lib.gd_server_cancel(self.h, ticket))

    def stats(self) -> dict:
        from ._lib import ServerStats

        s = ServerStats()
        check(self.lib.gd_server_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_ if k != "pad_"}

    def close(self) -> None:
        if self.h:
            self.lib.gd_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
