"""ctypes bindings of libgdock.so (include/gdock.h).

The library is the product: there is no Python or CPU fallback.  Loading
fails with an error if libgdock.so is missing, and every call that returns a
negative status raises GdockError with the library's message.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgdock.so"

GD_OK = 0
GD_E_INVALID = -1
GD_E_NOMEM = -2
GD_E_CAPACITY = -3
GD_E_CUDA = -4
GD_E_TIMEOUT = -5
GD_E_NODEVICE = -6
GD_E_STATE = -7
GD_E_BUSY = -8
GD_E_CANCELLED = -9

GD_KERNEL_BATCHED = 0
GD_KERNEL_PLAIN = 1
GD_PREC_FP32 = 0
GD_PREC_FP32_KAHAN = 1
GD_PREC_FP64 = 2

# Every extern "C" symbol include/gdock.h declares.
EXPORTED = [
    "gd_last_error", "gd_set_ngpu", "gd_get_ngpu",
    "SetDevice", "DeviceAlloc", "DeviceFree", "SetParaT", "CopyH2D", "InitCurand", "gd_rng_seed", "gd_rng_dock_reuse", "Dock",
    "gd_set_option", "gd_get_option", "gd_eval_poses",
    "gd_ensemble_create", "gd_ensemble_create_complex", "gd_ensemble_init", "gd_ensemble_run",
    "gd_ensemble_sync", "gd_ensemble_num_replicas", "gd_ensemble_replicas", "gd_ensemble_stats",
    "gd_ensemble_autotune", "gd_ensemble_destroy", "gd_ensemble_eval_poses",
    "gd_replica_range", "gd_ensemble_create_complex_range", "gd_load_complex", "gd_ensemble_cluster",
    "gd_ensemble_best_poses", "gd_ensemble_snapshot_bytes", "gd_ensemble_snapshot", "gd_ensemble_restore",
    "gd_layout", "gd_optimize_enepara", "gd_ensemble_stream", "gd_fp32_peak",
    "gd_eval_poses_noalloc", "gd_noalloc_scratch_bytes",
    "gd_server_config_default", "gd_server_create", "gd_server_submit", "gd_server_poll", "gd_server_drain",
    "gd_server_get_stats", "gd_server_destroy", "gd_server_cancel", "gd_check_report",
]


class ServerConfig(C.Structure):
    """gd_server_config_t."""
    _fields_ = [
        ("hbm_budget_bytes", C.c_ulonglong), ("max_active_replicas", C.c_int), ("max_jobs", C.c_int),
        ("max_replicas_per_job", C.c_int), ("max_atoms", C.c_int), ("steps_per_round", C.c_int),
        ("kde_stage", C.c_int), ("warps", C.c_int), ("device", C.c_int), ("replica_warps", C.c_int),
    ]


class Request(C.Structure):
    """gd_request_t."""
    _fields_ = [
        ("job", C.c_void_p), ("steps", C.c_int), ("steps_per_exchange", C.c_int),
        ("replicas_out", C.c_void_p), ("stats_out", C.c_void_p),
    ]


class Result(C.Structure):
    """gd_result_t."""
    _fields_ = [
        ("ticket", C.c_longlong), ("status", C.c_int), ("nrep", C.c_int), ("steps", C.c_int), ("pad_", C.c_int),
        ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
    ]


class ServerStats(C.Structure):
    """gd_server_stats_t."""
    _fields_ = [
        ("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
        ("queued", C.c_longlong), ("outstanding", C.c_longlong), ("rounds", C.c_longlong),
        ("launches", C.c_longlong), ("pose_evals", C.c_double), ("device_ms", C.c_double), ("now", C.c_double),
        ("used_bytes", C.c_ulonglong), ("peak_bytes", C.c_ulonglong),
        ("warps_per_cta", C.c_int), ("grid", C.c_int), ("max_active_replicas", C.c_int),
        ("pocket_staged", C.c_int), ("latency_rounds", C.c_longlong),
    ]


class LoadArgs(C.Structure):
    """gd_load_args_t."""
    _fields_ = [
        ("lig_sdf", C.c_char_p), ("lhm_ff", C.c_char_p), ("prt_pdb", C.c_char_p), ("ligand_id", C.c_char_p),
        ("molid", C.c_char_p), ("enepara0", C.c_void_p), ("enepara", C.c_void_p), ("num_temp", C.c_int),
        ("floor_temp", C.c_float), ("ceiling_temp", C.c_float), ("translation_step", C.c_float),
        ("rotation_step", C.c_float), ("steps_total", C.c_int), ("steps_per_dump", C.c_int),
        ("steps_per_exchange", C.c_int),
    ]


class Cluster(C.Structure):
    """gd_cluster_t."""
    _fields_ = [
        ("representative", C.c_int), ("size", C.c_int), ("relative_size", C.c_float), ("z_score", C.c_float),
        ("rep_energy", C.c_float), ("mean_energy", C.c_float), ("rep_rmsd", C.c_float), ("pad_", C.c_int),
    ]


class GdockError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gdock error {code}: {msg}")
        self.code = code


class JobDesc(C.Structure):
    """gd_job_desc_t."""
    _fields_ = [
        ("natom", C.c_int), ("nlig", C.c_int),
        ("lig_xyz", C.c_void_p), ("lig_type", C.c_void_p), ("lig_charge", C.c_void_p), ("lig_center", C.c_void_p),
        ("pocket", C.c_int),
        ("nkde", C.c_int), ("kde_xyz", C.c_void_p), ("kde_type", C.c_void_p),
        ("nmcs", C.c_int), ("mcs_xyz", C.c_void_p), ("mcs_tcc", C.c_void_p),
        ("psp_ncol", C.c_int), ("psp", C.c_void_p),
        ("ntmp", C.c_int), ("temperature", C.c_void_p),
        ("move_scale", C.c_float * 6),
        ("seed", C.c_uint64),
    ]


class PocketDesc(C.Structure):
    """gd_pocket_desc_t."""
    _fields_ = [
        ("npoint", C.c_int), ("nconf", C.c_int),
        ("xyz", C.c_void_p), ("type", C.c_void_p), ("cls", C.c_void_p), ("cdc", C.c_void_p),
        ("seq3r", C.c_void_p), ("hpp", C.c_void_p), ("ele", C.c_void_p), ("center", C.c_void_p),
    ]


_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libgdock.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    # GDOCK_LIB selects another build of the library (the bounds-checking
    # libgdock_check.so in its tests)
    p = Path(path) if path else Path(os.environ.get("GDOCK_LIB") or LIB_PATH)
    if not p.exists():
        raise GdockError(GD_E_STATE, f"{p} not built (python -m geauxdock_b200.build)")
    lib = C.CDLL(str(p))
    vp, ip, i, ll = C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_longlong
    sig = {
        "gd_last_error": (C.c_char_p, []),
        "gd_set_ngpu": (i, [i]), "gd_get_ngpu": (i, []),
        "SetDevice": (i, []), "DeviceAlloc": (i, [vp, vp, vp]), "DeviceFree": (i, [vp, vp, vp]),
        "SetParaT": (i, [vp, vp]), "CopyH2D": (i, [vp, vp, vp]), "InitCurand": (i, [vp]),
        "gd_rng_seed": (i, [vp, C.c_uint64]), "gd_rng_dock_reuse": (i, [vp, vp, vp]), "Dock": (i, [vp, vp, vp, vp, vp, vp]),
        "gd_set_option": (i, [C.c_char_p, ll]), "gd_get_option": (ll, [C.c_char_p]),
        "gd_eval_poses": (i, [vp, i, vp, vp, i, vp, vp, vp]),
        "gd_ensemble_create": (i, [vp, i, vp, i, vp, i, vp]),
        "gd_ensemble_create_complex": (i, [vp, i, vp, i, vp]),
        "gd_ensemble_init": (i, [vp]), "gd_ensemble_run": (i, [vp, i, i]),
        "gd_ensemble_sync": (i, [vp, C.POINTER(C.c_double), ip, ip]),
        "gd_ensemble_num_replicas": (i, [vp, i]), "gd_ensemble_replicas": (i, [vp, i, vp]),
        "gd_ensemble_stats": (i, [vp, i, vp]), "gd_ensemble_autotune": (i, [vp, i, C.c_char_p, i]),
        "gd_ensemble_destroy": (i, [vp]), "gd_layout": (ll, [C.c_char_p]),
        "gd_ensemble_eval_poses": (i, [vp, i, i, vp, vp, i, vp, vp, vp]),
        "gd_replica_range": (i, [vp, i, i, ip, ip]),
        "gd_load_complex": (i, [vp, vp]),
        "gd_ensemble_cluster": (i, [vp, i, i, vp, C.c_float, vp, i, ip, vp, vp]),
        "gd_ensemble_best_poses": (i, [vp, i, vp, vp]),
        "gd_ensemble_snapshot_bytes": (C.c_size_t, [vp]),
        "gd_ensemble_snapshot": (i, [vp, vp, C.c_size_t]), "gd_ensemble_restore": (i, [vp, vp, C.c_size_t]),
        "gd_ensemble_create_complex_range": (i, [vp, i, i, C.c_uint64, i, vp]),
        "gd_optimize_enepara": (i, [vp, vp]),
        "gd_ensemble_stream": (vp, [vp]), "gd_fp32_peak": (i, [C.POINTER(C.c_double)]),
        "gd_eval_poses_noalloc": (i, [vp, i, vp, vp, i, vp, vp, vp]), "gd_noalloc_scratch_bytes": (C.c_size_t, []),
        "gd_server_config_default": (None, [vp]),
        "gd_server_create": (i, [vp, i, vp, vp, vp]),
        "gd_server_submit": (i, [vp, vp, C.POINTER(ll)]),
        "gd_server_poll": (i, [vp, vp, i, i]),
        "gd_server_drain": (i, [vp, i]),
        "gd_server_get_stats": (i, [vp, vp]),
        "gd_server_destroy": (i, [vp]),
        "gd_server_cancel": (i, [vp, ll]),
        "gd_check_report": (i, [ip, i]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> int:
    """Raise GdockError for a negative status."""
    if rc < 0:
        msg = load().gd_last_error()
        raise GdockError(rc, msg.decode() if msg else "")
    return rc


def layout(what: str) -> int:
    return int(load().gd_layout(what.encode()))
