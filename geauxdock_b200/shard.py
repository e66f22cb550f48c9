"""One process per GPU (torchrun): each rank runs its shard of a Complex's
replicas and rank 0 gathers the final replica states.

The shard of rank g of N is SetParaT's split (src/backend_gpu/prepair.C:366-392),
cut at protein-conformation blocks when replica exchange is on, so exchange
partners never straddle ranks and the Monte Carlo data path needs no
collective.  Philox counters use the global replica index, so with one seed on
every rank each replica's trajectory does not depend on N.  The only
collective is the gather of the results at the end (NCCL between GPUs, gloo
on CPU).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import layout as Lo
from ._lib import check, load


def replica_range(cx: np.ndarray, world: int, rank: int) -> tuple[int, int]:
    """[begin, end) of rank's replicas among `world` ranks."""
    b, e = C.c_int(), C.c_int()
    check(load().gd_replica_range(C.c_void_p(cx.ctypes.data), world, rank, C.byref(b), C.byref(e)))
    return b.value, e.value + 1


def run_shard(cx: np.ndarray, steps: int, steps_per_exchange: int, seed: int, rank: int, world: int,
              device: int = 0) -> np.ndarray:
    """Initial energies and `steps` MC steps of this rank's replicas; returns their final states."""
    from .dock import Ensemble

    lib = load()
    b, e = replica_range(cx, world, rank)
    h = C.c_void_p()
    check(lib.gd_ensemble_create_complex_range(C.c_void_p(cx.ctypes.data), b, e - 1, seed, device, C.byref(h)))
    with Ensemble(h, 1) as ens:
        ens.init()
        if steps:
            ens.run(steps, steps_per_exchange)
        ens.sync()
        return ens.replicas(0)


def gather_replicas(local: np.ndarray, device=None) -> np.ndarray | None:
    """All ranks' replica states, in rank order, on rank 0 (None elsewhere).
    One all_gather of the sizes and one of the padded bytes."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(), dist.get_rank()
    raw = np.ascontiguousarray(local).view(np.uint8).reshape(-1)
    dev = torch.device(device) if device is not None else torch.device("cpu")
    n = torch.tensor([raw.size], dtype=torch.int64, device=dev)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(sizes, n)
    cap = int(max(int(s.item()) for s in sizes))
    buf = torch.zeros(cap, dtype=torch.uint8, device=dev)
    buf[:raw.size] = torch.from_numpy(raw.copy()).to(dev)
    parts = [torch.zeros(cap, dtype=torch.uint8, device=dev) for _ in range(world)]
    dist.all_gather(parts, buf)
    if rank != 0:
        return None
    out = [p[:int(s.item())].cpu().numpy() for p, s in zip(parts, sizes)]
    return np.concatenate(out).view(Lo.REPLICA)
