"""One process per GPU (torchrun), on one node or several: each rank runs its
shard of a Complex's replicas and rank 0 gathers the final replica states; or,
for many complexes, ranks take whole complexes from a shared queue.

The shard of rank g of N is SetParaT's split (src/backend_gpu/prepair.C:366-392),
cut at protein-conformation blocks when replica exchange is on, so exchange
partners never straddle ranks and the Monte Carlo data path needs no
collective.  Philox counters use the global replica index, so with one seed on
every rank each replica's trajectory does not depend on N.  The only
collective is the gather of the results at the end (NCCL between GPUs, gloo
on CPU).

Many complexes (the reference's MPI screening, src/main_mpi/server.C:27-66 and
client_gpu.C): the reference's rank 0 hands the next complex to whichever
client asks, and each client docks it with Dock.  Here every rank, rank 0
included, claims the next complex index from one counter in a key-value store
that all ranks share (a torch.distributed Store: TCPStore across nodes,
FileStore or HashStore for tests), docks it on its own GPU through the drop-in
Dock, and the results meet on rank 0 in one gather.  No rank only dispatches,
and there is no MPI.
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


def complex_seed(seed: int, index: int) -> int:
    """The RNG seed of complex `index` in a queue seeded with `seed`: a complex's
    result does not depend on which rank docks it or in what order."""
    return (seed + 0x9E3779B97F4A7C15 * (index + 1)) & 0xFFFFFFFFFFFFFFFF


def claim_jobs(store, n_jobs: int, key: str = "gd_next_complex"):
    """Yield the indices this rank claims, one at a time, from the counter `key`
    in `store`, until all n_jobs are taken.  Every index goes to exactly one rank;
    a fast rank simply claims more (the reference's idle client asking the server)."""
    while True:
        i = int(store.add(key, 1)) - 1
        if i >= n_jobs:
            return
        yield i


_queue_generation: dict = {}


def queue_key(store, key: str) -> str:
    """The counter key of this process's next queue on `store`: `key` with a
    generation suffix.  Every rank calls dock_queue the same number of times
    (it is collective, like gather_results), so the ranks agree on the
    generation, and a second queue on the same store starts from 0 instead of
    past the first queue's end."""
    g = _queue_generation.get((id(store), key), 0)
    _queue_generation[(id(store), key)] = g + 1
    return f"{key}/{g}"


def dock_queue(complexes, seed: int, store, key: str = "gd_next_complex") -> dict:
    """Dock the complexes this rank claims from the shared counter on this
    process's GPU (the library's `device_base` option selects it) through
    SetParaT / CopyH2D / Dock, each with RNG seed complex_seed(seed, index).
    Collective: every rank calls it, once per queue.
    Returns {index: final replica states of that complex}."""
    from .dock import DockSession

    out = {}
    qkey = queue_key(store, key)
    with DockSession(1) as s:
        for i in claim_jobs(store, len(complexes), qkey):
            cx = complexes[i].copy()
            s.seed(complex_seed(seed, i))
            s.dock(cx)
            out[i] = cx[0]["replica"][:int(cx[0]["size"]["n_rep"])].copy()
    return out


def gather_results(local: dict, n_jobs: int | None = None) -> dict | None:
    """Every rank's {index: result} merged on rank 0 (None elsewhere), in one
    all_gather_object of the process group.  With n_jobs, rank 0 checks that
    indices 0..n_jobs-1 all arrived, each once."""
    import torch.distributed as dist

    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, local)
    if dist.get_rank() != 0:
        return None
    merged = {}
    for part in parts:
        for i, r in part.items():
            if i in merged:
                raise RuntimeError(f"complex {i} docked twice")
            merged[i] = r
    if n_jobs is not None and sorted(merged) != list(range(n_jobs)):
        missing = sorted(set(range(n_jobs)) - set(merged))
        raise RuntimeError(f"{len(merged)} of {n_jobs} complexes gathered; missing {missing[:8]}")
    return dict(sorted(merged.items()))
