"""Multi-GPU partitioning exercised on CPU with gloo ranks: replicas are
independent, so ranks take disjoint shards with no data-path collective; one
all_gather of per-shard summaries at the end (what bench.py does with NCCL)."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch

    from bench import shard_range

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b, e = shard_range(3520, rank, world)
        summary = torch.tensor([float(b), float(e), float(e - b)], dtype=torch.float64)
        out = [torch.zeros(3, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(out, summary)
        t = torch.tensor([1.5 * (rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put(([o.tolist() for o in out], float(t)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_shards_cover_replicas(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    shards, tmax = q.get(timeout=10)
    assert tmax == 1.5 * world           # max over ranks, as the bench times ranks
    spans = sorted((int(b), int(e)) for b, e, _ in shards)
    assert spans[0][0] == 0 and spans[-1][1] == 3520
    assert all(spans[i][1] == spans[i + 1][0] for i in range(len(spans) - 1))
    assert np.isclose(sum(n for _, _, n in shards), 3520)
