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


def _shard_worker(rank, world, port, q):
    from geauxdock_b200 import params, shard, synth

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ep = params.optimize_enepara(params.default_enepara0())
        rng = np.random.default_rng(3)
        pk = synth.make_pocket(rng, 200, 4)
        job = synth.make_job(rng, pk, 10, 3, 50, 3, synth.ladder(4, 0.3, 3.0), seed=1)
        cx = synth.to_complex(job, pk, ep, steps_per_exchange=10)
        b, e = shard.replica_range(cx, world, rank)
        local = cx[0]["replica"][b:e].copy()
        local["step"] = rank                     # mark who sent it
        full = shard.gather_replicas(local)
        if rank == 0:
            q.put((b, e, full.tobytes(), cx[0]["replica"][:int(cx[0]["size"]["n_rep"])].tobytes()))
        else:
            q.put((b, e, None, None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_replica_shards_and_gather(world):
    """Each rank's replica range (SetParaT's exchange-aligned split) and the
    gather of the ranks' final states to rank 0, in replica order."""
    from geauxdock_b200 import layout as Lo

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = [q.get(timeout=10) for _ in range(world)]
    spans = sorted((b, e) for b, e, _, _ in got)
    block = 4 * 3                                    # n_tmp * n_lig: one protein-conformation block
    assert spans[0][0] == 0 and all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
    assert all(b % block == 0 for b, _ in spans)
    full, want = next((f, w) for _, _, f, w in got if f is not None)
    full = np.frombuffer(full, dtype=Lo.REPLICA)
    want = np.frombuffer(want, dtype=Lo.REPLICA)
    assert spans[-1][1] == len(want) == len(full)
    for (b, e), r in zip(spans, range(world)):
        assert np.all(full["step"][b:e] == r)
        assert np.array_equal(full["movematrix"][b:e], want["movematrix"][b:e])
        assert np.array_equal(full["idx_rep"][b:e], want["idx_rep"][b:e])


def _queue_worker(rank, world, port, store_path, n_jobs, q):
    import time

    from geauxdock_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        store = dist.FileStore(store_path, world)
        out = []
        # two queues on one store, as dock_queue runs them: the second starts
        # from index 0 again (its own generation of the counter key)
        for gen in range(2):
            local = {}
            for i in shard.claim_jobs(store, n_jobs, shard.queue_key(store, "gd_next_complex")):
                time.sleep(0.002 * (rank + 1))       # ranks of different speed
                local[i] = (rank, i * i + gen)      # stands in for docking complex i
            out.append((len(local), shard.gather_results(local, n_jobs)))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [3])
def test_gloo_complex_queue(world, tmp_path):
    """Ranks claim complexes from one shared counter (the reference's MPI
    server/client dispatch without a dispatching rank): every complex is taken
    exactly once, faster ranks take more, and the results meet on rank 0."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    n_jobs = 60
    procs = [ctx.Process(target=_queue_worker, args=(r, world, port, str(tmp_path / "store"), n_jobs, q))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(world))
    for gen in range(2):
        got = {r: res[r][gen] for r in range(world)}
        assert sum(n for n, _ in got.values()) == n_jobs
        merged = got[0][1]
        assert list(merged) == list(range(n_jobs))
        assert all(v[1] == i * i + gen for i, v in merged.items())
        assert {v[0] for v in merged.values()} == set(range(world))
        assert all(got[r][1] is None for r in range(1, world))


def test_gather_results_rejects_missing():
    """gather_results with n_jobs fails loudly when an index is missing
    (one gloo rank)."""
    from geauxdock_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        assert list(shard.gather_results({0: 1, 1: 2}, 2)) == [0, 1]
        with pytest.raises(RuntimeError, match="missing"):
            shard.gather_results({0: 1, 2: 3}, 3)
    finally:
        dist.destroy_process_group()
