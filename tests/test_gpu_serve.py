"""The request loop (gd_server_*): results equal the resident-ensemble path bit
for bit, each request's result is the same alone and in a mix of others that
arrive while it runs, admission respects the HBM budget, and bad requests
are refused at submission."""

import time

import numpy as np
import pytest

from geauxdock_b200 import dock, synth
from geauxdock_b200._lib import GD_E_CAPACITY, GD_E_INVALID, GdockError

pytestmark = pytest.mark.gpu


def _pockets():
    rng = np.random.default_rng(21)
    return [synth.make_pocket(rng, 350, 2), synth.make_pocket(rng, 700, 3)]


def _jobs(pockets, n, seed=5, sizes=(9, 33, 80, 17, 64, 45)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        pi = i % len(pockets)
        L = sizes[i % len(sizes)]
        out.append(synth.make_job(rng, pockets[pi], L, 2, 150, 5, synth.ladder(4, 0.3, 3.0), seed=100 + i,
                                  pocket_index=pi))
    return out


def _ensemble_result(pockets, job, enepara, steps, spx):
    with dock.Ensemble.from_jobs(pockets, [job], enepara) as e:
        e.init()
        e.run(steps, spx)
        e.sync()
        return e.replicas(0), e.stats(0)


def _serve(pockets, enepara, reqs, stagger_s=0.0, **cfg):
    with dock.Server(pockets, enepara, **cfg) as srv:
        tickets = []
        for job, steps, spx in reqs:
            tickets.append(srv.submit(job, steps, spx))
            if stagger_s:
                time.sleep(stagger_s)
        srv.drain(120_000)
        res = {r["ticket"]: r for r in srv.poll(len(reqs), 0)}
        st = srv.stats()
    assert len(res) == len(reqs)
    return [res[t] for t in tickets], st


def test_server_matches_ensemble(lib, enepara):
    pockets = _pockets()
    jobs = _jobs(pockets, 4)
    reqs = [(jobs[0], 120, 50), (jobs[1], 75, 30), (jobs[2], 50, 50), (jobs[3], 0, 0)]
    got, st = _serve(pockets, enepara, reqs, stagger_s=0.01)
    for (job, steps, spx), r in zip(reqs, got):
        assert r["status"] == 0 and r["steps"] == steps
        rep, stats = _ensemble_result(pockets, job, enepara, steps, spx)
        assert r["replicas"].tobytes() == rep.tobytes()
        assert np.array_equal(r["stats"], stats)
    assert st["completed"] == 4 and st["failed"] == 0 and st["outstanding"] == 0
    nrep = [j.nlig * j.ntmp * pockets[j.pocket].nconf for j in jobs]
    assert st["pose_evals"] == sum(n * (s + 1) for n, (_, s, _) in zip(nrep, reqs))


def test_same_alone_and_in_mix(lib, enepara):
    """A request gives the same bytes whether it runs alone or among requests
    that arrive before and while it runs (different sizes, pockets, step counts)."""
    pockets = _pockets()
    jobs = _jobs(pockets, 7, seed=8)
    probe = (jobs[3], 100, 25)
    alone, _ = _serve(pockets, enepara, [probe])
    mix_reqs = [(jobs[0], 150, 50), (jobs[1], 60, 20), probe, (jobs[2], 200, 50), (jobs[4], 30, 0),
                (jobs[5], 80, 40), (jobs[6], 100, 25)]
    mixed, st = _serve(pockets, enepara, mix_reqs, stagger_s=0.005, max_active_replicas=64)
    assert alone[0]["replicas"].tobytes() == mixed[2]["replicas"].tobytes()
    assert np.array_equal(alone[0]["stats"], mixed[2]["stats"])
    assert all(r["status"] == 0 for r in mixed)
    assert st["rounds"] >= 4


def test_admission_respects_budget(lib, enepara):
    """With room for one job at a time, each request is admitted only after the
    previous one finished, in submission order."""
    pockets = _pockets()
    jobs = [j for j in _jobs(pockets, 6, seed=11) if j.pocket == 1][:3]
    one = 400_000   # bytes: one of these jobs (about 280 kB each, mostly the psp gather) but not two
    got, st = _serve(pockets, enepara, [(j, 60, 30) for j in jobs], hbm_budget_bytes=one)
    for a, b in zip(got, got[1:]):
        assert b["t_admit"] >= a["t_done"] - 1e-3
    assert st["peak_bytes"] <= one


def test_bad_requests_refused(lib, enepara):
    pockets = _pockets()
    job = _jobs(pockets, 1)[0]
    with dock.Server(pockets, enepara, max_atoms=40, max_replicas_per_job=32) as srv:
        big = _jobs(pockets, 3)[2]          # 80 atoms
        with pytest.raises(GdockError) as ei:
            srv.submit(big, 10)
        assert ei.value.code == GD_E_CAPACITY
        job.pocket = 5
        with pytest.raises(GdockError) as ei:
            srv.submit(job, 10)
        assert ei.value.code == GD_E_INVALID
        job.pocket = 0
        with pytest.raises(GdockError) as ei:
            srv.submit(job, -1)
        assert ei.value.code == GD_E_INVALID
        t = srv.submit(job, 10, 5)
        srv.drain(60_000)
        (r,) = srv.poll(4, 0)
        assert r["ticket"] == t and r["status"] == 0


def test_cancel_queued_and_running(lib, enepara):
    """gd_server_cancel: a queued request is reported at once, a running one at
    the next round boundary, both with GD_E_CANCELLED; the server keeps serving
    and a later request's result equals its ensemble result."""
    from geauxdock_b200._lib import GD_E_CANCELLED, GD_E_STATE

    pockets = _pockets()
    jobs = _jobs(pockets, 3)
    # jobs 0 and 2 have 16 replicas (pocket 0), job 1 has 24 (pocket 1): with a
    # cap of 24 replicas per round the second request waits while the first runs
    with dock.Server(pockets, enepara, max_active_replicas=24) as srv:
        t_run = srv.submit(jobs[0], 200_000, 50)
        t_queued = srv.submit(jobs[2], 50, 50)
        srv.cancel(t_queued)
        t0 = time.time()
        while srv.stats()["rounds"] < 3 and time.time() - t0 < 60:
            time.sleep(0.01)
        srv.cancel(t_run)
        srv.drain(60_000)
        res = {r["ticket"]: r for r in srv.poll(8, 0)}
        assert res[t_queued]["status"] == GD_E_CANCELLED and res[t_queued]["steps"] == 0
        assert res[t_run]["status"] == GD_E_CANCELLED and 0 < res[t_run]["steps"] < 200_000
        with pytest.raises(GdockError) as ei:
            srv.cancel(t_run)                    # already reported
        assert ei.value.code == GD_E_STATE
        with pytest.raises(GdockError) as ei:
            srv.cancel(10_000)                   # never issued
        assert ei.value.code == GD_E_INVALID
        t_ok = srv.submit(jobs[1], 75, 30)
        srv.drain(60_000)
        (r,) = srv.poll(4, 0)
        st = srv.stats()
    assert r["ticket"] == t_ok and r["status"] == 0
    want, want_st = _ensemble_result(pockets, jobs[1], enepara, 75, 30)
    for f in want.dtype.names:
        assert r["replicas"][f].tobytes() == want[f].tobytes(), f
    assert st["completed"] == 1 and st["failed"] == 2 and st["outstanding"] == 0


def test_injected_allocation_failure(lib, enepara):
    """An allocation failure while admitting a request (injected on the host by
    the fail_alloc hook, as a failed cudaMalloc reports it) fails that request
    with GD_E_NOMEM; the other requests and the server carry on."""
    from geauxdock_b200._lib import GD_E_NOMEM, check

    pockets = _pockets()
    jobs = _jobs(pockets, 3)
    with dock.Server(pockets, enepara) as srv:
        check(lib.gd_set_option(b"fail_alloc", 1))
        try:
            t1 = srv.submit(jobs[0], 50, 50)
            srv.drain(60_000)
        finally:
            left = lib.gd_get_option(b"fail_alloc")
            check(lib.gd_set_option(b"fail_alloc", 0))
        assert left == 0
        t2 = srv.submit(jobs[1], 50, 50)
        t3 = srv.submit(jobs[2], 40, 20)
        srv.drain(60_000)
        res = {r["ticket"]: r for r in srv.poll(8, 0)}
        st = srv.stats()
    assert res[t1]["status"] == GD_E_NOMEM
    assert res[t2]["status"] == 0 and res[t3]["status"] == 0
    assert st["failed"] == 1 and st["completed"] == 2 and st["used_bytes"] == 0


def test_latency_mode_same_alone_and_in_mix(lib, enepara):
    """A server in latency mode (4 warps per replica): each request's result is
    the same, bit for bit, alone and in a mix of requests that arrive while it
    runs, and within the parity tolerance of the one-warp ensemble path."""
    pockets = _pockets()
    jobs = _jobs(pockets, 4, seed=9)
    reqs = [(jobs[0], 100, 25), (jobs[1], 60, 20), (jobs[2], 80, 40), (jobs[3], 50, 50)]
    alone = [_serve(pockets, enepara, [r], replica_warps=4)[0][0] for r in reqs[:2]]
    mix, st = _serve(pockets, enepara, reqs, stagger_s=0.005, replica_warps=4)
    for a, b in zip(alone, mix[:2]):
        assert a["status"] == 0 and b["status"] == 0
        for f in a["replicas"].dtype.names:
            assert a["replicas"][f].tobytes() == b["replicas"][f].tobytes(), f
    from oracle import tolerance as TOL

    job, steps, spx = reqs[0]
    want, _ = _ensemble_result(pockets, job, enepara, steps, spx)
    got = mix[0]["replicas"]
    same = np.all(got["movematrix"] == want["movematrix"], axis=1)
    assert same.mean() >= 0.9
    assert np.all(TOL.scaled_error(got["energy"][same], want["energy"][same]) <= 1.0)


def test_adaptive_latency_mode(lib, enepara):
    """replica_warps = -4: a round runs on 4 warps per replica when one wave of
    that split holds its replicas, else on 2 when one wave of that does, else on
    one.  A small request gives the bytes of the fixed 4-warp server; a request
    with more replicas than a 2-warp wave holds (about two thousand on a B200)
    gives the bytes of the one-warp server."""
    pockets = _pockets()
    jobs = _jobs(pockets, 4, seed=9)
    small = (jobs[0], 100, 25)
    fixed, _ = _serve(pockets, enepara, [small], replica_warps=4)
    adapt, st = _serve(pockets, enepara, [small], replica_warps=-4)
    assert st["latency_rounds"] == st["rounds"] > 0
    for f in fixed[0]["replicas"].dtype.names:
        assert fixed[0]["replicas"][f].tobytes() == adapt[0]["replicas"][f].tobytes(), f
    rng = np.random.default_rng(77)
    big_job = synth.make_job(rng, pockets[1], 30, 48, 150, 5, synth.ladder(32, 0.3, 3.0), seed=501, pocket_index=1)
    big = (big_job, 40, 20)                       # 48 x 3 x 32 = 4608 replicas
    one, _ = _serve(pockets, enepara, [big], max_replicas_per_job=8192, max_jobs=4)
    adapt2, st2 = _serve(pockets, enepara, [big], replica_warps=-4, max_replicas_per_job=8192, max_jobs=4)
    assert st2["completed"] == 1 and st2["latency_rounds"] == 0 < st2["rounds"]
    for f in one[0]["replicas"].dtype.names:
        assert one[0]["replicas"][f].tobytes() == adapt2[0]["replicas"][f].tobytes(), f
