"""GPU Monte Carlo against the FP64 oracle driven by the same Philox draws:
trajectories, Record contents of the drop-in Dock path, replica exchange, the
plain kernel, reproducibility and tile-shape independence."""

import numpy as np
import pytest

from geauxdock_b200 import dock, layout as Lo, synth
from geauxdock_b200._lib import GD_E_INVALID, GdockError, check
from oracle import tolerance as TOL

pytestmark = pytest.mark.gpu


def _small_ensemble(enepara, seed=4, L=18, P=300, nlig=3, nprt=2, temps=(0.3, 0.6, 1.2, 2.4)):
    rng = np.random.default_rng(seed)
    pk = synth.make_pocket(rng, P, nprt)
    job = synth.make_job(rng, pk, L, nlig, 120, 6, np.array(temps, np.float32), seed=seed)
    return synth.to_complex(job, pk, enepara)


def _oracle_run(O, cx, seed, steps, spx=0, record=None):
    ref = cx.copy()
    O.montecarlo(ref, record, 0, 1, seed)
    if steps:
        O.montecarlo(ref, record, 0, steps, seed, spx)
    return ref


def _close(a, b, tol=TOL.REL):
    """Energies agree within the parity tolerance (oracle/tolerance.py), with
    tol in place of its 1e-5: |a - b| <= tol * max(|b|, tau_i) per term."""
    s = TOL.scaled_error(a, b) * (TOL.REL / tol)
    assert np.all(s <= 1.0), float(s.max())


def _same_trajectory(got, want):
    """Replicas whose final pose matches the oracle exactly (the same accepted moves)."""
    return np.all(got["movematrix"] == want["movematrix"], axis=1)


def test_single_replica_trajectory(lib, enepara, oracle_lib):
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    ref = _oracle_run(oracle_lib, cx, 7, 300)
    with dock.Ensemble.from_complexes([cx], [7]) as ens:
        ens.init()
        ens.run(300)
        ens.sync()
        got = ens.replicas(0)
        st = ens.stats(0)
    want = ref[0]["replica"][:1]
    assert _same_trajectory(got, want).all()
    _close(got["energy"], want["energy"])
    assert st[0, 0] == 301 and 0 < st[0, 1] <= 301


def test_ensemble_with_exchange(lib, enepara, oracle_lib):
    cx = _small_ensemble(enepara)
    n = int(cx[0]["size"]["n_rep"])
    ref = _oracle_run(oracle_lib, cx, 3, 120, spx=20)
    with dock.Ensemble.from_complexes([cx], [3]) as ens:
        ens.init()
        ens.run(120, 20)
        ens.sync()
        got = ens.replicas(0)
        st = ens.stats(0)
    want = ref[0]["replica"][:n]
    same = _same_trajectory(got, want)
    # an acceptance decision can flip where FP32 and FP64 energies straddle the
    # threshold; after that the chain legitimately differs.  Nearly all agree:
    assert same.mean() >= 0.9, same.mean()
    _close(got["energy"][same], want["energy"][same])
    assert st[:, 2].sum() > 0, "no exchange attempted"
    assert st[:, 3].sum() > 0, "no exchange accepted"


def test_dock_drop_in_records(lib, enepara, oracle_lib):
    """Dock(): initial energy, two dump chunks, Records of the last chunk, final
    replicas copied back to the host Complex (backend_gpu.cu:63-133)."""
    cx = _small_ensemble(enepara, seed=9)
    cx[0]["mcpara"]["steps_total"] = 400
    cx[0]["mcpara"]["steps_per_dump"] = 200
    n = int(cx[0]["size"]["n_rep"])
    ref = cx.copy()
    rrec = Lo.aligned_zeros(Lo.RECORD, n)
    oracle_lib.montecarlo(ref, rrec, 0, 1, 11)
    oracle_lib.montecarlo(ref, rrec, 0, 200, 11)
    oracle_lib.montecarlo(ref, rrec, 200, 200, 11)
    work = cx.copy()
    with dock.DockSession(1, seed=11) as s:
        rec = s.dock(work)
    same = _same_trajectory(work[0]["replica"][:n], ref[0]["replica"][:n])
    assert same.mean() >= 0.9
    for r in np.nonzero(same)[0]:
        ne = int(rec[r]["next_entry"])
        assert ne == int(rrec[r]["next_entry"])
        got, want = rec[r]["replica"][:ne], rrec[r]["replica"][:ne]
        np.testing.assert_array_equal(got["step"], want["step"])
        assert np.all(got["step"] >= 200) and np.all(got["step"] < 400)
        np.testing.assert_array_equal(got["movematrix"], want["movematrix"])
        _close(got["energy"], want["energy"])
        np.testing.assert_array_equal(got["is_accept"], want["is_accept"])
    assert np.all(work[0]["replica"]["is_accept"][:n] == ref[0]["replica"]["is_accept"][:n])


def test_acceptance_and_best_energy_statistics(lib, enepara, oracle_lib):
    """Over every replica of a 96-replica ensemble (chains that diverged after a
    flipped decision included): acceptance rates and best-energy distributions
    of the GPU and the FP64 oracle agree statistically, and acceptance rises
    with temperature."""
    from scipy.stats import ks_2samp

    temps = (0.3, 0.45, 0.7, 1.0, 1.5, 2.2, 3.3, 5.0)
    cx = _small_ensemble(enepara, seed=17, nlig=4, nprt=3, temps=temps)
    cx[0]["mcpara"]["steps_total"] = 200
    cx[0]["mcpara"]["steps_per_dump"] = 200
    n = int(cx[0]["size"]["n_rep"])
    ref = cx.copy()
    rrec = Lo.aligned_zeros(Lo.RECORD, n)
    oracle_lib.montecarlo(ref, rrec, 0, 1, 23)
    oracle_lib.montecarlo(ref, rrec, 0, 200, 23)
    work = cx.copy()
    with dock.DockSession(1, seed=23) as s:
        rec = s.dock(work)

    def summary(records):
        acc = np.array([int(r["next_entry"]) for r in records], np.float64)   # accepted states + the initial one
        best = np.array([r["replica"][:int(r["next_entry"])]["energy"][:, 9].min() for r in records], np.float64)
        return acc, best

    acc_g, best_g = summary(rec[:n])
    acc_o, best_o = summary(rrec[:n])
    se = np.sqrt(acc_g.var() / n + acc_o.var() / n) + 1e-9
    assert abs(acc_g.mean() - acc_o.mean()) <= 3 * se, (acc_g.mean(), acc_o.mean(), se)
    assert ks_2samp(best_g, best_o).pvalue > 0.01
    tmp = work[0]["replica"]["idx_tmp"][:n]
    by_t = [acc_g[tmp == t].mean() for t in range(len(temps))]
    assert by_t[-1] > by_t[0], by_t


def test_dock_initial_energy_record(lib, enepara, oracle_lib):
    """With one dump chunk, Record entry 0 is the initial state at step 0 -- the
    entry the reference prints as its known-answer line (kernel_print.C:9-15)."""
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara, steps_total=200, steps_per_dump=200)
    with dock.DockSession(1, seed=5) as s:
        rec = s.dock(cx.copy())
    e, _ = oracle_lib.energy(cx, 0, 0, np.zeros(6, np.float32))
    first = rec[0]["replica"][0]
    assert first["step"] == 0 and rec[0]["next_entry"] >= 1
    TOL.check(first["energy"], e, "initial energy record")


def test_plain_kernel_matches_batched(lib, enepara):
    cx = _small_ensemble(enepara, seed=6)
    res = {}
    for kern in (0, 1):
        check(lib.gd_set_option(b"kernel", kern))
        try:
            with dock.Ensemble.from_complexes([cx], [5]) as ens:
                ens.init()
                ens.run(100, 25)
                ens.sync()
                res[kern] = ens.replicas(0)
        finally:
            check(lib.gd_set_option(b"kernel", 0))
    same = _same_trajectory(res[0], res[1])
    assert same.mean() >= 0.9
    _close(res[0]["energy"][same], res[1]["energy"][same], 2e-5)


def test_reproducible_and_tile_independent(lib, enepara):
    """Same seed -> bit-identical states, whatever the number of replicas per CTA
    and whether the protein conformation is staged in shared memory or read
    through L1."""
    cx = _small_ensemble(enepara, seed=2)
    out = []
    for warps, stage in ((0, -1), (3, 1), (7, 1), (5, 0), (0, 0)):
        check(lib.gd_set_option(b"warps", warps))
        check(lib.gd_set_option(b"stage", stage))
        try:
            with dock.Ensemble.from_complexes([cx], [21]) as ens:
                ens.init()
                ens.run(60, 15)
                ens.sync()
                out.append(ens.replicas(0))
        finally:
            check(lib.gd_set_option(b"warps", 0))
            check(lib.gd_set_option(b"stage", -1))
    for o in out[1:]:
        assert o.tobytes() == out[0].tobytes()


def test_batch_independent(lib, enepara):
    """A job's result is the same alone and batched with other jobs."""
    cxa = _small_ensemble(enepara, seed=31, L=12)
    cxb = _small_ensemble(enepara, seed=32, L=40, P=500)
    with dock.Ensemble.from_complexes([cxa], [1]) as e1:
        e1.init()
        e1.run(40, 10)
        e1.sync()
        alone = e1.replicas(0)
    with dock.Ensemble.from_complexes([cxb, cxa], [2, 1]) as e2:
        e2.init()
        e2.run(40, 10)
        e2.sync()
        mixed = e2.replicas(1)
    assert alone.tobytes() == mixed.tobytes()


def test_invalid_inputs_rejected(lib, enepara):
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    bad = cx.copy()
    bad[0]["lig"][0]["t2"][0] = 40                  # ligand type outside 0..23
    with pytest.raises(GdockError) as ei:
        dock.Ensemble.from_complexes([bad], [1])
    assert ei.value.code == GD_E_INVALID
    bad = cx.copy()
    bad[0]["mcs"][0]["x"][:] = Lo.MCS_INVALID_COORD   # an MCS row with no coordinate
    with pytest.raises(GdockError):
        dock.Ensemble.from_complexes([bad], [1])
    bad = cx.copy()
    bad[0]["enepara"]["p1a"][3, 7] = 0.0             # the FP32 pair form divides by p1a
    with pytest.raises(GdockError) as ei:
        dock.Ensemble.from_complexes([bad], [1])
    assert ei.value.code == GD_E_INVALID


def test_graph_replay_matches_launches(lib, enepara, oracle_lib):
    """Whole exchange intervals replayed from the captured graph (one exchange
    launch over every job, device step counter) leave the same bytes as
    chunk-by-chunk launches, for jobs with different ladders and a remainder
    chunk; each job still follows its own oracle chain."""
    cxs = [_small_ensemble(enepara, seed=41, L=14, temps=(0.3, 0.9, 2.7)),
           _small_ensemble(enepara, seed=42, L=30, P=420, nlig=2, temps=(0.2, 0.4, 0.8, 1.6, 3.2)),
           _small_ensemble(enepara, seed=43, L=9, nprt=1, nlig=1, temps=(1.0,))]
    seeds = [5, 6, 7]
    out = {}
    try:
        for graph in (1, 0):
            check(lib.gd_set_option(b"graph", graph))
            with dock.Ensemble.from_complexes(cxs, seeds) as ens:
                ens.init()
                ens.run(130, 20)
                ens.run(40, 20)
                _, _, nall = ens.sync(all_launches=True)
                out[graph] = [(ens.replicas(j).tobytes(), ens.stats(j).tobytes()) for j in range(3)]
                assert nall > 0
    finally:
        check(lib.gd_set_option(b"graph", 1))
    assert out[1] == out[0]
    for j, cx in enumerate(cxs):
        ref = _oracle_run(oracle_lib, cx, seeds[j], 170, spx=20)
        n = int(cx[0]["size"]["n_rep"])
        got = np.frombuffer(out[1][j][0], dtype=Lo.REPLICA)
        same = _same_trajectory(got, ref[0]["replica"][:n])
        assert same.mean() >= 0.9, (j, same.mean())


def test_dock_reuses_device_state(lib, enepara):
    """Repeated Dock calls on one set of handles (same protein and new ligand;
    new protein of the same shape; a new shape) give the same bytes whether
    the device state is kept and refilled between calls or rebuilt each call."""
    rng = np.random.default_rng(17)
    pka = synth.make_pocket(rng, 300, 2)
    pkb = synth.make_pocket(rng, 300, 2)
    temps = np.array([0.4, 1.6], np.float32)
    jobs = [synth.make_job(rng, pka, 20, 2, 100, 5, temps, seed=1),
            synth.make_job(rng, pka, 20, 2, 100, 5, temps, seed=2),
            synth.make_job(rng, pkb, 20, 2, 100, 5, temps, seed=3),
            synth.make_job(rng, pkb, 27, 3, 90, 4, temps, seed=4)]
    # call 2's pocket-specific potential is non-zero everywhere: its refill holds
    # more non-zero cells than the state was first packed with
    jobs[1].psp = np.where(jobs[1].psp == 0, np.float32(-0.25), jobs[1].psp).astype(np.float32)
    pks = [pka, pka, pkb, pkb]
    cxs = [synth.to_complex(j, p, enepara, steps_total=100, steps_per_dump=50, steps_per_exchange=25)
           for j, p in zip(jobs, pks)]
    def written(w, rec, n):
        # what a Dock call writes: the n replica states and each Record's entries
        # below next_entry (the rest of the device Record array is left as it was)
        reps = w[0]["replica"][:n]
        fields = tuple(reps[f].tobytes() for f in reps.dtype.names)
        entries = tuple(rec[r]["replica"][:int(rec[r]["next_entry"])].tobytes() for r in range(n))
        return fields, entries, rec["next_entry"][:n].tobytes()

    out = {}
    try:
        # kept state refilled on the GPU from the device Complex, refilled by the
        # host packer, and rebuilt on every call
        for mode, (cache, devpack) in {"device": (1, 1), "host": (1, 0), "rebuild": (0, 1)}.items():
            check(lib.gd_set_option(b"dock_cache", cache))
            check(lib.gd_set_option(b"dock_device_pack", devpack))
            res = []
            with dock.DockSession(1, seed=5) as s:
                for cx in cxs:
                    w = cx.copy()
                    rec = s.dock(w)
                    res.append(written(w, rec, int(cx[0]["size"]["n_rep"])))
                # calls 2 and 3 keep the shapes (new ligand; new protein of the same
                # shape) and refill the kept state; call 4 changes them
                assert s.reuse() == (4, 2 if cache else 0)
            out[mode] = res
    finally:
        check(lib.gd_set_option(b"dock_cache", 1))
        check(lib.gd_set_option(b"dock_device_pack", 1))
    for a, b, c in zip(out["device"], out["host"], out["rebuild"]):
        assert a == b == c


def test_dock_records_direct_to_pinned_host(lib, enepara):
    """With a page-locked Record array the kernels write the Records straight
    into it (option dock_record_direct): the replica states and every Record's
    entries below next_entry equal those of the copy path, and the entries past
    next_entry keep what the array held (nothing is copied over them)."""
    import torch

    rng = np.random.default_rng(23)
    pk = synth.make_pocket(rng, 300, 2)
    temps = np.array([0.3, 0.9, 2.7], np.float32)
    # one dump chunk: every entry this call writes is below next_entry (with more chunks,
    # entries an earlier chunk wrote past the last chunk's count stay, on both paths)
    cx = synth.to_complex(synth.make_job(rng, pk, 20, 2, 100, 5, temps, seed=3), pk, enepara,
                          steps_total=60, steps_per_dump=60, steps_per_exchange=20)
    n = int(cx[0]["size"]["n_rep"])

    def written(w, rec):
        reps = w[0]["replica"][:n]
        fields = tuple(reps[f].tobytes() for f in reps.dtype.names)
        entries = tuple(rec[r]["replica"][:int(rec[r]["next_entry"])].tobytes() for r in range(n))
        return fields, entries, rec["next_entry"][:n].tobytes()

    out = {}
    for mode, direct in (("copy", 0), ("direct", 1)):
        check(lib.gd_set_option(b"dock_record_direct", direct))
        try:
            buf = torch.full((Lo.RECORD.itemsize * n,), 0xAB, dtype=torch.uint8, pin_memory=True)
            rec = np.frombuffer(buf.numpy(), dtype=Lo.RECORD, count=n)
            with dock.DockSession(1, seed=9) as s:
                w = cx.copy()
                s.dock(w, rec)
                out[mode] = written(w, rec)
                ne = rec["next_entry"][:n].copy()
                assert (ne >= 1).all() and (ne <= 61).all()       # the initial state and the accepted moves
                tail = [rec[r]["replica"][int(ne[r]):].tobytes() for r in range(n)]
                untouched = all(t == b"\xab" * len(t) for t in tail)
                # the copy path overwrites the whole array with the device one
                assert untouched == bool(direct), mode
        finally:
            check(lib.gd_set_option(b"dock_record_direct", 1))
    assert out["copy"] == out["direct"]


def test_dock_device_refill_refuses_invalid(lib, enepara):
    """A Complex the device packer refuses on a refill (a ligand atom type out of
    range) fails the Dock call with GD_E_INVALID before any kernel reads it; the
    next valid call docks as a fresh session would."""
    rng = np.random.default_rng(41)
    pk = synth.make_pocket(rng, 300, 2)
    temps = np.array([0.4, 1.6], np.float32)
    cxs = [synth.to_complex(synth.make_job(rng, pk, 20, 2, 100, 5, temps, seed=s), pk, enepara, steps_total=100,
                            steps_per_dump=50) for s in (1, 2)]
    bad = cxs[1].copy()
    bad[0]["lig"][0]["t2"][3] = 40
    with dock.DockSession(1, seed=5) as s:
        s.dock(cxs[0].copy())
        with pytest.raises(GdockError) as ei:
            s.dock(bad)
        assert ei.value.code == GD_E_INVALID and "ligand atom type" in str(ei.value)
        w = cxs[1].copy()
        rec = s.dock(w)
    with dock.DockSession(1, seed=5) as s2:
        s2.dock(cxs[0].copy())
        s2.dock(cxs[0].copy())                   # same call count: the handle's seed advances per call
        w2 = cxs[1].copy()
        rec2 = s2.dock(w2)
    n = int(cxs[1][0]["size"]["n_rep"])
    for f in w[0]["replica"].dtype.names:
        assert w[0]["replica"][f][:n].tobytes() == w2[0]["replica"][f][:n].tobytes(), f
    assert rec["next_entry"][:n].tobytes() == rec2["next_entry"][:n].tobytes()


def test_sharded_run_equals_single(lib, enepara):
    """The replicas of a Complex split over 3 shards (the split ranks use), run
    one after another with one seed, equal the run of all replicas at once."""
    from geauxdock_b200 import shard

    rng = np.random.default_rng(23)
    pk = synth.make_pocket(rng, 260, 3)
    job = synth.make_job(rng, pk, 16, 2, 80, 4, synth.ladder(4, 0.3, 3.0), seed=1)
    cx = synth.to_complex(job, pk, enepara, steps_per_exchange=10)
    n = int(cx[0]["size"]["n_rep"])
    whole = shard.run_shard(cx, 60, 10, 9, 0, 1)
    parts = np.concatenate([shard.run_shard(cx, 60, 10, 9, r, 3) for r in range(3)])
    assert len(whole) == len(parts) == n
    for f in whole.dtype.names:
        assert whole[f].tobytes() == parts[f].tobytes(), f


def test_bounded_wait_reports_timeout(lib, enepara):
    """A staging barrier that never completes (the stall_test hook announces
    bytes no copy delivers) makes the kernel's bounded wait give up: the host
    gets GD_E_TIMEOUT, and the CUDA context runs the next ensemble normally."""
    from geauxdock_b200._lib import GD_E_TIMEOUT

    cx = _small_ensemble(enepara, seed=12)
    try:
        check(lib.gd_set_option(b"wait_limit", 4096))
        check(lib.gd_set_option(b"stall_test", 1))
        ens = dock.Ensemble.from_complexes([cx], [1])
        try:
            ens.init()
            with pytest.raises(GdockError) as ei:
                ens.sync()
            assert ei.value.code == GD_E_TIMEOUT
        finally:
            ens.close()
    finally:
        check(lib.gd_set_option(b"stall_test", 0))
        check(lib.gd_set_option(b"wait_limit", 0))
    with dock.Ensemble.from_complexes([cx], [1]) as ens:
        ens.init()
        ens.run(20, 10)
        ens.sync()
        assert np.isfinite(ens.replicas(0)["energy"][:int(cx[0]["size"]["n_rep"])]).all()


def test_complex_queue_matches_direct_dock(lib, enepara):
    """The multi-complex queue (one process here, a HashStore counter): each
    complex's result equals docking it alone with its derived seed, whatever
    else the same Dock handle docked before it."""
    import torch.distributed as dist

    from geauxdock_b200 import shard

    cxs = []
    for k, (L, P) in enumerate([(14, 220), (23, 310), (9, 150)]):
        rng = np.random.default_rng(40 + k)
        pk = synth.make_pocket(rng, P, 2)
        job = synth.make_job(rng, pk, L, 2, 60, 4, np.array([0.5, 1.0, 2.0], np.float32), seed=k)
        cxs.append(synth.to_complex(job, pk, enepara, steps_total=200, steps_per_dump=100))
    got = shard.dock_queue(cxs, 31, dist.HashStore())
    assert sorted(got) == [0, 1, 2]
    for i in (2, 0):
        cx = cxs[i].copy()
        with dock.DockSession(1, seed=0) as s:
            s.seed(shard.complex_seed(31, i))
            s.dock(cx)
        want = cx[0]["replica"][:int(cx[0]["size"]["n_rep"])]
        for f in want.dtype.names:                 # the fields; ReplicaMC's padding carries nothing
            assert got[i][f].tobytes() == want[f].tobytes(), (i, f)


def test_autotune_restores_state_and_runs(lib, enepara, oracle_lib):
    """The tile autotuner times candidate shapes on a snapshot of the replica
    state and restores it: the tuned ensemble then follows the oracle's
    trajectories.  FP32 candidates are the atom-pair shapes (even kpl)."""
    cx = _small_ensemble(enepara, seed=29)
    n = int(cx[0]["size"]["n_rep"])
    ref = _oracle_run(oracle_lib, cx, 8, 60)
    with dock.Ensemble.from_complexes([cx], [8]) as ens:
        ens.init()
        rep = ens.autotune(20)
        ens.run(60)
        ens.sync()
        got = ens.replicas(0)
    lines = rep.strip().splitlines()
    assert lines[-1].startswith("chosen:") and len(lines) > 2
    assert all("kpl=1 " not in l for l in lines[:-1])
    assert _same_trajectory(got, ref[0]["replica"][:n]).mean() >= 0.9


def test_empty_inputs(lib, enepara, oracle_lib):
    """Zero poses, zero steps: no error and no change.  Dock with steps_total = 0
    runs only the initial-energy step: every replica's energies are the oracle's
    for its stored pose, and no Record is written (the reference copies Records
    per dump chunk, backend_gpu.cu:63-133, and there is none)."""
    cx = _small_ensemble(enepara, seed=31)
    n = int(cx[0]["size"]["n_rep"])
    out, raw, _ = dock.eval_poses(cx, np.zeros((0, 2), np.int32), np.zeros((0, 6), np.float32))
    assert out.shape == (0, 10)
    with dock.Ensemble.from_complexes([cx], [3]) as ens:
        ens.init()
        ens.sync()
        before = ens.replicas(0).copy()
        ens.run(0)
        ens.sync()
        after = ens.replicas(0)
        for f in before.dtype.names:                # the fields; ReplicaMC's padding carries nothing
            assert after[f].tobytes() == before[f].tobytes(), f
        e0, _, _ = ens.eval_poses(0, np.zeros((0, 2), np.int32), np.zeros((0, 6), np.float32))
        assert e0.shape == (0, 10)
    work = cx.copy()
    work[0]["mcpara"]["steps_total"] = 0
    with dock.DockSession(1, seed=4) as s:
        rec = s.dock(work)
    got = work[0]["replica"][:n]
    for r in range(0, n, 7):
        want, _ = oracle_lib.energy(cx, int(got[r]["idx_lig"]), int(got[r]["idx_prt"]), cx[0]["replica"][r]["movematrix"])
        _close(got[r]["energy"], want)
        assert int(rec[r]["next_entry"]) == 0


def test_snapshot_restore_bit_identical(lib, enepara):
    """Checkpoint / resume: run(100) + snapshot, then restore into a fresh
    ensemble of the same jobs and seeds and run(100) more -- replicas and FP64
    statistics are bit-identical to an uninterrupted run(200) (exchange every
    20 steps, so the sweep index comes from the restored step counter)."""
    cx = _small_ensemble(enepara, seed=21)
    with dock.Ensemble.from_complexes([cx], [9]) as ens:
        ens.init()
        ens.run(200, 20)
        ens.sync()
        want, want_st = ens.replicas(0), ens.stats(0)
    with dock.Ensemble.from_complexes([cx], [9]) as ens:
        ens.init()
        ens.run(100, 20)
        ens.sync()
        snap = ens.snapshot()
        ens.run(60, 20)                          # diverges from the snapshot
        ens.sync()
    with dock.Ensemble.from_complexes([cx], [9]) as ens:
        ens.restore(snap)
        ens.run(100, 20)
        ens.sync()
        got, got_st = ens.replicas(0), ens.stats(0)
    for f in want.dtype.names:
        assert got[f].tobytes() == want[f].tobytes(), f
    assert got_st.tobytes() == want_st.tobytes()


def test_restore_refuses_other_seed(lib, enepara):
    cx = _small_ensemble(enepara, seed=22)
    with dock.Ensemble.from_complexes([cx], [1]) as a, dock.Ensemble.from_complexes([cx], [2]) as b:
        a.init()
        a.sync()
        snap = a.snapshot()
        with pytest.raises(GdockError) as ei:
            b.restore(snap)
        assert ei.value.code == GD_E_INVALID
        with pytest.raises(GdockError):
            b.restore(b"not a snapshot" * 4)


@pytest.mark.parametrize("g", [2, 4, 8])
def test_replica_warps_matches_oracle(lib, enepara, oracle_lib, g):
    """Latency mode: every replica split over g warps (pair rows, KDE points and
    hydrophobic sums divided, partials combined in warp order).  The chains
    follow the FP64 oracle's as the one-warp form does, and the result does not
    depend on how many replicas share a CTA (only on g)."""
    cx = _small_ensemble(enepara, seed=31, L=27, P=450)
    n = int(cx[0]["size"]["n_rep"])
    ref = _oracle_run(oracle_lib, cx, 3, 120, spx=20)
    res = {}
    try:
        check(lib.gd_set_option(b"replica_warps", g))
        for w in (g, 2 * g):
            check(lib.gd_set_option(b"warps", w))
            with dock.Ensemble.from_complexes([cx], [3]) as ens:
                ens.init()
                ens.run(120, 20)
                ens.sync()
                res[w] = ens.replicas(0)
    finally:
        check(lib.gd_set_option(b"replica_warps", 1))
        check(lib.gd_set_option(b"warps", 0))
    got, want = res[g], ref[0]["replica"][:n]
    same = _same_trajectory(got, want)
    assert same.mean() >= 0.9, same.mean()
    _close(got["energy"][same], want["energy"][same])
    for f in got.dtype.names:
        assert res[2 * g][f].tobytes() == got[f].tobytes(), f


def test_replica_warps_single_replica_trajectory(lib, enepara, oracle_lib):
    """One replica over 8 warps follows the oracle's chain for 300 steps."""
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    ref = _oracle_run(oracle_lib, cx, 7, 300)
    try:
        check(lib.gd_set_option(b"replica_warps", 8))
        with dock.Ensemble.from_complexes([cx], [7]) as ens:
            ens.init()
            ens.run(300)
            ens.sync()
            got = ens.replicas(0)
    finally:
        check(lib.gd_set_option(b"replica_warps", 1))
    want = ref[0]["replica"][:1]
    assert _same_trajectory(got, want).all()
    _close(got["energy"], want["energy"])
