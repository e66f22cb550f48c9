#!/usr/bin/env python
"""MC pose-evals/s of the B200 docking backend on the replica-ensemble workload.

Workload (one rank = one GPU): one synthetic complex with a 40-atom ligand in
20 conformations, 11 protein conformations of 1500 points, 400 KDE points,
16 MCS templates and 16 temperatures 0.3..3.0 -- 3520 replicas -- with a
replica-exchange sweep every 50 MC steps.  One bench step = one exchange
interval: 50 MC steps of all 3520 replicas plus the exchange sweep.

value      pose-evals/s over all ranks, device time (CUDA events on the
           library's stream), inputs resident in HBM, L2 flushed between steps
e2e        the same metric through the drop-in C ABI with host buffers
           (SetParaT + CopyH2D + Dock of steps_total = 200, Record copies back)
roofline   the batched Monte Carlo kernel against the measured FP32 FMA peak, and
           its special-function (MUFU) pipe use against the nominal MUFU rate
plain      the plain kernel (the reference's launch structure) on the same work:
           all replicas in one launch, and one launch per replica (the plain
           method's unit of work) on a sample of the replicas
cpu_baseline  the reference's own CPU Monte Carlo (built from its sources) on
           the box's host cores, a bounded sample of the same workload
screening  512 ligands of 12-64 atoms (204,800 replicas) in one persistent
           launch per exchange interval, against one plain launch per ligand
serving    the request loop under Poisson arrivals at 200 req/s and at 70 % of
           capacity: throughput, p50/p99 latency, against the plain kernel run
           one request at a time (a bounded sample of the 10,000-request stream)

--workload ensemble|screening|serving runs one leg.  --impl reference runs the
reference's CPU implementation instead (rank 0).
Multi-GPU (torchrun): the headline is weak scaling -- each rank docks its own
complex of the headline shape (independent objects, no data-path collective),
timing the max over ranks.  The "partition" leg then splits ONE complex's
replicas across the ranks with the library's own split (gd_replica_range, cut
at protein-conformation blocks) and gathers every final replica on rank 0 over
NCCL: strong scaling of the product's multi-GPU path, with the gather timed.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MC pose-evals/s batched+served vs plain kernel on 1 B200; p50/p99 dock latency"
UNIT = "pose-evals/s"
STEPS_PER_INTERVAL = 50
# DRAM bytes (read + write) of one Monte Carlo launch of this workload (3520
# replicas x 50 steps, tile 8 x kpl 4 x ab 8, pocket read through L1): a RECORDED
# constant, not measured by this script.  From one capture on a B200 of the kernel
# of commit ecc5177 (profiles/mc_kernel_ensemble3520_traffic.md):
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum
#       --clock-control none -k regex:mc_kernel -s 4 -c 1
#       python bench.py --steps 3 --warmup 3 --workload ensemble --skip-extras --tile 8,4,8,0
# (1,742,848 B read + 75,008 B written); it does not grow with the steps per launch.
TRAFFIC_BYTES_PER_LAUNCH = 1_742_848 + 75_008
# L2 sectors of the small-case ncu --set full capture of the same kernel (3520 replicas x 4 steps,
# profiles/mc_kernel_ensemble3520_small_full.md): 32 B each, per pose-eval
L2_BYTES_PER_POSE_EVAL = 14_684_063 * 32 / (3520 * 4)
TRAFFIC_SOURCE = ("recorded constant: ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                  "kernel of commit ecc5177, profiles/mc_kernel_ensemble3520_traffic.md")


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous shard [b, e) of n units for rank (the reference's maximising-balance split)."""
    per = -(-n // world)
    b = min(per * rank, n)
    return b, min(b + per, n)


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--mc-steps", type=int, default=STEPS_PER_INTERVAL,
                   help="MC steps per bench step (= steps between exchange sweeps)")
    p.add_argument("--tile", default="", help="warps,kpl,ab[,stage]: fixed tile shape (skips the autotuner)")
    p.add_argument("--skip-extras", action="store_true",
                   help="only the timed batched kernel (for profiling): no plain kernel, e2e, CPU baseline, "
                        "screening or serving legs")
    p.add_argument("--workload", choices=["all", "ensemble", "screening", "serving", "single"], default="all",
                   help="ensemble: the headline line only; screening / serving / single: that leg alone")
    p.add_argument("--single-steps", type=int, default=3000, help="MC steps of the single-replica leg")
    p.add_argument("--screen-ligands", type=int, default=512)
    p.add_argument("--screen-intervals", type=int, default=2)
    p.add_argument("--plain-ligands", type=int, default=48,
                   help="ligands of the screening set timed with the plain one-launch-per-ligand kernel")
    p.add_argument("--plain-replicas", type=int, default=16,
                   help="replicas of the ensemble timed with the plain kernel, one launch per replica")
    p.add_argument("--serve-requests", type=int, default=48,
                   help="requests of the run at the named arrival rate (which also measures the capacity)")
    p.add_argument("--serve-loads", default="0.7",
                   help="comma-separated fractions of the measured capacity to run below-capacity streams at")
    p.add_argument("--serve-load-requests", type=int, default=24, help="requests of each below-capacity stream")
    p.add_argument("--serve-rate", type=float, default=200.0, help="Poisson arrival rate, requests/s")
    p.add_argument("--serve-steps", type=int, default=2000)
    p.add_argument("--serve-max-active", type=int, default=0,
                   help="replicas per serving round (0: the server's default, four waves of resident replicas)")
    p.add_argument("--serve-round", type=int, default=STEPS_PER_INTERVAL, help="MC steps per serving round")
    p.add_argument("--serve-replica-warps", type=int, default=1,
                   help="warps per replica in the server (2, 4, 8: latency mode)")
    p.add_argument("--partition-intervals", type=int, default=5,
                   help="exchange intervals timed in the multi-GPU partition leg (one complex split across ranks)")
    return p.parse_args()


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def wait_first_sample(self, timeout_s: float = 3.0) -> None:
        """Block until nvidia-smi has written its first sample, so that its
        start-up (NVML initialisation) is over before the timed region begins."""
        t0 = time.perf_counter()
        while self.p is not None and self.p.poll() is None and time.perf_counter() - t0 < timeout_s:
            if os.path.getsize(self.f.name) > 0:
                return
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait(timeout=10)
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        load = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _workload(rank: int):
    from geauxdock_b200 import params, synth

    ep = params.optimize_enepara(params.default_enepara0())
    pk, job = synth.config2(seed=1 + rank)
    return ep, pk, job


def _config(n_rep: int, world: int, extra: dict | None = None) -> dict:
    c = {"workload": "replica ensemble: 1 complex, ligand 40 atoms x 20 conformations, pocket 1500 points x 11 "
                     "conformations, 400 KDE points, 16 MCS templates, 16 temperatures 0.3-3.0, exchange every "
                     f"{STEPS_PER_INTERVAL} steps",
         "replicas_per_gpu": n_rep, "mc_steps_per_bench_step": STEPS_PER_INTERVAL,
         "parallelism": f"one complex per GPU x{world} (independent objects, no data-path collective)",
         "l2": "flushed between timed steps (256 MiB write)"}
    if extra:
        c.update(extra)
    return c


def _cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), for the CPU baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


REF_BUILD = "g++ -O3 -fopenmp (the reference's Intel #pragma simd hints are ignored by g++)"


def cpu_reference_sample(cx, seconds: float) -> dict:
    """The reference's own CPU Monte Carlo (MonteCarlo_d, OpenMP over replicas) on
    all replicas of the complex for a number of steps sized to ~`seconds`."""
    os.environ.setdefault("OMP_PROC_BIND", "true")
    from geauxdock_b200 import layout as Lo
    from oracle import oracle as O

    if not O.have_ref():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libgdref.so was not built (reference sources absent)"}
    ref = O.ref()
    cores = os.cpu_count() or 1
    ref.gdref_set_threads(cores)
    work = cx.copy()
    n = int(work[0]["size"]["n_rep"])
    rec = Lo.aligned_zeros(Lo.RECORD, n)
    ref.gdref_montecarlo(work.ctypes.data, rec.ctypes.data, 0, 1)     # initial energies
    t0 = time.perf_counter()
    ref.gdref_montecarlo(work.ctypes.data, rec.ctypes.data, 0, 2)     # calibration: 2 steps
    t2 = time.perf_counter() - t0
    steps = int(max(2, min(200, round(seconds / max(t2 / 2, 1e-6)))))
    t0 = time.perf_counter()
    ref.gdref_montecarlo(work.ctypes.data, rec.ctypes.data, 2, steps)
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": UNIT, "cores": cores, "kind": "reference",
            "cpu_model": _cpu_model(), "build": REF_BUILD,
            "sample": f"{n} replicas x {steps} MC steps of the same complex, reference MonteCarlo_d "
                      f"(g++ -O3 -fopenmp, OMP_NUM_THREADS={cores}), {dt:.1f} s"}


def run_reference(args) -> None:
    """The reference's own CPU Monte Carlo on the headline workload.  This
    process never loads libgdock.so: the parameter tables come from the
    reference's OptimizeEnepara, the Complex from the numpy generator, and the
    line lists the in-tree libraries the process mapped."""
    rank, world, local = _dist()
    if rank != 0:
        return
    os.environ.setdefault("OMP_PROC_BIND", "true")
    from geauxdock_b200 import layout as Lo, params, synth
    from oracle import oracle as O

    if not O.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libgdref.so not built: the reference "
                                                              "sources were absent when build() ran"}))
        return
    ep = O.ref_optimize_enepara(params.default_enepara0())
    pk, job = synth.config2(seed=1)
    cx = synth.to_complex(job, pk, ep, steps_per_exchange=STEPS_PER_INTERVAL)
    n = int(cx[0]["size"]["n_rep"])
    ref = O.ref()
    cores = os.cpu_count() or 1
    ref.gdref_set_threads(cores)
    rec = Lo.aligned_zeros(Lo.RECORD, n)
    ref.gdref_montecarlo(cx.ctypes.data, rec.ctypes.data, 0, 1)
    per_step = 2            # MC steps of all replicas per bench step (a bounded sample)
    s = 0
    for _ in range(args.warmup):
        ref.gdref_montecarlo(cx.ctypes.data, rec.ctypes.data, s, per_step)
        s += per_step
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.gdref_montecarlo(cx.ctypes.data, rec.ctypes.data, s, per_step)
        s += per_step
    dt = time.perf_counter() - t0
    value = n * per_step * args.steps / dt
    sample = (f"{n} replicas x {per_step} MC steps per bench step, reference MonteCarlo_d built from its sources "
              f"(g++ -O3 -fopenmp, OMP_NUM_THREADS={cores})")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, Astex-like shapes)",
        "config": _config(n, world), "impl": "reference", "sample": sample,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample,
                         "cpu_model": _cpu_model(), "build": REF_BUILD},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "libraries_loaded": O.mapped_libraries(ROOT)}))


def _hbm_share(launch_ms: float) -> dict:
    """HBM bandwidth the Monte Carlo launch uses against the measured copy peak."""
    peak = None
    try:
        peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    gbs = TRAFFIC_BYTES_PER_LAUNCH / (launch_ms / 1e3) / 1e9
    return {"achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak if peak else None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured copy)" if peak else "unavailable"}


def _l2_rate(pose_evals_per_s: float) -> dict:
    """L2 bandwidth the batched kernel moves at this run's rate, from the recorded
    per-pose-eval L2 sectors of its small-case capture (no measured L2 peak exists
    to divide by)."""
    return {"achieved_gbs": L2_BYTES_PER_POSE_EVAL * pose_evals_per_s / 1e9,
            "source": "recorded constant: lts__t_sectors.sum x 32 B of the small-case capture per pose-eval "
                      "(profiles/mc_kernel_ensemble3520_small_full.md) x this run's pose-evals/s"}


def _mufu_share(natom: int, npoint: int, pose_evals_per_s: float, sm_mhz) -> dict:
    """Special-function (MUFU) pipe use of the Monte Carlo launch: the pair loop's
    4 MUFU ops per ligand atom x padded pocket point (rsqrt, rcp for Lennard-Jones,
    ex2 and rcp for the pmf sigmoid) against 16 per clock per SM x 148 SMs at the
    SM clock sampled during the timed region."""
    ppad = -(-npoint // 128) * 128
    ops = 4 * natom * ppad
    if not sm_mhz:
        return {"ops_per_pose_eval": ops, "frac": None}
    achieved = ops * pose_evals_per_s / 1e9
    peak = 16 * 148 * sm_mhz / 1e3
    return {"ops_per_pose_eval": ops, "achieved_gops": achieved, "peak_gops": peak, "frac": achieved / peak,
            "peak_source": "nominal 16 MUFU results per clock per SM x 148 SMs x sampled SM clock",
            "count": "pair loop only (4 per ligand atom x padded point); the sparse H-bond ex2 and KDE are extra"}


def _pct(x, q):
    import numpy as np

    return float(np.percentile(np.asarray(x, dtype=np.float64), q)) if len(x) else None


def run_single(args, local: int) -> dict:
    """The plain method's single complex: one 24-atom ligand, one 600-point
    pocket, 200 KDE points, 8 MCS templates, one temperature, ONE replica,
    3000 MC steps -- a latency workload (one replica is one warp of the batched
    kernel, one CTA of the plain kernel).  Device time of the 3000 steps
    (CUDA events), and the reference's own CPU Monte Carlo on the same replica
    (a bounded sample of the steps; one replica occupies one thread)."""
    import torch

    from geauxdock_b200 import dock, layout as Lo, params, synth
    from geauxdock_b200._lib import check, load

    lib = load()
    ep = params.optimize_enepara(params.default_enepara0())
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, ep, steps_total=args.single_steps, steps_per_dump=200)
    out = {"workload": "1 complex: ligand 24 atoms, pocket 600 points, 200 KDE points, 8 MCS templates, "
                       f"1 temperature, 1 replica, {args.single_steps} MC steps"}
    # batched kernel with the replica on 1, 2, 4, 8 warps (latency mode), and the plain kernel
    for name, kern, g in (("batched", 0, 1), ("batched_2_warps", 0, 2), ("batched_4_warps", 0, 4),
                          ("batched_8_warps", 0, 8), ("plain", 1, 1)):
        check(lib.gd_set_option(b"kernel", kern))
        check(lib.gd_set_option(b"replica_warps", g))
        try:
            with dock.Ensemble.from_complexes([cx], [1]) as ens:
                ens.init()
                ens.run(200)                 # warm-up
                ens.sync()
                st = torch.cuda.ExternalStream(lib.gd_ensemble_stream(ens.h), device=torch.device("cuda", local))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
                ens.run(args.single_steps)
                b.record(st)
                b.synchronize()
                ens.sync()
                ms = a.elapsed_time(b)
        finally:
            check(lib.gd_set_option(b"kernel", 0))
            check(lib.gd_set_option(b"replica_warps", 1))
        out[name] = {"value": args.single_steps / (ms / 1e3), "unit": UNIT, "ms": ms}
    from oracle import oracle as O

    if O.have_ref():
        ref = O.ref()
        ref.gdref_set_threads(1)
        work = cx.copy()
        rec = Lo.aligned_zeros(Lo.RECORD, 1)
        ref.gdref_montecarlo(work.ctypes.data, rec.ctypes.data, 0, 1)
        n = 200
        t0 = time.perf_counter()
        ref.gdref_montecarlo(work.ctypes.data, rec.ctypes.data, 0, n)
        dt = time.perf_counter() - t0
        ref.gdref_set_threads(os.cpu_count() or 1)
        out["cpu_reference"] = {"value": n / dt, "unit": UNIT, "cores": 1, "kind": "reference",
                                "sample": f"{n} of the {args.single_steps} MC steps, reference MonteCarlo_d"}
        out["speedup_batched_over_cpu"] = out["batched"]["value"] / out["cpu_reference"]["value"]
        out["speedup_batched_8_warps_over_cpu"] = out["batched_8_warps"]["value"] / out["cpu_reference"]["value"]
    return out


def run_screening(args, local: int) -> dict:
    """Batched uneven screening: ligands of U[12, 64] atoms x 10 conformations x
    5 protein conformations x 8 temperatures against one 2000-point pocket, all
    ligands in one persistent launch per exchange interval (replayed from a CUDA
    graph), against the plain kernel launched once per ligand."""
    import torch

    from geauxdock_b200 import dock, params, synth
    from geauxdock_b200._lib import check, load

    lib = load()
    ep = params.optimize_enepara(params.default_enepara0())
    pk, jobs = synth.config3(seed=1, nligand=args.screen_ligands)
    n_rep = sum(j.nlig * j.ntmp * pk.nconf for j in jobs)
    spi = STEPS_PER_INTERVAL
    check(lib.gd_set_option(b"kernel", 0))
    t0 = time.perf_counter()
    ens = dock.Ensemble.from_jobs([pk], jobs, ep, device=local)
    pack_s = time.perf_counter() - t0
    ens.init()
    ens.sync()
    tune = "" if args.no_autotune else ens.autotune(spi)
    ens.run(spi, spi)                    # warm-up: captures the interval graph
    ens.sync()
    stream = torch.cuda.ExternalStream(lib.gd_ensemble_stream(ens.h), device=torch.device("cuda", local))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.screen_intervals):
        ens.run(spi, spi)
    b.record(stream)
    b.synchronize()
    _, mc_launches, all_launches = ens.sync(all_launches=True)
    batched = n_rep * spi * args.screen_intervals / (a.elapsed_time(b) / 1e3)
    ens.close()

    # plain kernel, one launch per ligand per interval, on the first ligands
    sub = jobs[:args.plain_ligands]
    n_sub = sum(j.nlig * j.ntmp * pk.nconf for j in sub)
    check(lib.gd_set_option(b"kernel", 1))
    plain = dock.Ensemble.from_jobs([pk], sub, ep, device=local)
    plain.init()
    plain.run(spi, spi)
    plain.sync()
    pstream = torch.cuda.ExternalStream(lib.gd_ensemble_stream(plain.h), device=torch.device("cuda", local))
    a.record(pstream)
    plain.run(spi, spi)
    b.record(pstream)
    b.synchronize()
    _, plain_launches = plain.sync()
    plain_value = n_sub * spi / (a.elapsed_time(b) / 1e3)
    plain.close()
    check(lib.gd_set_option(b"kernel", 0))
    return {"workload": f"{args.screen_ligands} ligands of U[12,64] atoms x 10 conformations, 1 pocket of 2000 "
                        "points x 5 conformations, 600 KDE points, 16 MCS templates, 8 temperatures 0.3-3.0",
            "replicas": n_rep, "value": batched, "unit": UNIT,
            "timed": f"{args.screen_intervals} exchange intervals of {spi} MC steps (device time)",
            "launches": {"mc": mc_launches, "all": all_launches}, "pack_s": pack_s,
            "autotune": tune.strip().splitlines()[-1] if tune else "off",
            "plain_one_launch_per_ligand": {"value": plain_value, "unit": UNIT, "ligands": len(sub),
                                            "launches": plain_launches},
            "speedup_over_plain": batched / plain_value}


def run_partition(args, cx, world: int, rank: int, local: int, seed: int) -> dict | None:
    """One Complex sharded across the ranks (the product's multi-GPU path):
    each rank runs its replica range (gd_replica_range, SetParaT's split cut at
    protein-conformation blocks: exchange partners stay on one rank) with one
    seed on every rank, then rank 0 gathers every final replica state over NCCL
    (shard.gather_replicas).  Strong scaling: the complex's replicas are fixed,
    the ranks split them.  Device time of the Monte Carlo intervals, max over
    ranks; the gather timed separately on the host."""
    import ctypes as C

    import torch
    import torch.distributed as dist

    from geauxdock_b200 import dock, shard
    from geauxdock_b200._lib import check, load

    lib = load()
    b, e = shard.replica_range(cx, world, rank)
    h = C.c_void_p()
    check(lib.gd_ensemble_create_complex_range(C.c_void_p(cx.ctypes.data), b, e - 1, seed, local, C.byref(h)))
    spi = STEPS_PER_INTERVAL
    with dock.Ensemble(h, 1) as ens:
        ens.init()
        ens.run(spi, spi)                 # warm-up: captures the interval graph
        ens.sync()
        stream = torch.cuda.ExternalStream(lib.gd_ensemble_stream(ens.h), device=torch.device("cuda", local))
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.partition_intervals):
            ens.run(spi, spi)
        e1.record(stream)
        e1.synchronize()
        ens.sync()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        reps = ens.replicas(0)
    dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    allr = shard.gather_replicas(reps, device=f"cuda:{local}")
    gather_ms = 1e3 * (time.perf_counter() - t0)
    sizes = [None] * world
    dist.all_gather_object(sizes, e - b)
    if rank != 0:
        return None
    n = int(cx[0]["size"]["n_rep"])
    assert allr is not None and len(allr) == n
    ms = float(t.item())
    return {"workload": "the headline complex's replicas split across the ranks (gd_replica_range), one seed",
            "scaling": "strong", "replicas": n, "replicas_per_rank": sizes,
            "value": n * spi * args.partition_intervals / (ms / 1e3), "unit": UNIT,
            "ms_per_interval": ms / args.partition_intervals, "intervals": args.partition_intervals,
            "gather": {"ms": gather_ms, "bytes": int(allr.nbytes), "how": "shard.gather_replicas, NCCL all-gather"}}


def pe_n(job, pockets) -> int:
    return job.nlig * job.ntmp * pockets[job.pocket].nconf


def run_serving(args, local: int) -> dict:
    """Serving: Poisson arrivals of docking requests (ligands log-uniform in
    [8, 80] atoms, 10 x 5 x 8 replicas, 2000 MC steps) against 4 resident
    pockets of 800, 1500, 2200 and 3000 points, admitted by a 100 GB HBM
    budget.  Latency = completion - submission on the server's clock."""
    import numpy as np

    from geauxdock_b200 import dock, params, synth
    from geauxdock_b200._lib import check, load

    lib = load()
    check(lib.gd_set_option(b"kernel", 0))
    ep = params.optimize_enepara(params.default_enepara0())
    pockets = synth.serving_pockets(seed=1)
    rng = np.random.default_rng(7)
    n = args.serve_requests
    loads = [float(x) for x in args.serve_loads.split(",") if x.strip()]
    m = args.serve_load_requests
    jobs = [synth.serving_job(rng, pockets, seed=50_000 + i) for i in range(n + m * len(loads) + 2)]
    steps = args.serve_steps

    def stream(srv, batch, rate, seed):
        arr = np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, len(batch)))
        t0 = time.perf_counter()
        for j, t in zip(batch, arr):
            d = t0 + t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            srv.submit(j, steps, STEPS_PER_INTERVAL, results=False)
        srv.drain(900_000)
        res = srv.poll(len(batch), 0)
        assert len(res) == len(batch) and all(r["status"] == 0 for r in res), res[:2]
        lat = [r["t_done"] - r["t_submit"] for r in res]
        span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
        evals = sum(r["nrep"] * (r["steps"] + 1) for r in res)
        return {"rate_req_s": rate, "requests": len(batch), "p50_s": _pct(lat, 50), "p99_s": _pct(lat, 99),
                "mean_queue_s": float(np.mean([r["t_admit"] - r["t_submit"] for r in res])),
                "value": evals / span, "unit": UNIT, "req_per_s": len(batch) / span, "span_s": span}

    with dock.Server(pockets, ep, device=local, max_atoms=80, max_active_replicas=args.serve_max_active,
                     steps_per_round=args.serve_round, replica_warps=args.serve_replica_warps) as srv:
        srv.submit(jobs[-1], 100, STEPS_PER_INTERVAL, results=False)   # warm-up
        srv.submit(jobs[-2], 100, STEPS_PER_INTERVAL, results=False)
        srv.drain(900_000)
        srv.poll(4, 0)
        s0 = srv.stats()
        named = stream(srv, jobs[:n], args.serve_rate, 11)
        s1 = srv.stats()
        named["offered_over_capacity"] = args.serve_rate / named["req_per_s"]
        # below capacity: fractions of the request rate the saturated run sustained
        below = []
        for k, f in enumerate(loads):
            sa = srv.stats()
            b = stream(srv, jobs[n + k * m:n + (k + 1) * m], f * named["req_per_s"], 12 + k)
            sb = srv.stats()
            b["load"] = f
            b["gpu_busy_frac"] = (sb["device_ms"] - sa["device_ms"]) / 1e3 / b["span_s"]
            below.append(b)
        s2 = srv.stats()
    # plain kernel, one request at a time (one launch per request per interval), a few requests
    import torch

    check(lib.gd_set_option(b"kernel", 1))
    p_evals, p_ms = 0, 0.0
    for j in jobs[:3]:
        pe = dock.Ensemble.from_jobs(pockets, [j], ep, device=local)
        pe.init()
        pe.sync()
        st_ = torch.cuda.ExternalStream(lib.gd_ensemble_stream(pe.h), device=torch.device("cuda", local))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st_)
        pe.run(4 * STEPS_PER_INTERVAL, STEPS_PER_INTERVAL)
        b.record(st_)
        b.synchronize()
        pe.sync()
        p_ms += a.elapsed_time(b)
        p_evals += pe_n(j, pockets) * 4 * STEPS_PER_INTERVAL
        pe.close()
    check(lib.gd_set_option(b"kernel", 0))
    plain = {"value": p_evals / (p_ms / 1e3), "unit": UNIT,
             "sample": f"first 3 requests one at a time, {4 * STEPS_PER_INTERVAL} MC steps each (device time)"}
    dev_s = (s1["device_ms"] - s0["device_ms"]) / 1e3
    named["gpu_busy_frac"] = dev_s / named["span_s"]
    named["note"] = (f"the named rate is {named['offered_over_capacity']:.1f}x the measured capacity: its queue, "
                     "and so its latency, grow with the stream's length; these are the figures of a "
                     f"{named['requests']}-request burst")
    return {"workload": f"Poisson arrivals, ligands log-uniform [8,80] atoms, 10x5x8 replicas, {steps} MC steps, "
                        "exchange every 50, 4 resident pockets (800/1500/2200/3000 points x 5), 100 GB HBM budget",
            "named_rate": named, "below_capacity": below, "plain_one_launch_per_request": plain,
            "speedup_over_plain": named["value"] / plain["value"],
            "server": {"warps_per_cta": s2["warps_per_cta"], "grid": s2["grid"], "pocket_staged": s2["pocket_staged"],
                       "max_active_replicas": s2["max_active_replicas"], "rounds": s2["rounds"],
                       "launches": s2["launches"], "peak_bytes": s2["peak_bytes"]},
            "sample": f"{named['requests']} + {' + '.join(str(b['requests']) for b in below)} requests (the named "
                      "stream has 10000; bounded so the bench ends in minutes)"}


def run_ours(args) -> None:
    import ctypes as C

    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if args.workload in ("screening", "serving", "single"):
        if rank == 0:
            leg = {"screening": run_screening, "serving": run_serving, "single": run_single}[args.workload](args, local)
            print(json.dumps({"metric": METRIC, "workload": args.workload, **leg}))
        return
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from geauxdock_b200 import dock, layout as Lo, synth, workmodel
    from geauxdock_b200._lib import check, load

    lib = load()
    ep, pk, job = _workload(rank)
    cx = synth.to_complex(job, pk, ep, steps_total=200, steps_per_dump=200, steps_per_exchange=STEPS_PER_INTERVAL)
    n_rep = int(cx[0]["size"]["n_rep"])
    fpp = workmodel.job_flops_per_pose(job, pk, ep)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---------------- resident ensemble, batched kernel
    check(lib.gd_set_option(b"kernel", 0))
    if args.tile:
        t = [int(x) for x in args.tile.split(",")]
        check(lib.gd_set_option(b"warps", t[0]))
        check(lib.gd_set_option(b"kpl", t[1]))
        check(lib.gd_set_option(b"ab", t[2]))
        check(lib.gd_set_option(b"stage", t[3] if len(t) > 3 else 1))
        args.no_autotune = True
    ens = dock.Ensemble.from_complexes([cx], [1000 + rank], device=local)
    ens.init()
    ens.sync()
    tune = "" if args.no_autotune else ens.autotune(args.mc_steps)
    stream = torch.cuda.ExternalStream(lib.gd_ensemble_stream(ens.h), device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    spi = args.mc_steps
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            ens.run(spi, spi)
            flush.zero_()
    ens.sync()
    barrier()
    clocks = Clocks(local)
    clocks.wait_first_sample()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            ens.run(spi, spi)
            flush.zero_()
    e1.record(stream)
    e1.synchronize()
    barrier()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    kernel_ms, mc_launches, all_launches = ens.sync(all_launches=True)
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    pose_evals = n_rep * spi * args.steps
    value = world * pose_evals / (ms_max / 1e3)
    avg_launch_ms = kernel_ms / max(mc_launches, 1)
    flops_per_launch = fpp * n_rep * spi
    peak = C.c_double()
    check(lib.gd_fp32_peak(C.byref(peak)))
    achieved = flops_per_launch / (avg_launch_ms / 1e3) / 1e12
    ens.close()
    if args.skip_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "mc_steps_per_step": spi,
                              "roofline": {"achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                                           "frac": achieved / peak.value, "avg_launch_ms": avg_launch_ms},
                              "clocks": ck, "note": "profiling run (--skip-extras)"}))
        if world > 1:
            dist.destroy_process_group()
        return

    # ---------------- plain kernel, same work
    check(lib.gd_set_option(b"kernel", 1))
    plain = dock.Ensemble.from_complexes([cx], [1000 + rank], device=local)
    plain.init()
    plain.run(STEPS_PER_INTERVAL, STEPS_PER_INTERVAL)
    plain.sync()
    p_steps = 2
    pstream = torch.cuda.ExternalStream(lib.gd_ensemble_stream(plain.h), device=torch.device("cuda", local))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(pstream)
    for _ in range(p_steps):
        plain.run(STEPS_PER_INTERVAL, STEPS_PER_INTERVAL)
    b.record(pstream)
    b.synchronize()
    plain_value = n_rep * STEPS_PER_INTERVAL * p_steps / (a.elapsed_time(b) / 1e3)
    plain.close()

    # ---------------- plain kernel, one replica per launch (the plain method's
    # unit of work: one complex, one replica), on a strided sample of replicas;
    # device time of the launches summed, as if issued back to back
    one_ms, one_launches = 0.0, 0
    sample = list(range(0, n_rep, max(1, n_rep // args.plain_replicas)))[:args.plain_replicas]
    for r in sample:
        h = C.c_void_p()
        check(lib.gd_ensemble_create_complex_range(C.c_void_p(cx.ctypes.data), r, r, 1000 + rank, local,
                                                   C.byref(h)))
        one = dock.Ensemble(h, 1)
        one.init()
        one.sync()
        one.run(STEPS_PER_INTERVAL, 0)
        ms_r, nl_r = one.sync()
        one_ms += ms_r
        one_launches += nl_r
        one.close()
    plain_one = {"value": len(sample) * STEPS_PER_INTERVAL / (one_ms / 1e3), "unit": UNIT,
                 "replicas": len(sample), "launches": one_launches,
                 "sample": f"{len(sample)} replicas of the ensemble (every {n_rep // len(sample)}th), "
                           f"{STEPS_PER_INTERVAL} MC steps each, one plain launch per replica, device time"}
    check(lib.gd_set_option(b"kernel", 0))

    # ---------------- end to end through the drop-in C ABI, pinned host buffers
    cx_pin = torch.empty(Lo.COMPLEX.itemsize, dtype=torch.uint8, pin_memory=True)
    cx_h = np.frombuffer(cx_pin.numpy(), dtype=Lo.COMPLEX, count=1)
    cx_h[0] = cx[0]
    rec_pin = torch.empty(Lo.RECORD.itemsize * n_rep, dtype=torch.uint8, pin_memory=True)
    rec_h = np.frombuffer(rec_pin.numpy(), dtype=Lo.RECORD, count=n_rep)
    e2e_calls = 5
    e2e_times = []
    check(lib.gd_set_option(b"device_base", local))   # this rank's GPU for the drop-in API
    with dock.DockSession(1, seed=77 + rank) as s:
        s.dock(cx_h, rec_h)              # warm-up: builds the kept device state
        cx_h[0] = cx[0]
        s.dock(cx_h, rec_h)              # warm-up of the refill path the timed calls take
        barrier()
        for _ in range(e2e_calls):
            cx_h[0] = cx[0]              # a fresh input Complex (host setup, outside the timed call)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.dock(cx_h, rec_h)
            torch.cuda.synchronize()
            e2e_times.append(time.perf_counter() - t0)
    e2e_steps = int(cx[0]["mcpara"]["steps_total"])
    e2e_s = sum(e2e_times)
    # device-to-host bytes of a call: the Record entries the kernels wrote straight into the
    # pinned array as the chunk ran (with their next_entry words), or, on the copy path, the
    # whole Record array; then the final replica states
    rec_direct = bool(lib.gd_get_option(b"dock_record_direct"))
    rec_bytes = (int(rec_h["next_entry"].astype(np.int64).sum()) * Lo.REPLICA.itemsize + 4 * n_rep if rec_direct
                 else Lo.RECORD.itemsize * n_rep)
    if world > 1:                        # the slowest rank's time, as for the device-timed value
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * n_rep * e2e_steps * e2e_calls / e2e_s

    # the product's multi-GPU path: one complex's replicas split across the ranks + gather
    partition = run_partition(args, cx, world, rank, local, 1000) if world > 1 else None

    screening = serving = None
    single = None
    if world == 1 and args.workload == "all":
        single = run_single(args, local)
        screening = run_screening(args, local)
        serving = run_serving(args, local)

    if rank == 0:
        cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "skipped (--no-cpu-baseline)"}
        if not args.no_cpu_baseline and world == 1:
            cpu = cpu_reference_sample(cx, args.cpu_seconds)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, Astex-like shapes)",
            "config": _config(n_rep, world),
            "autotune": tune.strip().splitlines()[-1] if tune else "off",
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": Lo.COMPLEX.itemsize,
                    "d2h_bytes_per_step": rec_bytes + Lo.REPLICA.itemsize * n_rep,
                    "step": f"one Dock call: CopyH2D + initial energies + {e2e_steps} MC steps + Records to the "
                            "pinned host array" + (" (written by the kernels as the steps run)" if rec_direct
                                                   else " (copied after the chunk)"),
                    "calls": e2e_calls, "call_ms": [round(1e3 * t, 2) for t in e2e_times],
                    "timing": "host wall clock around each call (synchronised), summed; max over ranks"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                         "frac": achieved / peak.value,
                         "traffic": TRAFFIC_BYTES_PER_LAUNCH if spi == STEPS_PER_INTERVAL else None,
                         "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                         "traffic_source": TRAFFIC_SOURCE,
                         "hbm": _hbm_share(avg_launch_ms) if spi == STEPS_PER_INTERVAL else None,
                         "l2": _l2_rate(n_rep * spi / (avg_launch_ms / 1e3)),
                         "kernel": "gd::mc_kernel (batched Monte Carlo, 50 steps x 3520 replicas per launch)",
                         "flops_per_pose_eval": fpp, "avg_launch_ms": avg_launch_ms,
                         "peak_source": "measured this run: FP32 FMA microbenchmark gd_fp32_peak (2 flops/FMA); "
                                        "MEASURED_PEAKS.json has no FP32 figure",
                         "mufu": _mufu_share(len(job.lig_type), len(pk.type), n_rep * spi / (avg_launch_ms / 1e3),
                                             ck.get("sm_mhz"))},
            "plain_kernel": {"value": plain_value, "unit": UNIT, "speedup_batched_over_plain": value / world / plain_value,
                             "launch": "all replicas in one launch (the reference's Dock launch structure)"},
            "plain_one_replica_per_launch": {**plain_one,
                                             "speedup_batched_over_plain": value / world / plain_one["value"]},
            "cpu_baseline": cpu,
            "clocks": ck,
            "gpu_launches": all_launches,
        }
        if partition is not None:
            line["partition"] = partition
        if single is not None:
            line["single_complex"] = single
        if screening is not None:
            line["screening"] = screening
            line["serving"] = serving
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
