"""Small cases through the bounds-checking build (run by test_gpu_check.py in
a child process with GDOCK_LIB pointing at geauxdock_b200/libgdock_check.so).

Complexes of at most 8 ligand atoms and 64 pocket points (odd atom counts,
one-point conformations, ligand types without KDE points, one-row MCS) are
evaluated and run by the batched kernel at several tile shapes (replicas per
CTA, points per lane, atoms per block, pocket staged or read through L1) and
all three precisions; every result is checked against the FP64 oracle, the
same shape at different replica groupings must give identical bytes (a race
in a reduction would not), and after every case the kernel's bounds record
must be empty.  Prints one JSON line."""

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from geauxdock_b200 import dock, params, synth  # noqa: E402
from geauxdock_b200._lib import GD_PREC_FP32, GD_PREC_FP32_KAHAN, GD_PREC_FP64, check, load  # noqa: E402
from oracle import oracle as O, tolerance as TOL  # noqa: E402

SITES = ["", "ligand pair", "pair table", "H-bond table", "pair header", "pocket point", "pocket potential",
         "KDE point", "MCS template", "type group", "MCS weight", "ligand conformation", "protein conformation",
         "replica", "temperature", "", "type table"]


def report(lib):
    import ctypes as C

    out = (C.c_int * 4)()
    check(lib.gd_check_report(out, 1))
    return list(out)


def main() -> None:
    lib = load()
    assert "check" in str(lib._name), lib._name
    ep = params.optimize_enepara(params.default_enepara0())
    rng = np.random.default_rng(5)
    shapes = [(8, 64, 12, 2, 2, 2, (0.3, 0.9, 2.7)), (7, 37, 9, 1, 1, 2, (0.5, 1.5)), (1, 1, 0, 1, 1, 1, (1.0,)),
              (5, 64, 6, 3, 3, 1, (0.4,)), (8, 63, 20, 4, 1, 3, (0.3, 0.6, 1.2, 2.4))]
    # (warps per CTA, kpl, ab, stage[, warps per replica: latency mode])
    tiles = [(1, 2, 8, 0), (3, 2, 8, 0), (3, 2, 8, 1), (2, 2, 4, 1), (4, 4, 4, 0), (2, 4, 8, 1), (2, 1, 8, 0),
             (4, 2, 8, 0, 2), (8, 2, 8, 1, 4), (8, 4, 8, 0, 8)]
    violations, worst, cases, raced = [], 0.0, 0, []
    report(lib)
    for si, (L, P, K, M, nlig, nprt, temps) in enumerate(shapes):
        pk = synth.make_pocket(rng, P, nprt)
        job = synth.make_job(rng, pk, L, nlig, K, M, np.array(temps, np.float32), seed=si + 1)
        cx = synth.to_complex(job, pk, ep)
        n = 12
        conf = np.stack([rng.integers(0, nlig, n), rng.integers(0, nprt, n)], axis=1).astype(np.int32)
        mm = synth.config4_poses(si + 3, n, radius=3.0)
        e64 = np.array([O.energy(cx, int(c[0]), int(c[1]), m)[0] for c, m in zip(conf, mm)])
        runs = {}
        for tile in tiles:
            g = tile[4] if len(tile) > 4 else 1
            for k, v in zip(("warps", "kpl", "ab", "stage", "replica_warps"), (*tile[:4], g)):
                check(lib.gd_set_option(k.encode(), v))
            for prec in (GD_PREC_FP32, GD_PREC_FP32_KAHAN, GD_PREC_FP64):
                if prec == GD_PREC_FP64 and (tile[1] != 1 or g > 1):
                    continue
                check(lib.gd_set_option(b"precision", prec))
                with dock.Ensemble.from_complexes([cx], [7]) as ens:
                    out, _, _ = ens.eval_poses(0, conf, mm, prec)
                    worst = max(worst, float(TOL.scaled_error(out, e64).max()))
                    ens.init()
                    ens.run(40, 10 if len(temps) > 1 else 0)
                    ens.sync()
                    reps = ens.replicas(0)
                cases += 1
                key = (tile[1], tile[2], prec, g)
                b = reps.tobytes()
                if key in runs and runs[key] != b:
                    raced.append({"shape": si, "tile": tile, "precision": prec})
                runs.setdefault(key, b)
                r = report(lib)
                if r[0]:
                    violations.append({"shape": si, "tile": tile, "precision": prec, "site": SITES[r[1]],
                                       "index": r[2], "length": r[3]})
    check(lib.gd_set_option(b"precision", GD_PREC_FP32_KAHAN))
    for k, v in (("warps", 0), ("kpl", 0), ("ab", 0), ("stage", -1), ("replica_warps", 1)):
        check(lib.gd_set_option(k.encode(), v))
    print(json.dumps({"cases": cases, "violations": violations, "raced": raced, "max_scaled_error": worst}))


if __name__ == "__main__":
    main()
