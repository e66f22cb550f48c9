"""Regenerate the golden fixtures of tests/golden/ (run in a container that has
the reference sources and oracle/_ref built: make -C oracle ref).

  philox_kat.txt      the Philox4x32-10 known-answer vectors of Random123
                      (src/module/Random123/examples/kat_vectors), one per line:
                      ctr0..3 key0..1 out0..3 in hex
  ref_energies_c1.npz 64 seeded poses of the synthetic single-complex config
                      (synth.config1(seed=1), poses synth.config4_poses(11, 64, 4.0)):
                      the reference's own FP32 energies (MonteCarlo_d, s2max = 1)
                      and the FP64 oracle's energies
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from geauxdock_b200 import layout as Lo, params, synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

from oracle.refpath import reference_path  # noqa: E402

REF = Path(sys.argv[1]) if len(sys.argv) > 1 else reference_path()


def philox_kat():
    lines = (REF / "src/module/Random123/examples/kat_vectors").read_text().splitlines()
    out = []
    for ln in lines:
        t = ln.split()
        if len(t) == 12 and t[0] == "philox4x32" and t[1] == "10":
            out.append(" ".join(t[2:]))
    (HERE / "philox_kat.txt").write_text("\n".join(out) + "\n")
    print("philox_kat.txt:", len(out), "vectors")


def ref_energies():
    ep = params.optimize_enepara(params.default_enepara0())
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, ep)
    mm = synth.config4_poses(11, 64, radius=4.0)
    mm[0] = 0.0
    work = cx.copy()
    c = work[0]
    c["size"]["n_rep"] = len(mm)
    for i, m in enumerate(mm):
        c["replica"][i]["movematrix"] = m
        c["replica"][i]["idx_lig"] = c["replica"][i]["idx_prt"] = c["replica"][i]["idx_tmp"] = 0
    e_ref = O.ref_energies(work)
    e64 = np.array([O.energy(cx, 0, 0, m)[0] for m in mm])
    raw64 = np.array([O.energy(cx, 0, 0, m)[1] for m in mm])
    np.savez_compressed(HERE / "ref_energies_c1.npz", mm=mm, e_ref=e_ref, e64=e64, raw64=raw64)
    print("ref_energies_c1.npz:", len(mm), "poses")


if __name__ == "__main__":
    philox_kat()
    ref_energies()
