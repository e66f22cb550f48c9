"""The algorithmic work model behind the roofline's FLOP/s (geauxdock_b200/workmodel.py).

The per-item counts are the reference formulas' operations as written
(energy_prt_v1.cu, energy_kde_v1.cu, energy_mcs_v1.cu,
kernel_cuda_l1_montecarlo.cu); these tests pin how the model combines them:
the hydrogen-bond surcharge goes to (atom, point) pairs whose type pair has
hdb0 > 0.1, the KDE count to (atom, KDE point) pairs of the same type, and the
figure the measurements quote for the replica-ensemble workload stays what they
quote."""

import numpy as np

from geauxdock_b200 import workmodel as W


def _enepara(hdb0):
    return {"hdb0": hdb0}


def test_hand_counted_case():
    hdb0 = np.zeros((24, 31), np.float32)
    hdb0[0, 1] = 0.5      # above the 0.1 guard: the pair gets the hydrogen-bond term
    hdb0[1, 2] = 0.05     # below it: no surcharge
    lig = [0, 1]
    pocket = [0, 1, 2]
    kde = [0, 0, 1, 5, -1, 30]   # types outside [0, 24) are not KDE points of any ligand type
    f = W.flops_per_pose(lig, pocket, kde, 2, _enepara(hdb0))
    expected = (57 * 2 * 3          # every (atom, point) pair
                + 7 * 1             # atom 0 (type 0) x point 1 (type 1)
                + 11 * (2 + 1)      # atom 0 matches two type-0 KDE points, atom 1 one type-1 point
                + 9 * 2 * 2 + 4 * 2  # MCS: 2 rows x 2 atoms, 2 rows
                + 50 * 2 + 55)      # per atom, per pose
    assert f == expected == 581


def test_counts_match_explicit_loops():
    rng = np.random.default_rng(5)
    hdb0 = np.where(rng.random((24, 31)) < 0.15, rng.uniform(0.0, 3.0, (24, 31)), 0.0).astype(np.float32)
    lig = rng.integers(0, 24, 37)
    pocket = rng.integers(0, 31, 211)
    kde = rng.integers(-1, 26, 90)
    nmcs = 7
    n_hdb = sum(1 for a in lig for p in pocket if hdb0[a, p] > np.float32(0.1))
    k_match = sum(1 for a in lig for k in kde if 0 <= k < 24 and k == a)
    L, P = len(lig), len(pocket)
    expected = 57 * L * P + 7 * n_hdb + 11 * k_match + 9 * nmcs * L + 4 * nmcs + 50 * L + 55
    assert W.flops_per_pose(lig, pocket, kde, nmcs, _enepara(hdb0)) == expected


def test_replica_ensemble_figure():
    """3,506,976 FLOPs per pose evaluation of the replica-ensemble workload (40 atoms, 1500
    points, 400 KDE points, 16 MCS templates, seed 1), the figure behind its roofline."""
    from geauxdock_b200 import params, synth

    ep = params.optimize_enepara(params.default_enepara0())
    pk, job = synth.config2(seed=1)
    assert W.job_flops_per_pose(job, pk, ep) == 3_506_976
