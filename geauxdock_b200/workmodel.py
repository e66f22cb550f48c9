"""Algorithmic work model of one pose evaluation (one MC step of one replica).

Counting convention: every FP32 + - * / as one flop, sqrt/exp/log as one flop
(and one special-function op), fused multiply-adds counted as two flops.  On
the reference formulas as written (src/backend_gpu/energy_prt_v1.cu,
energy_kde_v1.cu, energy_mcs_v1.cu, kernel_cuda_l1_montecarlo.cu):

  protein-ligand pair   57 flops, + 7 when the (ligand type, point type) pair
                        has hydrogen-bond parameters (hdb0 > 0.1)
  KDE matched pair      11 flops (pairs of the same atom type only)
  MCS cell               9 flops;  per MCS row 4;  per ligand atom 6 + 2
  per pose              rotation 22, transform 42 per atom, normalisation,
                        total and Metropolis 33

FLOPs/pose = (57 + 7 f_hdb) L P + 11 K_match + 9 M L + 4 M + 50 L + 55,
with f_hdb and K_match counted from the complex's types.
"""

from __future__ import annotations

import numpy as np

PAIR_FLOPS = 57
HDB_FLOPS = 7
KDE_FLOPS = 11
MCS_CELL_FLOPS = 9
MCS_ROW_FLOPS = 4
PER_ATOM_FLOPS = 50
PER_POSE_FLOPS = 55
# bytes read per pair-loop item from on-chip memory (not HBM): protein point
# 36 B (9 words, geauxdock_soa.h:52-72), KDE point 16 B
PROTEIN_POINT_BYTES = 36
KDE_POINT_BYTES = 16


def flops_per_pose(lig_type, pocket_type, kde_type, nmcs: int, enepara) -> float:
    """FLOPs of one pose evaluation for ligand atom types, pocket point types, KDE types."""
    lt = np.asarray(lig_type)
    pt = np.asarray(pocket_type)
    kt = np.asarray(kde_type)
    L, P = len(lt), len(pt)
    hdb_active = np.asarray(enepara["hdb0"]) > np.float32(0.1)          # [24, 31]
    n_hdb = int(hdb_active[lt][:, pt].sum())
    kcount = np.bincount(kt[(kt >= 0) & (kt < 24)], minlength=24)
    k_match = int(kcount[lt].sum())
    return float(PAIR_FLOPS * L * P + HDB_FLOPS * n_hdb + KDE_FLOPS * k_match + MCS_CELL_FLOPS * nmcs * L
                 + MCS_ROW_FLOPS * nmcs + PER_ATOM_FLOPS * L + PER_POSE_FLOPS)


def job_flops_per_pose(job, pocket, enepara) -> float:
    return flops_per_pose(job.lig_type, pocket.type, job.kde_type, len(job.mcs_tcc), enepara)
