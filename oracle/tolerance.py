"""The parity tolerance of the FP32 kernels against the FP64 oracle (TEST
INFRASTRUCTURE ONLY: the tests and the smoke check use it).

A ReplicaMC.energy term e_i (the ten normalised terms a_i E_i / L + b_i and
their weighted total, src/backend_gpu/kernel_cuda_l1_montecarlo.cu:460-476)
passes when

    |e_i - e64_i| <= REL * max(|e64_i|, TAU[i])

that is, relative error at most REL = 1e-5 wherever |e64_i| >= TAU[i], and the
absolute error REL * TAU[i] below that scale.

TAU[i] is the magnitude under which an FP32 evaluation of term i cannot
promise a relative error: every term is a sum of many contributions of both
signs (pair terms; per-atom restraints that subtract hpl2; the total's
weighted terms), and FP32 rounding leaves an absolute error of the order of
2^-24 times the sum of the contributions' magnitudes, however small the sum
itself comes out.  Each TAU[i] is the smallest of 0.05, 0.25, 0.5, 1 that
is at least twice the largest absolute FP32 error of term i, divided by REL,
among the poses where |e64_i| < TAU[i], measured over the 10^6 poses of the
precision workload (64 atoms x 3000 points x 1000 KDE points, the largest sums
of the test workloads; tests/test_gpu_precision.py reports it): the
electrostatic and hydrophobic sums cancel most (charges of both signs;
per-atom quadratics minus hpl2; at most 1.4e-6 and 1.5e-6 there over the
kernels measured), the KDE and MCS sums least (below 1.4e-7).  Terms that never fell below 0.25 on that workload
(Lennard-Jones, pmf, hydrogen bond, distance, total) keep 0.25.

The pocket-specific term (index 3) is in addition a step function of the
distance (a pair counts iff d <= pmf0, src/backend_gpu/energy_prt_v1.cu:109-115):
where an FP32 distance and the FP64 one fall on either side of pmf0, one
table value is in one sum and not the other.  Tests count such poses
separately (psp_step_poses) and check the total there after removing the
step.
"""

from __future__ import annotations

import numpy as np

REL = 1e-5
TERMS = ("vdw", "ele", "pmf", "psp", "hdb", "hpc", "kde", "lhm", "dst", "total")
#              vdw   ele   pmf   psp   hdb   hpc   kde   lhm   dst   total
TAU = np.array([0.25, 0.5, 0.25, 0.05, 0.25, 0.5, 0.05, 0.05, 0.25, 0.25])


def scaled_error(x, ref) -> np.ndarray:
    """|x - ref| / (REL * max(|ref|, TAU)) per term (last axis: the ten terms);
    a term passes where this is <= 1."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(x - ref) / (REL * np.maximum(np.abs(ref), TAU))


def relative_error(x, ref, tau=TAU) -> np.ndarray:
    """|x - ref| / max(|ref|, tau): the relative error where |ref| >= tau."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(x - ref) / np.maximum(np.abs(ref), tau)


def check(x, ref, what: str = "") -> np.ndarray:
    """Assert every term of x is within the tolerance of ref; returns the
    per-term maximum of scaled_error."""
    s = scaled_error(x, ref)
    if s.size and s.max() > 1.0:
        idx = np.unravel_index(int(np.argmax(s)), s.shape)
        xi, ri = np.asarray(x, np.float64)[idx], np.asarray(ref, np.float64)[idx]
        term = TERMS[idx[-1]] if s.shape[-1] == len(TERMS) else idx[-1]
        raise AssertionError(f"{what}: term {term} at {idx[:-1]}: {xi!r} vs FP64 {ri!r} "
                             f"(|diff| {abs(xi - ri):.3g} > {REL:g} * max(|ref|, tau))")
    return s.reshape(-1, s.shape[-1]).max(axis=0) if s.size else s
