"""GPU pose energies (gd_eval_poses, the batched kernel's energy code) against
the FP64 oracle and the reference's own FP32 routine, per term.

Tolerance (oracle/tolerance.py): each of the ten ReplicaMC.energy terms must
satisfy |e_gpu - e_64| <= 1e-5 * max(|e_64|, tau_i), relative error 1e-5 above
the term's stated scale tau_i, for the FP32 kernels; the FP64 kernel is held
to 1e-9 relative in the same form.  Against the reference's own FP32 routine
the GPU must be within the reference's own distance from FP64 plus that bound.
"""

from pathlib import Path

import numpy as np
import pytest

from geauxdock_b200 import dock, synth
from geauxdock_b200._lib import GD_PREC_FP32, GD_PREC_FP32_KAHAN, GD_PREC_FP64, check
from oracle import tolerance as TOL

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
TOL64 = 1e-9


def _oracle_energies(O, cx, conf, mm):
    return np.array([O.energy(cx, int(c[0]), int(c[1]), m)[0] for c, m in zip(conf, mm)])


def _check(e, ref, what):
    return TOL.check(e, ref, what)


def _check_vs_reference(out, e_ref, e64, what):
    """The GPU within the reference FP32 routine's own distance from FP64 plus
    the parity bound, of the reference's values."""
    out, e_ref, e64 = (np.asarray(a, np.float64) for a in (out, e_ref, e64))
    bound = np.abs(e_ref - e64) + TOL.REL * np.maximum(np.abs(e64), TOL.TAU)
    gap = np.abs(out - e_ref)
    assert np.all(gap <= bound), f"{what}: {float((gap - bound).max()):.3g} beyond the bound"


@pytest.mark.parametrize("prec", [GD_PREC_FP32, GD_PREC_FP32_KAHAN, GD_PREC_FP64])
def test_golden_config1(lib, enepara, prec):
    """Committed poses of config 1 against the committed reference FP32 and FP64 energies."""
    g = np.load(GOLDEN / "ref_energies_c1.npz")
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    conf = np.zeros((len(g["mm"]), 2), np.int32)
    out, raw, _ = dock.eval_poses(cx, conf, g["mm"], prec)
    _check(out, g["e64"], "vs FP64 oracle")
    _check_vs_reference(out, g["e_ref"], g["e64"], "vs reference FP32")


def test_fp64_kernel_matches_oracle(lib, enepara, oracle_lib):
    pk, job = synth.config1(1)
    cx = synth.to_complex(job, pk, enepara)
    mm = synth.config4_poses(21, 48, radius=5.0)
    conf = np.zeros((48, 2), np.int32)
    _, _, out64 = dock.eval_poses(cx, conf, mm, GD_PREC_FP64, want64=True)
    ref = _oracle_energies(oracle_lib, cx, conf, mm)
    # FP64 pair arithmetic; the float constants -1/sqrt(2 pi) and 1/kde3 of the
    # reference (kernel_cuda_l1_montecarlo.cu:14, :194) bound terms 4 and 6 at ~1e-7
    err = TOL.relative_error(out64, ref)
    assert np.delete(err, [4, 6, 9], axis=1).max() <= TOL64
    assert err.max() <= 2e-7


@pytest.mark.parametrize("prec", [GD_PREC_FP32, GD_PREC_FP32_KAHAN])
def test_ensemble_all_conformations(lib, enepara, oracle_lib, prec):
    """Every (ligand conf, protein conf) pair of a multi-conformation complex,
    poses spread over the pocket, against the oracle."""
    rng = np.random.default_rng(12)
    pk = synth.make_pocket(rng, 1100, 4)
    job = synth.make_job(rng, pk, 47, 5, 350, 11, [1.0], seed=2)
    cx = synth.to_complex(job, pk, enepara)
    conf = np.array([(l, p) for l in range(5) for p in range(4)] * 3, np.int32)
    mm = synth.config4_poses(13, len(conf), radius=6.0)
    out, raw, _ = dock.eval_poses(cx, conf, mm, prec)
    _check(out, _oracle_energies(oracle_lib, cx, conf, mm), "ensemble vs oracle")


def test_edge_sizes(lib, enepara, oracle_lib):
    """Tiny and cap-sized complexes: 1 atom / 1 point / no KDE points of the ligand's
    types; 64 atoms x 2048 points (the reference's MAXLIG x MAXPRO)."""
    rng = np.random.default_rng(3)
    for L, P, K, M in [(1, 1, 0, 1), (2, 5, 3, 1), (64, 2048, 1000, 32), (31, 129, 40, 3)]:
        pk = synth.make_pocket(rng, P, 1)
        job = synth.make_job(rng, pk, L, 1, K, M, [1.0], seed=1)
        cx = synth.to_complex(job, pk, enepara)
        mm = synth.config4_poses(L + P, 12, radius=5.0)
        conf = np.zeros((12, 2), np.int32)
        out, _, _ = dock.eval_poses(cx, conf, mm, GD_PREC_FP32)
        _check(out, _oracle_energies(oracle_lib, cx, conf, mm), f"L={L} P={P}")


@pytest.mark.parametrize("kind", ["none", "dense", "other_types"])
@pytest.mark.parametrize("kpl", [2, 4])
def test_pocket_specific_cells(lib, enepara, oracle_lib, kind, kpl):
    """The pocket-specific term walked over the potential's non-zero cells: no
    cell at all, every (class-2 point, ligand type) cell, and cells only for
    types the ligand does not have (none of them walked), at 2 and 4 points per
    lane; close contacts (poses near the cavity centre) so that d <= pmf0 holds
    for many pairs."""
    rng = np.random.default_rng(11)
    pk = synth.make_pocket(rng, 400, 2)
    job = synth.make_job(rng, pk, 17, 2, 120, 4, [1.0], seed=5)
    present = np.zeros(24, bool)
    present[np.unique(job.lig_type)] = True
    if kind == "none":
        job.psp = np.zeros_like(job.psp)
    elif kind == "dense":
        job.psp = rng.uniform(-1.0, -0.1, size=job.psp.shape).astype(np.float32)
    else:
        job.psp = np.where(present[:, None], 0.0, rng.uniform(-1.0, -0.1, size=job.psp.shape)).astype(np.float32)
    cx = synth.to_complex(job, pk, enepara)
    n = 24
    mm = synth.config4_poses(kpl + 40, n, radius=2.0)
    conf = np.stack([np.arange(n) % 2, (np.arange(n) // 2) % 2], axis=1).astype(np.int32)
    res = [oracle_lib.energy(cx, int(c[0]), int(c[1]), m) for c, m in zip(conf, mm)]
    ref = np.array([r[0] for r in res])
    ref_raw = np.array([r[1] for r in res])
    check(lib.gd_set_option(b"kpl", kpl))
    try:
        out, raw, _ = dock.eval_poses(cx, conf, mm, GD_PREC_FP32_KAHAN)
    finally:
        check(lib.gd_set_option(b"kpl", 0))
    # raw term 3: the pocket-specific sum before normalisation
    if kind != "dense":
        assert np.all(ref_raw[:, 3] == 0.0) and np.all(raw[:, 3] == 0.0)
    else:
        assert np.count_nonzero(ref_raw[:, 3]) > n // 2
    _check(out, ref, f"psp {kind}, kpl {kpl}")


@pytest.mark.parametrize("L", [127, 128])
def test_batched_atom_cap(lib, enepara, oracle_lib, L):
    """The batched path's atom cap (128, beyond the Complex's 64): the largest
    per-atom-pair tables, and an odd count whose last pair has a dummy half."""
    rng = np.random.default_rng(L)
    pk = synth.make_pocket(rng, 700, 2)
    job = synth.make_job(rng, pk, L, 2, 300, 6, [1.0], seed=L)
    n = 24
    mm = synth.config4_poses(L, n, radius=4.0)
    conf = np.stack([np.arange(n) % 2, (np.arange(n) // 2) % 2], axis=1).astype(np.int32)
    e_or, _ = oracle_lib.energy_desc(pk, job, enepara, conf, mm)
    with dock.Ensemble.from_jobs([pk], [job], enepara) as e:
        for prec in (GD_PREC_FP32, GD_PREC_FP32_KAHAN):
            out, _, _ = e.eval_poses(0, conf, mm, prec)
            _check(out, e_or, f"L={L} precision {prec}")


def test_reference_fp32_direct(lib, enepara, oracle_lib):
    """GPU against the reference's own CPU energy routine run here (oracle/_ref),
    on config 2 (40 atoms x 1500 points): the GPU is within the parity bound of
    FP64, and within the reference's own distance from FP64 plus that bound of
    the reference."""
    if not oracle_lib.have_ref():
        pytest.skip("reference library not built")
    pk, job = synth.config2(1)
    cx = synth.to_complex(job, pk, enepara)
    n = 64
    mm = synth.config4_poses(31, n, radius=5.0)
    work = cx.copy()
    conf = np.zeros((n, 2), np.int32)
    for i in range(n):
        r = work[0]["replica"][i * 50]
        r["movematrix"] = mm[i]
        conf[i] = (r["idx_lig"], r["idx_prt"])
    e_ref = oracle_lib.ref_energies(work)[np.arange(n) * 50].astype(np.float64)
    e64 = _oracle_energies(oracle_lib, cx, conf, mm)
    out, _, _ = dock.eval_poses(cx, conf, mm, GD_PREC_FP32)
    _check(out, e64, "vs FP64 oracle")
    _check_vs_reference(out, e_ref, e64, "vs reference FP32")


def test_eval_order_independent(lib, enepara):
    """Results do not depend on how poses are grouped into CTAs."""
    pk, job = synth.config2(1)
    cx = synth.to_complex(job, pk, enepara)
    rng = np.random.default_rng(0)
    conf = np.stack([rng.integers(0, 20, 100), rng.integers(0, 11, 100)], axis=1).astype(np.int32)
    mm = synth.config4_poses(2, 100)
    a, _, _ = dock.eval_poses(cx, conf, mm)
    perm = rng.permutation(100)
    b, _, _ = dock.eval_poses(cx, conf[perm], mm[perm])
    np.testing.assert_array_equal(a[perm], b)
