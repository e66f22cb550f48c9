"""Synthetic generator invariants (the shapes and distributions of the benchmark configs)."""

import numpy as np

from geauxdock_b200 import layout as Lo, synth


def test_ligand_chain(enepara):
    rng = np.random.default_rng(3)
    pk = synth.make_pocket(rng, 500, 2)
    job = synth.make_job(rng, pk, 40, 5, 100, 8, [1.0], seed=1)
    x = job.lig_xyz[0]
    bonds = np.linalg.norm(np.diff(x, axis=0), axis=1)
    np.testing.assert_allclose(bonds, 1.5, atol=1e-5)
    u, v = x[:-2] - x[1:-1], x[2:] - x[1:-1]
    ang = np.degrees(np.arccos(np.sum(u * v, 1) / np.linalg.norm(u, axis=1) / np.linalg.norm(v, axis=1)))
    assert ang.min() >= 99 - 1e-3 and ang.max() <= 119 + 1e-3
    assert abs(float(job.lig_charge.sum())) < 1e-5
    assert job.lig_charge.min() >= -1.0 and job.lig_charge.max() <= 1.0
    for c in job.lig_xyz:
        np.testing.assert_allclose(c.mean(axis=0), 0.0, atol=1e-5)
    assert set(job.lig_type.tolist()) <= set(range(24))


def test_pocket_cavity_and_types():
    rng = np.random.default_rng(5)
    pk = synth.make_pocket(rng, 1500, 3)
    d = np.linalg.norm(pk.xyz[0] - pk.center[0], axis=1)
    assert d.min() > 4.0 and np.abs(pk.xyz[0] - pk.center[0]).max() <= 12.0
    assert set(pk.type.tolist()) <= set(range(30))
    # cdc = (c == 0 && residue == GLY) || c == 2 (util_optimize_soa.C:230)
    np.testing.assert_array_equal(pk.cdc, (((pk.cls == 0) & (pk.res == 12)) | (pk.cls == 2)).astype(np.int32))
    assert set(pk.cls[pk.type == 0].tolist()) == {0} and set(pk.cls[pk.type == 1].tolist()) == {1}
    jitter = pk.xyz[1] - pk.xyz[0]
    assert 0.2 < float(jitter.std()) < 0.4


def test_complex_fits_reference_layout(enepara):
    pk, job = synth.config2(1)
    cx = synth.to_complex(job, pk, enepara, steps_per_exchange=50)
    c = cx[0]
    assert c["size"]["n_rep"] == 20 * 11 * 16 == 3520
    assert c["size"]["lig_natom"] == 40 and c["size"]["prt_npoint"] == 1500
    r = c["replica"][3519]
    assert (r["idx_prt"], r["idx_tmp"], r["idx_lig"]) == (10, 15, 19)
    mb = c["temp"]["minus_beta"][:16]
    np.testing.assert_allclose(-1.0 / mb, synth.ladder(16, 0.3, 3.0), rtol=1e-6)
    assert np.all(c["kde"]["t"][:400][:-1] <= c["kde"]["t"][:400][1:])
    m = c["mcs"][0]
    assert m["ncol"] >= 1 and np.sum(m["x"][:40] != Lo.MCS_INVALID_COORD) == m["ncol"]


def test_poses_in_ball():
    mm = synth.config4_poses(1, 2000, radius=6.0)
    assert np.linalg.norm(mm[:, :3], axis=1).max() <= 6.0
    assert np.abs(mm[:, 4]).max() <= np.pi / 2 + 1e-6
