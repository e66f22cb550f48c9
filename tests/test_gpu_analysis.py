"""Post-analysis on the GPU against a numpy restatement: best pose per replica,
its RMSD to the native pose, and leader clustering of the best poses in energy
order (a pose joins the first cluster whose leader is within the cut-off)."""

import numpy as np
import pytest

from geauxdock_b200 import dock, synth

pytestmark = pytest.mark.gpu


def _rot(mm):
    s1, c1 = np.sin(mm[3]), np.cos(mm[3])
    s2, c2 = np.sin(mm[4]), np.cos(mm[4])
    s3, c3 = np.sin(mm[5]), np.cos(mm[5])
    return np.array([[c1 * c2, c1 * s2 * s3 - c3 * s1, s1 * s3 + c1 * c3 * s2],
                     [c2 * s1, c1 * c3 + s1 * s2 * s3, c3 * s1 * s2 - c1 * s3],
                     [-s2, c2 * s3, c2 * c3]])


def _coords(job, il, mm):
    return job.lig_xyz[il].astype(np.float64) @ _rot(mm.astype(np.float64)).T + mm[:3] + job.lig_center[il]


@pytest.mark.parametrize("cut", [0.5, 1.5, 3.0])
def test_cluster_matches_numpy(lib, enepara, cut):
    rng = np.random.default_rng(31)
    pk = synth.make_pocket(rng, 400, 2)
    job = synth.make_job(rng, pk, 22, 4, 120, 6, synth.ladder(6, 0.3, 3.0), seed=7)
    with dock.Ensemble.from_jobs([pk], [job], enepara) as ens:
        ens.init()
        ens.run(150, 25)
        ens.sync()
        reps = ens.replicas(0)
        mm, e = ens.best_poses(0)
        cl, cof, rmsd = ens.cluster(0, rmsd_cut=cut)
    n = len(e)
    native = _coords(job, 0, np.zeros(6, np.float32))
    poses = [_coords(job, int(reps["idx_lig"][r]), mm[r]) for r in range(n)]
    want_rmsd = np.array([np.sqrt(((p - native) ** 2).sum(1).mean()) for p in poses])
    np.testing.assert_allclose(rmsd, want_rmsd, atol=2e-4)
    order = sorted(range(n), key=lambda r: (e[r], r))
    leaders, want = [], np.full(n, -1)
    for r in order:
        for c, l in enumerate(leaders):
            if np.sqrt(((poses[r] - poses[l]) ** 2).sum(1).mean()) <= cut:
                want[r] = c
                break
        else:
            want[r] = len(leaders)
            leaders.append(r)
    assert np.array_equal(cof, want)
    assert len(cl) == len(leaders)
    assert [c["representative"] for c in cl] == leaders
    assert sum(c["size"] for c in cl) == n
    for c, l in zip(cl, leaders):
        members = np.nonzero(want == want[l])[0]
        assert c["size"] == len(members)
        assert c["mean_energy"] == pytest.approx(e[members].mean(), rel=1e-5)
        assert c["rep_energy"] == pytest.approx(e[l], rel=1e-6)
        assert c["rep_rmsd"] == pytest.approx(want_rmsd[l], abs=2e-4)
