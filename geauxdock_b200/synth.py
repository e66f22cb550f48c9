"""Seeded synthetic docking complexes with the shapes of the benchmark configs.

The reference measures on the Astex set (data/astex); seeded synthetic inputs
with its structure stand in for it:

* ligand: a random-walk chain of L heavy atoms, 1.5 A bonds, bond angles
  109 +- 10 deg, uniform torsions; atom types uniform over the 24 ligand types
  of the parameter file; charges U[-0.5, 0.5] shifted to zero net charge;
  conformations 1.. are torsion-perturbed copies; every conformation is
  centred on its own centroid (the ligand-centre frame of load.C:285-307);
* pocket: residues with uniform residue codes coarse-grained as the
  reference's protein loader does (CA, peptide plate, side-chain points,
  load.C:538-616), point positions uniform in a 24 A cube around the centre
  outside a 4 A cavity, hpp/ele/cdc/seq3r derived as util_optimize_soa.C:198-231;
  conformations 1.. jittered N(0, 0.3 A);
* pocket-specific potential: ~5% of (ligand type, residue) cells U[-1, 0];
* KDE: points N(cavity centre, 3 A) with uniform types;
* MCS: rows of random atom subsets (>= 1 atom), targets at the native atom
  positions jittered 0.5 A, tcc U[0.1, 0.5];
* temperatures: the geometric ladder of SetTemperature (util.C:326-355);
* moves: 0.5 A and 5 deg.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import layout as Lo
from . import params

MOVE_SCALE = np.array([0.5, 0.5, 0.5] + [math.radians(5.0)] * 3, dtype=np.float32)


@dataclass
class Pocket:
    xyz: np.ndarray          # [nconf, P, 3]
    type: np.ndarray         # [P]
    cls: np.ndarray          # [P]
    cdc: np.ndarray          # [P]
    seq3r: np.ndarray        # [P]
    hpp: np.ndarray          # [P]
    ele: np.ndarray          # [P]
    center: np.ndarray       # [nconf, 3]
    nres: int
    res: np.ndarray = None   # [P] residue code of each point

    @property
    def npoint(self) -> int:
        return self.xyz.shape[1]

    @property
    def nconf(self) -> int:
        return self.xyz.shape[0]


@dataclass
class Job:
    lig_xyz: np.ndarray      # [nlig, L, 3] ligand-centre frame
    lig_type: np.ndarray     # [L]
    lig_charge: np.ndarray   # [L]
    lig_center: np.ndarray   # [nlig, 3]
    kde_xyz: np.ndarray      # [K, 3]
    kde_type: np.ndarray     # [K]
    mcs_xyz: np.ndarray      # [M, L, 3]
    mcs_tcc: np.ndarray      # [M]
    psp: np.ndarray          # [24, ncol]
    temps: np.ndarray        # [ntmp]
    move_scale: np.ndarray = field(default_factory=lambda: MOVE_SCALE.copy())
    seed: int = 1
    pocket: int = 0

    @property
    def natom(self) -> int:
        return self.lig_xyz.shape[1]

    @property
    def nlig(self) -> int:
        return self.lig_xyz.shape[0]

    @property
    def ntmp(self) -> int:
        return len(self.temps)


def ladder(n: int, floor: float, ceiling: float) -> np.ndarray:
    """Temperatures of SetTemperature (src/frontend/util.C:326-355), in float."""
    if n == 1:
        return np.array([floor], dtype=np.float32)
    ratio = np.float32(math.exp(math.log(np.float32(ceiling) / np.float32(floor)) / float(np.float32(n - 1))))
    out, a = [], np.float32(floor)
    for _ in range(n):
        out.append(a)
        a = np.float32(a * ratio)
    return np.array(out, dtype=np.float32)


def make_pocket(rng: np.random.Generator, npoint: int, nconf: int, ep0=None, center=(0.0, 0.0, 0.0),
                cube: float = 24.0, cavity: float = 4.0, jitter: float = 0.3) -> Pocket:
    ep0 = params.default_enepara0() if ep0 is None else ep0
    t, c, d, seq = [], [], [], []
    k = 0
    while len(t) < npoint:
        rc = int(rng.integers(20))
        pts = [(0, 0, k)]
        if k > 1:
            pts.append((1, 1, k - 1))   # peptide plate of the previous residue
        pts += [(pt, pc, k) for pt, pc in params.SIDE_CHAIN[rc]]
        for pt, pc, r in pts:
            if len(t) < npoint:
                t.append(pt)
                c.append(pc)
                d.append(rc)
                seq.append(r + 1)
        k += 1
    t, c, d, seq = (np.array(v, dtype=np.int32) for v in (t, c, d, seq))
    cen = np.asarray(center, dtype=np.float64)
    pos = np.empty((npoint, 3))
    n = 0
    while n < npoint:
        p = rng.uniform(-cube / 2, cube / 2, size=(2 * npoint, 3))
        p = p[np.linalg.norm(p, axis=1) > cavity]
        m = min(len(p), npoint - n)
        pos[n:n + m] = p[:m]
        n += m
    pos += cen
    xyz = np.empty((nconf, npoint, 3), dtype=np.float32)
    xyz[0] = pos
    for i in range(1, nconf):
        xyz[i] = pos + rng.normal(0.0, jitter, size=pos.shape)
    cdc = (((c == 0) & (d == params.GLY)) | (c == 2)).astype(np.int32)
    hpp = ep0["hpp"][d].astype(np.float32)
    ele = np.where(t == 0, ep0["ele"][d + 30], ep0["ele"][t]).astype(np.float32)
    centers = np.tile(cen.astype(np.float32), (nconf, 1))
    return Pocket(xyz, t, c, cdc, seq, hpp, ele, centers, k, d)


def _chain(rng: np.random.Generator, L: int) -> np.ndarray:
    pos = np.zeros((L, 3))
    if L > 1:
        v = rng.normal(size=3)
        pos[1] = 1.5 * v / np.linalg.norm(v)
    for i in range(2, L):
        u = pos[i - 2] - pos[i - 1]
        u /= np.linalg.norm(u)
        r = rng.normal(size=3)
        n1 = np.cross(u, r)
        n1 /= np.linalg.norm(n1)
        n2 = np.cross(u, n1)
        th = math.radians(rng.uniform(99.0, 119.0))
        ph = rng.uniform(0.0, 2 * math.pi)
        v = math.cos(th) * u + math.sin(th) * (math.cos(ph) * n1 + math.sin(ph) * n2)
        pos[i] = pos[i - 1] + 1.5 * v
    return pos


def _torsion_perturb(rng: np.random.Generator, pos: np.ndarray, n: int = 3) -> np.ndarray:
    out = pos.copy()
    L = len(out)
    for _ in range(n if L > 3 else 0):
        b = int(rng.integers(1, L - 2))
        axis = out[b + 1] - out[b]
        axis /= np.linalg.norm(axis)
        ang = rng.uniform(-math.pi / 3, math.pi / 3)
        K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
        R = np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * K @ K
        out[b + 2:] = (out[b + 2:] - out[b + 1]) @ R.T + out[b + 1]
    return out


def make_job(rng: np.random.Generator, pocket: Pocket, natom: int, nlig: int, nkde: int, nmcs: int,
             temps, seed: int = 1, pocket_index: int = 0) -> Job:
    base = _chain(rng, natom)
    confs = [base] + [_torsion_perturb(rng, base) for _ in range(nlig - 1)]
    lig = np.stack([c - c.mean(axis=0) for c in confs]).astype(np.float32)
    ltype = rng.integers(0, 24, size=natom).astype(np.int32)
    q = rng.uniform(-0.5, 0.5, size=natom)
    charge = (q - q.mean()).astype(np.float32)
    cen = pocket.center[0].astype(np.float32)
    lcenter = np.tile(cen, (nlig, 1))
    kde_xyz = (cen + rng.normal(0.0, 3.0, size=(nkde, 3))).astype(np.float32)
    kde_type = rng.integers(0, 24, size=nkde).astype(np.int32)
    native = lig[0] + cen
    mcs = np.full((nmcs, natom, 3), Lo.MCS_INVALID_COORD, dtype=np.float32)
    for m in range(nmcs):
        sel = rng.random(natom) < 0.5
        if not sel.any():
            sel[rng.integers(natom)] = True
        mcs[m, sel] = (native[sel] + rng.normal(0.0, 0.5, size=(int(sel.sum()), 3))).astype(np.float32)
    tcc = rng.uniform(0.1, 0.5, size=nmcs).astype(np.float32)
    ncol = int(pocket.seq3r.max()) + 1
    psp = np.where(rng.random((24, ncol)) < 0.05, rng.uniform(-1.0, 0.0, size=(24, ncol)), 0.0).astype(np.float32)
    return Job(lig, ltype, charge, lcenter, kde_xyz, kde_type, mcs, tcc, psp,
               np.asarray(temps, dtype=np.float32), MOVE_SCALE.copy(), seed, pocket_index)


# ------------------------------------------------------ reference Complex
def to_complex(job: Job, pocket: Pocket, enepara: np.ndarray, steps_total: int = 200, steps_per_dump: int = 200,
               steps_per_exchange: int = 0) -> np.ndarray:
    """A reference-layout Complex record (within the reference's caps)."""
    L, nlig, P, nprt = job.natom, job.nlig, pocket.npoint, pocket.nconf
    if L > Lo.MAXLIG or P > Lo.MAXPRO or nlig > Lo.MAX_CONF_LIG or nprt > Lo.MAX_CONF_PRT:
        raise ValueError(f"exceeds the Complex caps: L={L} P={P} nlig={nlig} nprt={nprt}")
    if job.psp.shape[1] > Lo.MAXPRO or len(job.kde_type) > Lo.MAXKDE or len(job.mcs_tcc) > Lo.MAX_MCS_ROW:
        raise ValueError("psp/kde/mcs exceed the Complex caps")
    cx = Lo.aligned_zeros(Lo.COMPLEX)
    c = cx[0]
    order = np.argsort(job.lig_type, kind="stable")
    for i in range(nlig):
        g = c["lig"][i]
        x = job.lig_xyz[i]
        for k, ax in enumerate("xyz"):
            g[ax + "1"][:L] = x[order, k]
            g[ax + "2"][:L] = x[:, k]
            g[ax + "3"][:L] = x[order, k]
        g["t1"][:L] = job.lig_type[order]
        g["c1"][:L] = job.lig_charge[order]
        g["t2"][:L] = job.lig_type
        g["c2"][:L] = job.lig_charge
        g["t3"][:L] = job.lig_type[order]
        g["c3"][:L] = job.lig_charge[order]
        g["center"] = job.lig_center[i]
        g["lig_natom"] = L
    porder = np.argsort(pocket.cls, kind="stable")   # OptimizeProtein sorts by class (util_optimize_soa.C:236-267)
    for i in range(nprt):
        p = c["prt"][i]
        for k, ax in enumerate("xyz"):
            p[ax][:P] = pocket.xyz[i, porder, k]
        for f in ("type", "cls", "cdc", "seq3r", "hpp", "ele"):
            dst = {"type": "t", "cls": "c"}.get(f, f)
            p[dst][:P] = getattr(pocket, f)[porder]
        p["pocket_center"] = pocket.center[i]
        p["prt_npoint"] = P
    c["psp"]["psp"][:24, :job.psp.shape[1]] = job.psp
    korder = np.argsort(job.kde_type, kind="stable")   # OptimizeKde (util_optimize_soa.C:336-372)
    K = len(korder)
    c["kde"]["t"][:K] = job.kde_type[korder]
    for k, ax in enumerate("xyz"):
        c["kde"][ax][:K] = job.kde_xyz[korder, k]
    c["kde"]["kde_npoint"] = K
    M = len(job.mcs_tcc)
    for m in range(M):
        row = c["mcs"][m]
        row["x"][:] = Lo.MCS_INVALID_COORD
        row["y"][:] = Lo.MCS_INVALID_COORD
        row["z"][:] = Lo.MCS_INVALID_COORD
        for k, ax in enumerate("xyz"):
            row[ax][:L] = job.mcs_xyz[m, :, k]
        row["ncol"] = int((job.mcs_xyz[m, :, 0] != Lo.MCS_INVALID_COORD).sum())
        row["tcc"] = job.mcs_tcc[m]
    c["enepara"] = enepara
    ntmp = job.ntmp
    for t in range(ntmp):
        c["temp"][t]["t"] = job.temps[t]
        c["temp"][t]["minus_beta"] = np.float32(0.0) - np.float32(np.float32(1.0) / job.temps[t])
        c["temp"][t]["order"] = t
    nrep = nlig * nprt * ntmp
    if nrep > Lo.MAX_REP:
        raise ValueError(f"{nrep} replicas exceed MAX_REP")
    for p in range(nprt):                               # SetReplica (util.C:371-406)
        for t in range(ntmp):
            for l in range(nlig):
                r = ntmp * nlig * p + nlig * t + l
                rep = c["replica"][r]
                rep["idx_rep"], rep["idx_prt"], rep["idx_tmp"], rep["idx_lig"] = r, p, t, l
    sz = c["size"]
    sz["n_lig"], sz["n_prt"], sz["n_tmp"], sz["n_rep"] = nlig, nprt, ntmp, nrep
    sz["lig_natom"], sz["prt_npoint"], sz["kde_npoint"], sz["mcs_nrow"] = L, P, K, M
    mp = c["mcpara"]
    mp["steps_total"], mp["steps_per_dump"], mp["steps_per_exchange"] = steps_total, steps_per_dump, steps_per_exchange
    mp["move_scale"] = job.move_scale
    c["lig_file"] = b"synthetic.sdf"
    c["prt_file"] = b"synthetic.pdb"
    c["rep_begin"], c["rep_end"] = 0, nrep - 1
    return cx


# ------------------------------------------------ cap-free descriptions
def job_desc(job: Job, keep: list):
    """ctypes gd_job_desc_t for `job`; arrays it points to are appended to keep."""
    from ._lib import JobDesc

    def ptr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    d = JobDesc()
    d.natom, d.nlig = job.natom, job.nlig
    d.lig_xyz, d.lig_type = ptr(job.lig_xyz, np.float32), ptr(job.lig_type, np.int32)
    d.lig_charge, d.lig_center = ptr(job.lig_charge, np.float32), ptr(job.lig_center, np.float32)
    d.pocket = job.pocket
    d.nkde = len(job.kde_type)
    d.kde_xyz, d.kde_type = ptr(job.kde_xyz, np.float32), ptr(job.kde_type, np.int32)
    d.nmcs = len(job.mcs_tcc)
    d.mcs_xyz, d.mcs_tcc = ptr(job.mcs_xyz, np.float32), ptr(job.mcs_tcc, np.float32)
    d.psp_ncol = job.psp.shape[1]
    d.psp = ptr(job.psp, np.float32)
    d.ntmp = job.ntmp
    d.temperature = ptr(job.temps, np.float32)
    for i in range(6):
        d.move_scale[i] = float(job.move_scale[i])
    d.seed = int(job.seed)
    return d


def pocket_desc(p: Pocket, keep: list):
    from ._lib import PocketDesc

    def ptr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    d = PocketDesc()
    d.npoint, d.nconf = p.npoint, p.nconf
    d.xyz = ptr(p.xyz, np.float32)
    d.type, d.cls, d.cdc, d.seq3r = (ptr(getattr(p, f), np.int32) for f in ("type", "cls", "cdc", "seq3r"))
    d.hpp, d.ele = ptr(p.hpp, np.float32), ptr(p.ele, np.float32)
    d.center = ptr(p.center, np.float32)
    return d


# ------------------------------------------------------ benchmark configs
def config1(seed: int = 1):
    """Single complex: L=24, P=600, K=200, M=8, 1 temperature, 1 replica."""
    rng = np.random.default_rng(seed)
    pk = make_pocket(rng, 600, 1)
    job = make_job(rng, pk, 24, 1, 200, 8, [0.044], seed=seed)
    return pk, job


def config2(seed: int = 1):
    """Replica ensemble: L=40 x 20 conformations, P=1500 x 11, K=400, M=16, 16 temperatures 0.3..3.0."""
    rng = np.random.default_rng(seed)
    pk = make_pocket(rng, 1500, 11)
    job = make_job(rng, pk, 40, 20, 400, 16, ladder(16, 0.3, 3.0), seed=seed)
    return pk, job


def config3(seed: int = 1, nligand: int = 512):
    """Batched uneven screening: ligands of U[12, 64] atoms x 10 conformations vs one P=2000 x 5 pocket,
    K=600, M=16, 8 temperatures."""
    rng = np.random.default_rng(seed)
    pk = make_pocket(rng, 2000, 5)
    temps = ladder(8, 0.3, 3.0)
    jobs = [make_job(rng, pk, int(rng.integers(12, 65)), 10, 600, 16, temps, seed=seed + 1000 * (j + 1))
            for j in range(nligand)]
    return pk, jobs


def config4_poses(seed: int, n: int, radius: float = 6.0) -> np.ndarray:
    """Random poses: uniform rotations (ZYX angles, middle angle asin(U[-1,1])) and translations
    uniform in a ball of `radius` about the cavity centre."""
    rng = np.random.default_rng(seed)
    mm = np.empty((n, 6), dtype=np.float32)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    mm[:, :3] = v * (radius * rng.random(n) ** (1.0 / 3.0))[:, None]
    mm[:, 3] = rng.uniform(-math.pi, math.pi, size=n)
    mm[:, 4] = np.arcsin(rng.uniform(-1.0, 1.0, size=n))
    mm[:, 5] = rng.uniform(-math.pi, math.pi, size=n)
    return mm


def config4(seed: int = 1):
    """Precision study complex: L=64, P=3000, K=1000, M=16."""
    rng = np.random.default_rng(seed)
    pk = make_pocket(rng, 3000, 1)
    job = make_job(rng, pk, 64, 1, 1000, 16, [1.0], seed=seed)
    return pk, job


def serving_pockets(seed: int = 1, sizes=(800, 1500, 2200, 3000), nconf: int = 5):
    rng = np.random.default_rng(seed)
    return [make_pocket(rng, s, nconf) for s in sizes]


def serving_job(rng: np.random.Generator, pockets, seed: int, lo: int = 8, hi: int = 80) -> Job:
    """A serving request: log-uniform ligand size, random resident pocket, 10 x 5 x 8 replicas."""
    L = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
    pi = int(rng.integers(len(pockets)))
    return make_job(rng, pockets[pi], L, 10, 600, 16, ladder(8, 0.3, 3.0), seed=seed, pocket_index=pi)
