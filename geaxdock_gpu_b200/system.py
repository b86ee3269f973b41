"""Seeded synthetic docking systems with the shapes of the benchmark configurations.

No public docking benchmark ships with this code, so the workloads are generated:

  config 0  P=1,500 points (24 types), L=28 atoms (12 types) x 8 conformers, K=40 KDE points,
            1 protein conformer x 8 ligand conformers x 16 temperatures = 128 replicas
  config 1  P=3,000 points x 11 conformers (N(0, 0.3 A) jitter), L=40 x 31 conformers,
            20 temperatures = 6,820 replicas
  config 2  2,048 ligands (L ~ U{10..64}, 8 conformers) docked to 8 pockets
            (P ~ U{1,200..6,000}, 4 conformers), round-robin, 16 temperatures = 1,048,576 replicas

Distributions (fixed here, the configurations leave them open):
  * protein points uniform in a sphere around the pocket centre with a 3.0 A minimum pair
    distance by random sequential placement; the radius is 20 A or, when 20 A cannot hold the
    points at that spacing, the radius giving 0.02 points / A^3; points closer than 6 A to the
    pocket centre are left out so the ligand starts in a cavity;
  * point class c cycles 0..3, residue code d ~ U{0..19}, residue id = point index // 3,
    per-point electrostatic value ele ~ N(0, 0.3), hydrophobicity hpp from the force field's
    normalised table, hydrophobic flag (c == 0 and d == 12) or c == 2;
  * ligand: bonded chain with 1.5 A bonds and 109.5 degree angles, random torsions per
    conformer, centred on its centroid; charges N(0, 0.3) re-centred to zero net charge;
  * KDE points within 4 A of the pocket centre, ligand types;
  * MCS: 8 positions, tcc ~ U(0.1, 0.5), 70 % of ligand atoms valid at the reference pose
    + N(0, 1 A);
  * PSP: N(0, 0.5) for the residues of class-2 points;
  * force field: the given raw parameter set (normally the reference's `paras`) with the
    contact-potential well depths pmf1 replaced by N(0, 1);
  * temperatures: geometric in kT from 0.3 to 3.0; moves Gaussian, 0.1 A and 0.05 rad.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import abi

N_PROT_TYPES = 24
N_LIG_TYPES = 12
MCS_LD = abi.MAXLIG + 2


@dataclass
class Workload:
    name: str
    ff: abi.EnePara
    complexes: List[abi.ComplexArrays]
    params: abi.McParams
    n_steps: int

    @property
    def n_rep(self):
        return sum(c.n_rep for c in self.complexes)


def _sphere_points(rng, n, radius, min_dist, hole):
    """Random sequential placement in a sphere with a minimum distance (cell grid)."""
    cell = min_dist
    grid = {}
    pts = np.zeros((n, 3), np.float64)
    m = 0
    tries = 0
    while m < n:
        tries += 1
        if tries > 400 * n:
            raise RuntimeError("placement failed; lower the density")
        v = rng.uniform(-radius, radius, 3)
        r = np.linalg.norm(v)
        if r > radius or r < hole:
            continue
        key = tuple((v // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        if np.sum((pts[j] - v) ** 2) < min_dist * min_dist:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        pts[m] = v
        grid.setdefault(key, []).append(m)
        m += 1
    return pts


def _chain(rng, n, n_conf):
    """Bonded chain (1.5 A bonds, 109.5 deg angles), random torsions per conformer."""
    bond, ang = 1.5, math.radians(109.5)
    out = np.zeros((n_conf, n, 3))
    for c in range(n_conf):
        x = np.zeros((n, 3))
        if n > 1:
            x[1] = [bond, 0, 0]
        if n > 2:
            x[2] = x[1] + bond * np.array([-math.cos(ang), math.sin(ang), 0.0])
        for i in range(3, n):
            a, b, cc = x[i - 3], x[i - 2], x[i - 1]
            bc = cc - b
            bc /= np.linalg.norm(bc)
            nrm = np.cross(b - a, bc)
            if np.linalg.norm(nrm) < 1e-8:
                nrm = np.cross(bc, [0, 0, 1.0])
            nrm /= np.linalg.norm(nrm)
            m = np.cross(nrm, bc)
            tor = rng.uniform(-math.pi, math.pi)
            d2 = np.array([-bond * math.cos(ang), bond * math.sin(ang) * math.cos(tor),
                           bond * math.sin(ang) * math.sin(tor)])
            x[i] = cc + d2[0] * bc + d2[1] * m + d2[2] * nrm
        out[c] = x - x.mean(axis=0)
    return out


def forcefield(raw: abi.EneParaRaw, seed: int, fold=None) -> abi.EnePara:
    """Raw parameters with pmf1 ~ N(0, 1), folded by `fold` (OptimizeEnepara, src/util.C:717-760);
    the library's gd_fold_enepara when None. A caller that must not load the library passes
    another fold with the same arithmetic."""
    if fold is None:
        from .engine import fold_enepara as fold
    rng = np.random.default_rng(seed)
    r = abi.EneParaRaw.from_buffer_copy(bytes(raw))
    pmf = np.ctypeslib.as_array(r.pmf)  # [30][24][2] view
    pmf[:N_PROT_TYPES, :N_LIG_TYPES, 1] = rng.normal(0.0, 1.0, (N_PROT_TYPES, N_LIG_TYPES))
    return fold(r)


def make_complex(rng, ff: abi.EnePara, L: int, n_lig: int, P: int, n_prt: int, n_tmp: int,
                 K: int = 40, M: int = 8, protein=None, pocket=None) -> abi.ComplexArrays:
    """One complex; `protein` (base coordinates, per-point attributes, conformers) may be shared."""
    center = np.zeros(3) if pocket is None else pocket
    if protein is None:
        protein = make_protein(rng, ff, P, n_prt, center)
    px, pt, pc, pe, ps, pf, ph, psp = protein
    lig = _chain(rng, L, n_lig)
    lig_t = rng.integers(0, N_LIG_TYPES, L)
    q = rng.normal(0.0, 0.3, L)
    q -= q.mean()
    temp = np.zeros(n_tmp, abi.TEMP_DTYPE)
    kt = np.geomspace(0.3, 3.0, n_tmp) if n_tmp > 1 else np.array([0.3])
    temp["t"] = kt
    temp["minus_beta"] = (-1.0 / kt).astype(np.float32)
    temp["order"] = np.arange(n_tmp)
    kde = center + rng.uniform(-4.0, 4.0, (K, 3))
    kde_t = rng.integers(0, N_LIG_TYPES, K)
    ref = lig[0] + center
    mx = np.full((M, MCS_LD), abi.MCS_INVALID_COORD, np.float32)
    my, mz = mx.copy(), mx.copy()
    for m in range(M):
        valid = rng.random(L) < 0.7
        noisy = ref + rng.normal(0.0, 1.0, (L, 3))
        for a in np.nonzero(valid)[0]:
            mx[m, a + 1], my[m, a + 1], mz[m, a + 1] = noisy[a]
    return abi.ComplexArrays(
        lig_x=lig[:, :, 0], lig_y=lig[:, :, 1], lig_z=lig[:, :, 2],
        lig_center=np.tile(center, (n_lig, 1)),
        lig_t=np.tile(lig_t, (n_lig, 1)), lig_c=np.tile(q, (n_lig, 1)),
        lig_n=np.tile(np.arange(L), (n_lig, 1)),
        prt_x=px[:, :, 0], prt_y=px[:, :, 1], prt_z=px[:, :, 2], prt_t=pt, prt_c=pc,
        prt_ele=pe, prt_seq3r=ps, prt_hflag=pf, prt_hpp=ph, pocket_center=center, psp=psp,
        kde_x=kde[:, 0], kde_y=kde[:, 1], kde_z=kde[:, 2], kde_t=kde_t,
        mcs_x=mx, mcs_y=my, mcs_z=mz, mcs_tcc=rng.uniform(0.1, 0.5, M), temp=temp)


def make_protein(rng, ff: abi.EnePara, P: int, n_prt: int, center):
    density = 0.02
    radius = max(20.0, (3.0 * P / (4.0 * math.pi * density)) ** (1.0 / 3.0) + 6.0 * 0.5)
    base = _sphere_points(rng, P, radius, 3.0, 6.0) + center
    conf = np.stack([base + (rng.normal(0.0, 0.3, base.shape) if (n_prt > 1) else 0.0)
                     for _ in range(n_prt)])
    t = rng.integers(0, N_PROT_TYPES, P)
    c = np.arange(P) % 4
    d = rng.integers(0, 20, P)
    ele = rng.normal(0.0, 0.3, P)
    seq3r = np.arange(P) // 3
    hflag = ((c == 0) & (d == 12)) | (c == 2)
    hpp = np.array(ff.hpp[:], np.float32)[d]
    n_res = int(seq3r.max()) + 1
    psp = np.zeros((abi.MAXTP2, n_res), np.float32)
    res2 = np.unique(seq3r[c == 2])
    psp[:N_LIG_TYPES, res2] = rng.normal(0.0, 0.5, (N_LIG_TYPES, res2.size))
    tile = lambda a: np.tile(a, (n_prt, 1))
    return (conf, tile(t), tile(c), tile(ele), tile(seq3r), tile(hflag.astype(np.int32)),
            tile(hpp), psp)


def config(cfg: int, raw: abi.EneParaRaw, seed: int = 42, n_ligands: Optional[int] = None,
           n_steps: Optional[int] = None, fold=None) -> Workload:
    """The benchmark configurations 0, 1, 2 (n_ligands shrinks config 2 for tests); `fold` as
    in forcefield()."""
    rng = np.random.default_rng(seed)
    ff = forcefield(raw, seed, fold)
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=abi.STEPS_PER_DUMP,
                           move_scale=(0.1, 0.1, 0.1, 0.05, 0.05, 0.05),
                           move_kind=abi.MOVE_GAUSSIAN, record=1, seed=seed)
    if cfg == 0:
        cx = make_complex(rng, ff, L=28, n_lig=8, P=1500, n_prt=1, n_tmp=16)
        return Workload("config0", ff, [cx], params, n_steps or 5000)
    if cfg == 1:
        cx = make_complex(rng, ff, L=40, n_lig=31, P=3000, n_prt=11, n_tmp=20)
        return Workload("config1", ff, [cx], params, n_steps or 20000)
    if cfg == 2:
        nl = 2048 if n_ligands is None else n_ligands
        pockets = []
        for j in range(8):
            P = int(rng.integers(1200, 6001))
            center = np.array([100.0 * j, 0.0, 0.0])
            pockets.append((make_protein(rng, ff, P, 4, center), center))
        cxs = []
        for i in range(nl):
            L = int(rng.integers(10, 65))
            prot, center = pockets[i % 8]
            cxs.append(make_complex(rng, ff, L=L, n_lig=8, P=prot[0].shape[1], n_prt=4,
                                    n_tmp=16, protein=prot, pocket=center))
        params.steps_per_dump = 100
        return Workload("config2", ff, cxs, params, n_steps or 5000)
    raise ValueError("config must be 0, 1 or 2")


def config1_batch(raw: abi.EneParaRaw, indices, seed: int = 42, fold=None) -> Workload:
    """Complexes `indices` of the batch that stands for config 1 on several GPUs: complex i is
    a config-1 complex (P = 3,000 x 11 conformers, L = 40 x 31 conformers, 20 temperatures)
    drawn with seed + i, all under the force field of `seed`; complex 0 is config 1's own.
    A rank generates only its shard's complexes."""
    ff = forcefield(raw, seed, fold)
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=abi.STEPS_PER_DUMP,
                           move_scale=(0.1, 0.1, 0.1, 0.05, 0.05, 0.05),
                           move_kind=abi.MOVE_GAUSSIAN, record=1, seed=seed)
    cxs = []
    for i in indices:
        rng = np.random.default_rng(seed + i)
        cxs.append(make_complex(rng, ff, L=40, n_lig=31, P=3000, n_prt=11, n_tmp=20))
    return Workload("config1-batch", ff, cxs, params, 20000)
