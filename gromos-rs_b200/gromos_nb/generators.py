"""Seeded synthetic systems for the benchmark workloads (no external data).

SPC water: O-H 0.1 nm, H-O-H 109.47 deg, charges O -0.82 / H +0.41, LJ on
O-O only (C6 = 2.6171e-3 kJ mol^-1 nm^6, C12 = 2.634129e-6 kJ mol^-1 nm^12).
Molecules sit on a cubic lattice of ceil(N^(1/3))^3 sites (the first N of a
seeded shuffle), with a uniform +-0.05 nm jitter per axis and a uniform random
orientation.  Orientations that bring an H of one molecule within 0.15 nm of
an atom of another are re-drawn (seeded) until no such contact remains.

Solute (REMD / FEP / serving workloads): charge groups of 3-5 atoms within
0.15 nm of a CG centre (centres >= 0.55 nm apart), placed in a cavity (waters whose O is within 0.35 nm
of a solute atom are removed); charges ~ N(0, 0.3 e) shifted to zero net
charge per CG; C6/C12 = SPC O values x U[0.5, 2] combined by geometric mean;
all intra-CG pairs excluded.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .system import NonbondedParams, System, Topology, csr_from_lists, water_topology

SPC_C6 = 2.6171e-3
SPC_C12 = 2.634129e-6
SPC_Q = (-0.82, 0.41, 0.41)
OH = 0.1
HOH = math.radians(109.47)


def _spc_frame() -> np.ndarray:
    return np.array([[0.0, 0.0, 0.0], [OH, 0.0, 0.0], [OH * math.cos(HOH), OH * math.sin(HOH), 0.0]])


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from uniform unit quaternions (Shoemake's method)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _bad_molecules(pos: np.ndarray, mol: np.ndarray, box: float, dmin: float, is_h: np.ndarray) -> np.ndarray:
    """Molecules with an H closer than dmin to an atom of another molecule."""
    from scipy.spatial import cKDTree

    wrapped = np.mod(pos, box)
    tree = cKDTree(wrapped, boxsize=box)
    pairs = tree.query_pairs(dmin, output_type="ndarray")
    if pairs.size == 0:
        return np.zeros(0, dtype=np.int64)
    a, b = pairs[:, 0], pairs[:, 1]
    sel = (mol[a] != mol[b]) & (is_h[a] | is_h[b])
    return np.unique(np.concatenate([mol[a[sel]], mol[b[sel]]]))


def _bad_moved(kept_tree, kept_mol: np.ndarray, kept_is_h: np.ndarray, pos: np.ndarray, mol: np.ndarray,
               box: float, dmin: float, is_h: np.ndarray, moved: np.ndarray, check: np.ndarray) -> np.ndarray:
    """Molecules of ``check`` with an H-involving contact closer than dmin to
    another molecule: against the never-moved molecules (``kept_tree``) and
    against the current positions of the ``moved`` ones."""
    from scipy.spatial import cKDTree

    atoms = (3 * check[:, None] + np.arange(3)[None, :]).reshape(-1)
    matoms = (3 * moved[:, None] + np.arange(3)[None, :]).reshape(-1)
    q = np.mod(pos[atoms], box)
    mtree = cKDTree(np.mod(pos[matoms], box), boxsize=box)
    out = set()
    for a, nb in zip(atoms, kept_tree.query_ball_point(q, dmin)):
        if any(is_h[a] or kept_is_h[b] for b in nb):
            out.add(int(mol[a]))
    for a, nb in zip(atoms, mtree.query_ball_point(q, dmin)):
        for bi in nb:
            b = matoms[bi]
            if mol[b] != mol[a] and (is_h[a] or is_h[b]):
                out.add(int(mol[a]))
                break
    return np.array(sorted(out), dtype=np.int64)


def spc_positions(n_waters: int, box: float, seed: int, jitter: float = 0.05, dmin: float = 0.15,
                  max_rounds: int = 200) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n_side = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    spacing = box / n_side
    grid = np.stack(np.meshgrid(np.arange(n_side), np.arange(n_side), np.arange(n_side), indexing="ij"),
                    axis=-1).reshape(-1, 3)
    sites = grid[rng.permutation(grid.shape[0])[:n_waters]]
    centers = (sites + 0.5) * spacing + rng.uniform(-jitter, jitter, size=(n_waters, 3))
    frame = _spc_frame()
    R = _random_rotations(rng, n_waters)
    mol = np.repeat(np.arange(n_waters), 3)
    is_h = np.tile(np.array([False, True, True]), n_waters)

    def place(Rm):
        return (centers[:, None, :] + np.einsum("nij,aj->nai", Rm, frame)).reshape(-1, 3)

    from scipy.spatial import cKDTree

    pos = place(R)
    bad = _bad_molecules(pos, mol, box, dmin, is_h)
    if bad.size:
        # the first round's bad molecules are the only ones ever re-oriented:
        # the others keep the positions indexed here
        moved = bad.copy()
        keep = np.ones(n_waters, dtype=bool)
        keep[moved] = False
        katoms = np.nonzero(np.repeat(keep, 3))[0]
        tree = cKDTree(np.mod(pos[katoms], box), boxsize=box)
        tmol = mol[katoms]
        tis_h = is_h[katoms]
    for _ in range(max_rounds):
        if bad.size == 0:
            break
        # re-orient the molecules in contact, then re-check only those
        R[bad] = _random_rotations(rng, bad.size)
        pos.reshape(n_waters, 3, 3)[bad] = centers[bad][:, None, :] + np.einsum("nij,aj->nai", R[bad], frame)
        bad = _bad_moved(tree, tmol, tis_h, pos, mol, box, dmin, is_h, moved, bad)
    return pos


def spc_water_system(n_waters: int, box: float, seed: int, rcutp: float = 1.4, rcutl: float = 1.4,
                     epsrf: float = 61.0, nsnb: int = 5, c6: float = SPC_C6, c12: float = SPC_C12,
                     name: str = "") -> System:
    topo = water_topology(n_waters, charges=SPC_Q, c6=c6, c12=c12)
    pos = spc_positions(n_waters, box, seed)
    params = NonbondedParams(rcutp=rcutp, rcutl=rcutl, skin=0.0, epsilon=1.0, epsrf=epsrf, kappa=0.0,
                             nsnb=nsnb, algorithm=2, boundary=1)
    return System(topo=topo, pos=pos, box=np.array([box, box, box]), params=params,
                  name=name or f"spc{n_waters}")


def box_for_waters(n_waters: int, density: float = 33.4) -> float:
    """Cubic box edge for a water number density (molecules per nm^3)."""
    return (n_waters / density) ** (1.0 / 3.0)


def solvated_solute_system(n_waters: int, n_solute_atoms: int, seed: int, rc: float = 1.4, epsrf: float = 61.0,
                           nsnb: int = 5, box: Optional[float] = None, perturbed: bool = False,
                           alpha_lj: float = 0.5, alpha_crf: float = 0.5, lam: float = 0.0,
                           name: str = "", single_atom_cgs: bool = False) -> System:
    """A water box of ``n_waters`` SPC with a seeded ``n_solute_atoms`` solute.

    The solute is built of CGs of 3-5 atoms (neutral CGs); with
    ``single_atom_cgs`` every solute atom is its own CG (LJ ions with seeded
    partial charges, neutral as a whole).  This library has no bonded terms,
    so the atoms of a multi-atom CG are free to drift apart: over a few
    hundred MD steps a CG spreads beyond what its centre-based cutoff test
    covers and the run fails; single-atom CGs keep long MD runs stable.
    With ``perturbed`` every solute atom gets independent state-A/B charges
    and C6/C12 (drawn as above) and soft-core alphas.  Returned atom order:
    solute first, then waters.
    """
    rng = np.random.default_rng(seed)
    if box is None:
        box = box_for_waters(n_waters + n_solute_atoms // 3)
    if single_atom_cgs:
        if n_solute_atoms < 1:
            raise ValueError("a solute needs at least 1 atom")
        sizes = [1] * n_solute_atoms
    else:
        # solute CG sizes: 3-5 atoms each
        if n_solute_atoms < 3:
            raise ValueError("a solute needs at least 3 atoms")
        sizes = []
        left = n_solute_atoms
        while left >= 6:
            s = int(rng.integers(3, 6))
            if left - s < 3:
                s = left - 3
            sizes.append(s)
            left -= s
        sizes.append(left)
    ncg = len(sizes)
    min_sep = 0.35 if single_atom_cgs else 0.55
    # CG centres near the box centre, at least min_sep apart as periodic
    # minimum images (seeded rejection), so atoms of different CGs stay
    # >= 0.25 nm apart; the box grows when the solute does not fit
    spread = max(0.35, 0.42 * ncg ** (1.0 / 3.0))
    cg_centres = []
    tries = 0

    def min_dist(c):
        if not cg_centres:
            return np.inf
        d = np.asarray(cg_centres) - c
        d -= box * np.round(d / box)
        return float(np.sqrt((d * d).sum(axis=1)).min())

    while len(cg_centres) < ncg:
        c = box / 2 + rng.uniform(-min(spread, box / 2), min(spread, box / 2), size=3)
        if min_dist(c) >= min_sep:
            cg_centres.append(c)
        tries += 1
        if tries > 200 * ncg:
            if spread >= box / 2:
                box *= 1.02
                cg_centres = [x - (box / 1.02) / 2 + box / 2 for x in cg_centres]
            spread *= 1.1
            tries = 0
    cg_centres = np.asarray(cg_centres)
    if single_atom_cgs:  # an atom at its centre: solute atoms stay >= min_sep apart
        sol_pos = cg_centres.copy()
    else:
        sol_pos = []
        for c, s in zip(cg_centres, sizes):
            d = rng.normal(size=(s, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            sol_pos.append(c + d * rng.uniform(0.05, 0.15, size=(s, 1)))
        sol_pos = np.concatenate(sol_pos)
    # waters: fill the box at liquid density, carve a cavity around the solute,
    # grow the box (seeded, 2% steps) until n_waters remain, keep a seeded subset
    from scipy.spatial import cKDTree

    while True:
        n_fill = int(round(33.4 * box ** 3))
        wpos = spc_positions(max(n_fill, n_waters), box, seed + 7919).reshape(-1, 3, 3)
        tree = cKDTree(np.mod(sol_pos, box), boxsize=box)
        d, _ = tree.query(np.mod(wpos[:, 0, :], box))
        ok = np.nonzero(d > 0.35)[0]
        if ok.size >= n_waters:
            break
        box *= 1.02
        sol_pos = sol_pos - (box / 1.02) / 2 + box / 2
    keep = np.sort(rng.permutation(ok)[:n_waters])
    wpos = wpos[keep].reshape(-1, 3)
    nsa = sol_pos.shape[0]
    nat = nsa + 3 * n_waters

    def draw_params(k):
        q = rng.normal(0.0, 0.3, size=k)
        f6 = rng.uniform(0.5, 2.0, size=k)
        f12 = rng.uniform(0.5, 2.0, size=k)
        return q, f6, f12

    qa, f6a, f12a = draw_params(nsa)
    off = np.concatenate([[0], np.cumsum(sizes)])
    if single_atom_cgs:
        qa -= qa.mean()
    else:
        for c in range(ncg):
            qa[off[c]:off[c + 1]] -= qa[off[c]:off[c + 1]].mean()
    # atom types: 0 = SPC O, 1 = H, 2.. = one type per solute atom (state A), then state B types
    ntypes = 2 + nsa * (2 if perturbed else 1)
    c6_of = np.zeros(ntypes)
    c12_of = np.zeros(ntypes)
    c6_of[0], c12_of[0] = SPC_C6, SPC_C12
    c6_of[2:2 + nsa] = SPC_C6 * f6a
    c12_of[2:2 + nsa] = SPC_C12 * f12a
    if perturbed:
        qb, f6b, f12b = draw_params(nsa)
        if single_atom_cgs:
            qb -= qb.mean()
        else:
            for c in range(ncg):
                qb[off[c]:off[c + 1]] -= qb[off[c]:off[c + 1]].mean()
        c6_of[2 + nsa:] = SPC_C6 * f6b
        c12_of[2 + nsa:] = SPC_C12 * f12b
    lj = np.zeros((ntypes, ntypes, 4))
    c6m = np.sqrt(np.outer(c6_of, c6_of))
    c12m = np.sqrt(np.outer(c12_of, c12_of))
    lj[:, :, 0] = c6m
    lj[:, :, 1] = c12m
    lj[:, :, 2] = c6m
    lj[:, :, 3] = c12m
    charge = np.concatenate([qa, np.tile(SPC_Q, n_waters)])
    iac = np.concatenate([2 + np.arange(nsa), np.tile([0, 1, 1], n_waters)]).astype(np.int32)
    cg_off = np.concatenate([off, nsa + 3 * np.arange(1, n_waters + 1)]).astype(np.int32)
    excl = [[] for _ in range(nat)]
    for c in range(ncg):
        for a in range(off[c], off[c + 1]):
            excl[a] = [b for b in range(off[c], off[c + 1]) if b != a]
    for m in range(n_waters):
        b = nsa + 3 * m
        excl[b], excl[b + 1], excl[b + 2] = [b + 1, b + 2], [b, b + 2], [b, b + 1]
    excl_off, excl_flat = csr_from_lists(excl, nat)
    egroup = np.concatenate([np.zeros(nsa, dtype=np.int32), np.ones(3 * n_waters, dtype=np.int32)])
    topo = Topology(charge=charge, iac=iac, lj=lj, cg_offsets=cg_off, n_solute_atoms=nsa, n_solute_cg=ncg,
                    excl_off=excl_off, excl=excl_flat, o14_off=np.zeros(nat + 1, dtype=np.int32),
                    o14=np.zeros(0, dtype=np.int32), egroup=egroup, n_egroups=2, atoms_per_solvent=3)
    if perturbed:
        topo.pert_idx = np.concatenate([np.arange(nsa), -np.ones(3 * n_waters)]).astype(np.int32)
        topo.pert_a_iac = (2 + np.arange(nsa)).astype(np.int32)
        topo.pert_b_iac = (2 + nsa + np.arange(nsa)).astype(np.int32)
        topo.pert_a_q = qa.copy()
        topo.pert_b_q = qb.copy()
        topo.pert_alpha_lj = np.full(nsa, alpha_lj)
        topo.pert_alpha_crf = np.full(nsa, alpha_crf)
        topo.pp_i = np.zeros(0, dtype=np.int32)
        topo.pp_j = np.zeros(0, dtype=np.int32)
        topo.pp_a_type = np.zeros(0, dtype=np.int32)
        topo.pp_b_type = np.zeros(0, dtype=np.int32)
    params = NonbondedParams(rcutp=rc, rcutl=rc, skin=0.0, epsilon=1.0, epsrf=epsrf, kappa=0.0, nsnb=nsnb,
                             algorithm=2, boundary=1, lam=lam, nlam=1, alphlj=1.0, alphc=1.0)
    pos = np.concatenate([sol_pos, wpos])
    return System(topo=topo, pos=pos, box=np.array([box, box, box]), params=params,
                  name=name or f"solute{nsa}_w{n_waters}")


# Named workloads (sizes from the benchmark configurations)
def config1_spc1000(seed: int = 1001) -> System:
    """1000 SPC waters, 3.104 nm box, single range 1.4 nm, EPSRF 61, NSNB 5."""
    return spc_water_system(1000, 3.104, seed, rcutp=1.4, rcutl=1.4, epsrf=61.0, nsnb=5, name="spc1000")


def config2_spc30000(seed: int = 1002) -> System:
    """30000 SPC waters, 9.65 nm box, twin range 0.8/1.4 nm, EPSRF 61, NSNB 5."""
    return spc_water_system(30000, 9.65, seed, rcutp=0.8, rcutl=1.4, epsrf=61.0, nsnb=5, name="spc30000")


# ---- MD inputs ---------------------------------------------------------------
SPC_MASS = (15.9994, 1.008, 1.008)     # O, H, H (amu)
SOLUTE_MASS = 12.011                   # synthetic solute atoms (amu)
SPC_DHH = 2.0 * OH * math.sin(HOH / 2.0)   # H-H distance of the rigid SPC triangle (nm)
BOLTZ = 0.00831446261815324            # kJ mol^-1 K^-1


def masses(system: System) -> np.ndarray:
    """Per-atom masses: SPC masses for solvent atoms, 12.011 for solute atoms."""
    t = system.topo
    m = np.full(t.n_atoms, SOLUTE_MASS)
    n_w = (t.n_atoms - t.n_solute_atoms) // 3
    m[t.n_solute_atoms:] = np.tile(SPC_MASS, n_w)
    return m


def maxwell_velocities(mass: np.ndarray, temperature: float, seed: int) -> np.ndarray:
    """Seeded Maxwell-Boltzmann velocities (nm/ps), sigma = sqrt(k_B T / m) per component."""
    rng = np.random.default_rng(seed)
    sig = np.sqrt(BOLTZ * temperature / np.asarray(mass, dtype=np.float64))
    return rng.normal(size=(len(mass), 3)) * sig[:, None]
