"""Topology / parameter containers for the nonbonded path.

The fields mirror the subset of gromos-rs's ``Topology``
(crates/gromos-core/src/topology.rs:619-712) and IMD parameters
(crates/gromos-io/src/imd.rs:81-92, 168-176) that the charge-group pairlist
and the LJ + reaction-field evaluation read.  Everything is stored as flat
NumPy arrays so that it crosses the C ABI (include/gromos_nb.h) without
conversion.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence

import numpy as np


def csr_from_lists(lists: Sequence[Sequence[int]], n: int):
    """Per-atom index lists -> (offsets[n+1], flat) int32 CSR."""
    off = np.zeros(n + 1, dtype=np.int32)
    for i in range(n):
        off[i + 1] = off[i] + (len(lists[i]) if i < len(lists) else 0)
    flat = np.zeros(int(off[-1]), dtype=np.int32)
    for i in range(min(n, len(lists))):
        flat[off[i]:off[i + 1]] = np.asarray(lists[i], dtype=np.int32)
    return off, flat


@dataclasses.dataclass
class Topology:
    """Flat topology for the nonbonded path.

    * CGs are contiguous atom ranges ``cg_offsets[c]:cg_offsets[c+1]``; solute
      CGs come first (``n_solute_cg``), then one CG per solvent molecule, as
      gromos-rs builds them (topology.rs:1204-1262, gromos-io topology.rs:1094-1127).
    * ``excl_off/excl``: symmetric, sorted, de-duplicated exclusions
      (gromos-io topology.rs:1294-1298).
    * ``o14_off/o14``: 1-4 partners as stored by the reader (INE14 lists).
    * ``lj``: ``[n_types, n_types, 4]`` = (c6, c12, cs6, cs12).
    """

    charge: np.ndarray
    iac: np.ndarray
    lj: np.ndarray
    cg_offsets: np.ndarray
    n_solute_atoms: int
    n_solute_cg: int
    excl_off: np.ndarray
    excl: np.ndarray
    o14_off: np.ndarray
    o14: np.ndarray
    egroup: Optional[np.ndarray] = None
    n_egroups: int = 1
    atoms_per_solvent: int = 3
    four_pi_eps_i: float = 138.9354
    # perturbation (PERTATOMPARAM, PERTATOMPAIR); alpha already scaled by ALPHLJ/ALPHC
    pert_idx: Optional[np.ndarray] = None
    pert_a_iac: Optional[np.ndarray] = None
    pert_b_iac: Optional[np.ndarray] = None
    pert_a_q: Optional[np.ndarray] = None
    pert_b_q: Optional[np.ndarray] = None
    pert_alpha_lj: Optional[np.ndarray] = None
    pert_alpha_crf: Optional[np.ndarray] = None
    pp_i: Optional[np.ndarray] = None
    pp_j: Optional[np.ndarray] = None
    pp_a_type: Optional[np.ndarray] = None
    pp_b_type: Optional[np.ndarray] = None

    @property
    def n_atoms(self) -> int:
        return int(self.charge.shape[0])

    @property
    def n_cg(self) -> int:
        return int(self.cg_offsets.shape[0] - 1)

    @property
    def n_types(self) -> int:
        return int(self.lj.shape[0])

    @property
    def n_pert(self) -> int:
        return 0 if self.pert_a_q is None else int(self.pert_a_q.shape[0])

    @property
    def n_pert_pairs(self) -> int:
        return 0 if self.pp_i is None else int(self.pp_i.shape[0])

    def atom_to_cg(self) -> np.ndarray:
        sizes = np.diff(self.cg_offsets)
        return np.repeat(np.arange(self.n_cg, dtype=np.int32), sizes)

    def normalized(self) -> "Topology":
        """Return a copy with contiguous arrays of the ABI dtypes."""
        t = dataclasses.replace(self)
        t.charge = np.ascontiguousarray(self.charge, dtype=np.float64)
        t.iac = np.ascontiguousarray(self.iac, dtype=np.int32)
        t.lj = np.ascontiguousarray(self.lj, dtype=np.float64)
        t.cg_offsets = np.ascontiguousarray(self.cg_offsets, dtype=np.int32)
        for name in ("excl_off", "excl", "o14_off", "o14"):
            setattr(t, name, np.ascontiguousarray(getattr(self, name), dtype=np.int32))
        if self.egroup is not None:
            t.egroup = np.ascontiguousarray(self.egroup, dtype=np.int32)
        for name in ("pert_idx", "pert_a_iac", "pert_b_iac", "pp_i", "pp_j", "pp_a_type", "pp_b_type"):
            v = getattr(self, name)
            if v is not None:
                setattr(t, name, np.ascontiguousarray(v, dtype=np.int32))
        for name in ("pert_a_q", "pert_b_q", "pert_alpha_lj", "pert_alpha_crf"):
            v = getattr(self, name)
            if v is not None:
                setattr(t, name, np.ascontiguousarray(v, dtype=np.float64))
        return t


@dataclasses.dataclass
class NonbondedParams:
    """IMD PAIRLIST / NONBONDED / PERTURBATION fields used by the path.

    ``CRFParameters::new(rcutl, epsilon, epsrf, kappa)`` is built from them
    exactly as gromos-md does (md.rs:326-330, 815), and the pairlist container
    as ``PairlistContainer::new(rcutp, rcutl, skin)`` with ``nsnb``
    (md.rs:836-841).
    """

    rcutp: float = 1.4
    rcutl: float = 1.4
    skin: float = 0.0
    epsilon: float = 1.0
    epsrf: float = 61.0
    kappa: float = 0.0
    nsnb: int = 5
    algorithm: int = 2          # 0 standard, 2 grid_cell (pairlist.rs:815-825)
    boundary: int = 1           # 0 vacuum, 1 rectangular
    lam: float = 0.0            # RLAM
    nlam: int = 1               # NLAM
    alphlj: float = 1.0         # ALPHLJ (already folded into per-atom alphas)
    alphc: float = 1.0          # ALPHC


@dataclasses.dataclass
class System:
    topo: Topology
    pos: np.ndarray             # (n_atoms, 3) float64
    box: np.ndarray             # (3,) float64
    params: NonbondedParams
    name: str = ""

    def copy(self) -> "System":
        return System(self.topo, self.pos.copy(), self.box.copy(), dataclasses.replace(self.params), self.name)


def water_topology(n_waters: int, charges=(-0.82, 0.41, 0.41), iac=(0, 1, 1),
                   c6=2.6171e-3, c12=2.634129e-6, four_pi_eps_i: float = 138.9354) -> Topology:
    """Topology of ``n_waters`` rigid 3-site SPC solvent molecules.

    Solvent only (NPM=0): one CG per molecule, all intra-molecular pairs
    excluded (Topology::solvate, topology.rs:1204-1262), LJ on O-O only.
    """
    nat = 3 * n_waters
    charge = np.tile(np.asarray(charges, dtype=np.float64), n_waters)
    iacs = np.tile(np.asarray(iac, dtype=np.int32), n_waters)
    lj = np.zeros((2, 2, 4), dtype=np.float64)
    lj[0, 0] = (c6, c12, c6, c12)
    cg_off = np.arange(0, nat + 1, 3, dtype=np.int32)
    excl_lists: List[List[int]] = []
    for m in range(n_waters):
        b = 3 * m
        excl_lists += [[b + 1, b + 2], [b, b + 2], [b, b + 1]]
    excl_off, excl = csr_from_lists(excl_lists, nat)
    o14_off = np.zeros(nat + 1, dtype=np.int32)
    return Topology(charge=charge, iac=iacs, lj=lj, cg_offsets=cg_off, n_solute_atoms=0,
                    n_solute_cg=0, excl_off=excl_off, excl=excl, o14_off=o14_off,
                    o14=np.zeros(0, dtype=np.int32), atoms_per_solvent=3,
                    four_pi_eps_i=four_pi_eps_i)
