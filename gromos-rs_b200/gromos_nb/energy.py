"""Single-point and trajectory energies on the device.

Mirrors ``gromos_forces::energy`` (crates/gromos-forces/src/energy.rs):
``EnergyParams`` (:31-66), ``SinglePointEnergy`` (:68-90) and
``single_point_energy`` (:96-239), whose nonbonded part -- a fresh
charge-group pairlist with one cutoff (``PairlistContainer::new(cutoff,
cutoff, 0.0)``), the LJ + CRF inner loops without virial, the RF-excluded and
1-4 terms -- runs here through ``gr_energy_frames``.  Bonded terms are not
part of this library: ``bond``, ``angle``, ``dihedral``, ``improper`` and
``special`` are 0 and ``potential`` is the nonbonded sum; a caller adds its
bonded energy as the reference does (energy.rs:233-237).

``trajectory_energies`` evaluates many frames in one library call, the loop
of the ener tool (crates/gromos-analysis/src/bin/energy/ener.rs:106-124).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Tuple

import numpy as np

from .nonbonded import Forcefield
from .system import NonbondedParams, System, Topology


@dataclasses.dataclass
class EnergyParams:
    """Parameters of a single-point evaluation (energy.rs:31-66, same defaults)."""

    cutoff: float = 1.4
    epsilon: float = 1.0
    rf_epsilon: float = 78.5
    rf_kappa: float = 0.0
    pairlist_freq: int = 1
    ntf: Tuple[bool, bool, bool, bool] = (True, True, True, True)
    atoms_per_solvent: int = 3
    quartic_bonds: bool = True


@dataclasses.dataclass
class SinglePointEnergy:
    """Energy components (energy.rs:68-90); only the nonbonded ones are computed here."""

    bond: float = 0.0
    angle: float = 0.0
    dihedral: float = 0.0
    improper: float = 0.0
    lj: float = 0.0
    crf: float = 0.0
    special: float = 0.0
    potential: float = 0.0


def _nonbonded_params(params: EnergyParams, box_dims) -> NonbondedParams:
    # vacuum when the box has no x extent (energy.rs:108-117)
    rect = box_dims is not None and float(np.asarray(box_dims, dtype=np.float64)[0]) > 0.0
    return NonbondedParams(rcutp=params.cutoff, rcutl=params.cutoff, skin=0.0, epsilon=params.epsilon,
                           epsrf=params.rf_epsilon, kappa=params.rf_kappa, nsnb=1, boundary=1 if rect else 0)


def _context(topo: Topology, positions, box_dims, params: EnergyParams, device: int) -> Forcefield:
    if params.atoms_per_solvent != topo.atoms_per_solvent:
        raise ValueError("EnergyParams.atoms_per_solvent differs from the topology's solvent size")
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(topo.n_atoms, 3)
    nb = _nonbonded_params(params, box_dims)
    box = np.asarray(box_dims, dtype=np.float64) if nb.boundary == 1 else np.ones(3)
    return Forcefield(System(topo=topo, pos=pos.copy(), box=box.copy(), params=nb), kernel="fixed", device=device)


def single_point_energy(topo: Topology, positions, box_dims, params: EnergyParams,
                        device: int = 0) -> SinglePointEnergy:
    """Nonbonded energy of one configuration (energy.rs:96-239)."""
    return trajectory_energies(topo, [positions], None if box_dims is None else [box_dims], params, device)[0]


def trajectory_energies(topo: Topology, frames, boxes, params: EnergyParams,
                        device: int = 0) -> List[SinglePointEnergy]:
    """``single_point_energy`` of every frame, all frames in one library call.

    ``frames``: (n_frames, n_atoms, 3) positions; ``boxes``: (n_frames, 3) edge
    lengths or None (vacuum).  All frames share the boundary type of the first.
    """
    fr = np.ascontiguousarray(frames, dtype=np.float64).reshape(-1, topo.n_atoms, 3)
    if len(fr) == 0:
        return []
    bx: Optional[np.ndarray] = None if boxes is None else np.asarray(boxes, dtype=np.float64).reshape(len(fr), 3)
    ff = _context(topo, fr[0], None if bx is None else bx[0], params, device)
    try:
        rect = ff.system.params.boundary == 1
        r = ff.energy_frames(fr, bx if rect else None)
    finally:
        ff.close()
    out = []
    for lj, crf in zip(r["e_lj"], r["e_crf"]):
        out.append(SinglePointEnergy(lj=float(lj), crf=float(crf), potential=float(lj) + float(crf)))
    return out
