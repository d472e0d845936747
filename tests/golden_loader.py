"""Load a tests/golden/*.npz fixture back into a gromos_nb System."""
from __future__ import annotations

import json
import os

import numpy as np

from gromos_nb.system import NonbondedParams, System, Topology

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

FIXTURE_NAMES = sorted(f[:-4] for f in os.listdir(GOLDEN_DIR) if f.endswith(".npz"))


def load_fixture(name: str):
    z = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    kw = {}
    for k in ("pert_idx", "pert_a_iac", "pert_b_iac", "pert_a_q", "pert_b_q", "pert_alpha_lj",
              "pert_alpha_crf", "pp_i", "pp_j", "pp_a_type", "pp_b_type"):
        if k in z:
            kw[k] = z[k]
    topo = Topology(charge=z["charge"], iac=z["iac"], lj=z["lj"], cg_offsets=z["cg_offsets"],
                    n_solute_atoms=meta["n_solute_atoms"], n_solute_cg=meta["n_solute_cg"],
                    excl_off=z["excl_off"], excl=z["excl"], o14_off=z["o14_off"], o14=z["o14"],
                    egroup=z["egroup"], n_egroups=meta["n_egroups"],
                    atoms_per_solvent=meta["atoms_per_solvent"],
                    four_pi_eps_i=meta["four_pi_eps_i"], **kw)
    params = NonbondedParams(**meta["params"])
    s = System(topo=topo, pos=z["pos"].copy(), box=z["box"].copy(), params=params, name=name)
    expected = {"e_lj": meta["expected_e_lj"], "e_crf": meta["expected_e_crf"],
                "e_covalent": meta["expected_e_covalent"], "forces": z["expected_forces"],
                "nonbonded_groups": z["expected_nonbonded_groups"],
                "reference_ignores": meta.get("reference_ignores")}
    if "vel" in z:   # MD fixture: initial velocities, masses, expected trajectory
        expected["md"] = {k: z[k] for k in ("vel", "mass", "traj_steps", "traj_pos", "final_pos", "final_vel")}
        expected["md"].update({k: meta[k] for k in ("dt", "nstlim", "bath_temp0", "bath_tau",
                                                   "solvent_constraints")})
    return s, expected
