"""Regenerate the golden fixtures in tests/golden/ from the gromos-rs repository.

The gromosXX v1.6.0 double-precision reference runs shipped with gromos-rs
(crates/gromos-md/tests/gromosXX_references/<system>/) are converted into
small .npz files: the nonbonded topology arrays, step-0 positions and box,
IMD parameters, and the step-0 LJ / CRF energy totals (ENERGY03 '# totals'
lines 11-12), the per-energy-group '# nonbonded' block and the step-0
FREEFORCERED forces.  Step 0 depends only on the input configuration, so
these are known-answer tests for the nonbonded path.

The MD fixture (nacl_1water_settle: leap-frog + SETTLE, no bath coupling)
also carries the masses, the initial velocities, the SETTLE lengths, the time
step and every frame of expected/trajectory.trc plus the final configuration.

Usage (where a gromos-rs checkout is available; its path is required):
    python tests/golden/make_golden.py <path to the gromos-rs repository>
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "gromos-rs_b200"))

from gromos_nb import gromos_io  # noqa: E402

# (fixture dir, topology, configuration, imd, ptp) relative to gromosXX_references
FIXTURES = [
    ("water_216_box", "water_216_box.topo", "water_216_box.conf", "water_216_box.in", None),
    ("water_1000_spc_gridcell", "water_1000_spc.topo", "water_1000_spc.cnf",
     "water_1000_spc_gridcell.in", None),
    ("ch4_water_fep", "../shared/ch4_spc.top", "../shared/ch4_spc.cnf", "ch4_water_fep.in",
     "../shared/ch4_spc_dummy.ptp"),
    ("nacl_water_box", "nacl_water_box.topo", "nacl_water_box.conf", "nacl_water_box.in", None),
    ("water_3_box_twinrange", None, None, None, None),
    ("water_10_box", None, None, None, None),
    ("nacl_3water_box", None, None, None, None),
    ("pair_lj", "pair_lj.topo", "pair_lj.conf", "pair_lj.in", None),
    ("pair_lj_mixed", None, None, None, None),
    ("nacl_pair", None, None, None, None),
    ("nacl_pair_box", None, None, None, None),
    # 1-4 pairs (INE14) in vacuum; step-0 forces include the bonded terms
    ("aladip_vacuum", "../shared/aladip.topo", "aladip_vacuum.conf", "aladip_vacuum.in", None),
    ("butane_vacuum", "butane_vacuum.topo", "butane_vacuum.conf", "butane_vacuum.in", None),
    # perturbed atoms + a PERTATOMPAIR at lambda 0.125 (input.toml names these inputs)
    ("aladip_vacuum_fep", "../shared/aladip.topo", "../aladip_vacuum/aladip_vacuum.conf",
     "aladip_vacuum_fep.in", "../shared/aladip.pttopo"),
    # leap-frog + SETTLE trajectory (MD fixture)
    ("nacl_1water_settle", "nacl_1water_settle.topo", "nacl_1water_settle.conf", "nacl_1water_settle.in", None),
]

MD_FIXTURES = {"nacl_1water_settle"}

# Fixtures that gromos-rs's own harness marks #[ignore] (the reason is recorded in the .npz)
REFERENCE_IGNORES = {
    "aladip_vacuum_fep": "crates/gromos-md/tests/test_gromosXX_references.rs:562 ignores this fixture "
                         "(gromos-rs notes it as a known FEP mismatch with gromosXX)",
}


def _find(d, ext):
    c = [f for f in sorted(os.listdir(d)) if f.endswith(ext)]
    return c[0] if c else None


def convert(ref_root: str, name, topo, conf, imd, ptp):
    base = os.path.join(ref_root, "crates/gromos-md/tests/gromosXX_references", name)
    topo = topo or _find(base, ".topo") or _find(base, ".top")
    conf = conf or _find(base, ".conf") or _find(base, ".cnf")
    imd = imd or _find(base, ".in")
    j = lambda p: os.path.normpath(os.path.join(base, p)) if p else None  # noqa: E731
    s = gromos_io.load_system(j(topo), j(conf), j(imd), j(ptp), name=name)
    ene = gromos_io.read_energy03_step(os.path.join(base, "expected/energies.tre"), 0)
    frc = gromos_io.read_forces_step(os.path.join(base, "expected/forces.trf"), 0)
    t = s.topo.normalized()
    arrays = dict(
        pos=s.pos, box=s.box, charge=t.charge, iac=t.iac, lj=t.lj, cg_offsets=t.cg_offsets,
        excl_off=t.excl_off, excl=t.excl, o14_off=t.o14_off, o14=t.o14,
        egroup=t.egroup, expected_forces=frc,
        expected_nonbonded_groups=np.asarray(ene["nonbonded"], dtype=np.float64),
    )
    if t.pert_idx is not None:
        arrays.update(pert_idx=t.pert_idx, pert_a_iac=t.pert_a_iac, pert_b_iac=t.pert_b_iac,
                      pert_a_q=t.pert_a_q, pert_b_q=t.pert_b_q, pert_alpha_lj=t.pert_alpha_lj,
                      pert_alpha_crf=t.pert_alpha_crf, pp_i=t.pp_i, pp_j=t.pp_j,
                      pp_a_type=t.pp_a_type, pp_b_type=t.pp_b_type)
    meta = dict(
        name=name, n_solute_atoms=t.n_solute_atoms, n_solute_cg=t.n_solute_cg,
        n_egroups=t.n_egroups, atoms_per_solvent=t.atoms_per_solvent,
        four_pi_eps_i=t.four_pi_eps_i, params=s.params.__dict__,
        expected_e_lj=ene["e_lj"], expected_e_crf=ene["e_crf"],
        expected_e_covalent=ene["totals"][3], source=f"gromosXX_references/{name}",
        reference_ignores=REFERENCE_IGNORES.get(name),
    )
    if name in MD_FIXTURES:
        imd_d = gromos_io.read_imd(j(imd))
        steps, frames = gromos_io.read_position_trajectory(os.path.join(base, "expected/trajectory.trc"))
        fpos, _ = gromos_io.read_configuration(os.path.join(base, "expected/final.conf"))
        cons = gromos_io.read_solvent_constraints(j(topo))
        arrays.update(vel=gromos_io.read_velocities(j(conf)), mass=gromos_io.read_masses(j(topo), imd_d["nsm"]),
                      traj_steps=np.asarray(steps, dtype=np.int32), traj_pos=np.stack(frames),
                      final_pos=fpos, final_vel=gromos_io.read_velocities(os.path.join(base, "expected/final.conf")))
        meta.update(dt=imd_d["dt"], nstlim=imd_d["nstlim"], bath_temp0=imd_d["bath_temp0"],
                    bath_tau=imd_d["bath_tau"], solvent_constraints=cons)
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(out, **arrays)
    return out


def main(ref_root: str, names=None):
    for fx in FIXTURES:
        if names and fx[0] not in names:
            continue
        print(convert(ref_root, *fx))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <gromos-rs repository> [fixture names...]")
    main(sys.argv[1], set(sys.argv[2:]))
