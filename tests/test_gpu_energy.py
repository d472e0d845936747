"""single_point_energy / gr_energy_frames: energies of many configurations.

* the reference's fixtures against the FP64 oracle with one cutoff (RCUTL),
  and against the gromosXX step-0 energies where the single-cutoff result is
  the step-0 twin-range result (it is not where the solvent short list's
  first-atom image and the long list's per-atom images differ, in boxes near
  twice the cutoff; the oracle restates both rules);
* a trajectory of displaced frames in changing boxes against the FP64 oracle
  (relative 1e-5), and bit for bit against one ``Forcefield.apply`` per frame;
* frames whose lists overflow are computed again and still agree.
"""
import dataclasses

import numpy as np
import pytest

import oracle_binding as ob
from golden_loader import FIXTURE_NAMES, load_fixture
from gromos_nb import generators as g
from gromos_nb.energy import EnergyParams, single_point_energy, trajectory_energies
from gromos_nb.nonbonded import Forcefield
from gromos_nb.system import System

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-9)


# single_point_energy has no lambda (crates/gromos-forces/src/energy.rs:96-239): it evaluates the
# topology's regular charges and types, so the perturbed fixtures are left out
UNPERTURBED_FIXTURES = [n for n in FIXTURE_NAMES if n not in ("ch4_water_fep", "aladip_vacuum_fep")]


@pytest.mark.parametrize("name", UNPERTURBED_FIXTURES)
def test_single_point_energy_fixtures(name):
    s, ex = load_fixture(name)
    p = s.params
    params = EnergyParams(cutoff=p.rcutl, epsilon=p.epsilon, rf_epsilon=p.epsrf, rf_kappa=p.kappa,
                          atoms_per_solvent=s.topo.atoms_per_solvent)
    box = s.box if p.boundary == 1 else np.zeros(3)
    e = single_point_energy(s.topo, s.pos, box, params)
    single = s.copy()
    single.params = dataclasses.replace(p, rcutp=p.rcutl, skin=0.0)
    o = ob.OracleForcefield(single).apply()
    for key, got in (("e_lj", e.lj), ("e_crf", e.crf)):
        assert rel(got, o[key]) <= 1e-5 or abs(got - o[key]) <= 1e-6, (key, got, o[key])
        if abs(o[key] - ex[key]) <= 1e-8 * max(abs(ex[key]), 1e-12) + 1e-12:   # fixture pins this case
            assert rel(got, ex[key]) <= 1e-5 or abs(got - ex[key]) <= 1e-6, (key, got, ex[key])
    assert e.potential == e.lj + e.crf and e.bond == 0.0


def _frames(s, n, seed):
    rng = np.random.default_rng(seed)
    frames, boxes = [], []
    for k in range(n):
        scale = 1.0 + 0.01 * (k % 3)          # box breathing: positions scale with the box
        frames.append(s.pos * scale + rng.normal(0.0, 0.01, s.pos.shape))
        boxes.append(s.box * scale)
    return np.array(frames), np.array(boxes)


def test_trajectory_energies_match_oracle_and_single_calls():
    s = g.spc_water_system(1000, 3.11, seed=5, rcutp=1.0, rcutl=1.0)
    params = EnergyParams(cutoff=1.0, epsilon=1.0, rf_epsilon=s.params.epsrf, rf_kappa=0.0)
    frames, boxes = _frames(s, 6, seed=7)
    es = trajectory_energies(s.topo, frames, boxes, params)
    assert len(es) == len(frames)
    for k, e in enumerate(es):
        sk = System(topo=s.topo, pos=frames[k], box=boxes[k],
                    params=dataclasses.replace(s.params, rcutp=1.0, rcutl=1.0, skin=0.0, nsnb=1))
        o = ob.OracleForcefield(sk).apply(frames[k])
        escale = max(abs(o["e_lj"]), abs(o["e_crf"]))
        assert abs(e.lj - o["e_lj"]) <= 1e-5 * escale, (k, e.lj, o["e_lj"])
        assert abs(e.crf - o["e_crf"]) <= 1e-5 * escale, (k, e.crf, o["e_crf"])
        ff = Forcefield(sk)
        r = ff.apply(frames[k])
        ff.close()
        assert r["e_lj"] == e.lj and r["e_crf"] == e.crf, k


def test_energy_frames_redo_after_list_overflow():
    s = g.spc_water_system(1000, 3.11, seed=6, rcutp=1.0, rcutl=1.0)
    s.params = dataclasses.replace(s.params, skin=0.0, nsnb=1)
    frames, boxes = _frames(s, 3, seed=8)
    # a sparse first frame (box stretched by 40%) sizes the lists; the dense frames overflow them
    frames = np.concatenate([s.pos[None] * 1.4, frames])
    boxes = np.concatenate([s.box[None] * 1.4, boxes])
    ff = Forcefield(s, list_capacity=32)
    r = ff.energy_frames(frames, boxes, groups=True)
    ff.close()
    ref = Forcefield(s)
    want = ref.energy_frames(frames, boxes)
    ref.close()
    np.testing.assert_array_equal(r["e_lj"], want["e_lj"])
    np.testing.assert_array_equal(r["e_crf"], want["e_crf"])
    assert r["egroup_lj"].shape == (len(frames), 1, 1)
    np.testing.assert_array_equal(r["egroup_lj"][:, 0, 0], r["e_lj"])


def test_energy_frames_vacuum_pair():
    s, ex = load_fixture("pair_lj")
    params = EnergyParams(cutoff=s.params.rcutl, rf_epsilon=s.params.epsrf, rf_kappa=s.params.kappa,
                          atoms_per_solvent=s.topo.atoms_per_solvent)
    shifted = [s.pos + 0.1 * k for k in range(3)]   # a rigid shift changes nothing in vacuum
    es = trajectory_energies(s.topo, shifted, None, params)
    assert all(e.lj == es[0].lj and e.crf == es[0].crf for e in es)
    assert rel(es[0].lj, ex["e_lj"]) <= 1e-5 or abs(es[0].lj - ex["e_lj"]) <= 1e-6
