"""GPU MD steps (leap-frog + SETTLE around the force call) against the oracle.

The device runs Forcefield::apply, LeapFrogVelocity, LeapFrogPosition and
SETTLE (md.rs:1144-1230 sequence, no thermostat) with positions and
velocities resident; the oracle runs the same sequence in FP64.  Forces
differ by the FP32 pair arithmetic (<= 1e-5 RMS relative), so trajectories
agree closely over a few tens of steps:
* positions: max |dx| <= 1e-5 nm after 20 steps,
* velocities: RMS relative error <= 1e-4,
* kinetic energy: relative 1e-5, nonbonded energies of the last step: 1e-5,
* SETTLE: every O-H and H-H distance within 1e-9 nm of its constraint.
"""
import numpy as np
import pytest

import oracle_binding as ob
from gromos_nb import generators as g
from gromos_nb.nonbonded import Forcefield

pytestmark = pytest.mark.gpu


def run_both(s, n_steps, seed=7, T=300.0):
    m = g.masses(s)
    v = g.maxwell_velocities(m, T, seed)
    ff = Forcefield(s)
    ff.upload_positions(s.pos)
    ff.md_init(m, v, dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
    st = ff.md_run(n_steps)
    x, vg = ff.md_state()
    ff.close()
    orc = ob.OracleForcefield(s)
    xo, vo, so = orc.md_run(s.pos, v, m, n_steps, dt=0.002, dist_oh=0.1, dist_hh=g.SPC_DHH)
    orc.close()
    return x, vg, st, xo, vo, so


def check(s, x, vg, st, xo, vo, so):
    assert st["settle_failures"] == 0 and so["settle_failures"] == 0
    assert np.abs(x - xo).max() <= 1e-5
    assert np.sqrt(((vg - vo) ** 2).sum() / (vo ** 2).sum()) <= 1e-4
    assert abs(st["e_kin"] - so["e_kin"]) <= 1e-5 * abs(so["e_kin"])
    esc = max(abs(so["e_lj"]), abs(so["e_crf"]))
    assert abs(st["e_lj"] - so["e_lj"]) <= 1e-5 * esc
    assert abs(st["e_crf"] - so["e_crf"]) <= 1e-5 * esc
    nsa = s.topo.n_solute_atoms
    w = x[nsa:].reshape(-1, 3, 3)
    assert np.abs(np.linalg.norm(w[:, 1] - w[:, 0], axis=1) - 0.1).max() <= 1e-9
    assert np.abs(np.linalg.norm(w[:, 2] - w[:, 0], axis=1) - 0.1).max() <= 1e-9
    assert np.abs(np.linalg.norm(w[:, 2] - w[:, 1], axis=1) - g.SPC_DHH).max() <= 1e-9


def test_md_water_twin_range_vs_oracle():
    s = g.spc_water_system(800, box=g.box_for_waters(800), seed=31, rcutp=0.8, rcutl=1.2, nsnb=5)
    check(s, *run_both(s, 20))


def test_md_solvated_solute_vs_oracle():
    s = g.solvated_solute_system(600, 30, seed=1005, rc=1.0)
    check(s, *run_both(s, 12))


def test_md_settle_fixture_vs_gromosxx():
    """nacl_1water_settle (gromosXX leap-frog + SETTLE, no bath, 10 steps of 2 fs) on the device:
    every written frame and the final configuration within 2e-9 nm of the gromosXX output
    (9 decimals), final velocities within 1e-8 nm/ps; the oracle reproduces the same file to
    1e-9 (test_oracle_pins.py), so the device stays within FP32-pair-arithmetic noise of it."""
    from golden_loader import load_fixture
    s, ex = load_fixture("nacl_1water_settle")
    md = ex["md"]
    cons = {(i, j): d for i, j, d in md["solvent_constraints"]}
    ff = Forcefield(s)
    ff.upload_positions(s.pos)
    ff.md_init(md["mass"], md["vel"], dt=md["dt"], settle=True, dist_oh=cons[(0, 1)], dist_hh=cons[(1, 2)],
               tau=-1.0)
    done = 0
    for step, frame in zip(md["traj_steps"][1:], md["traj_pos"][1:]):
        st = ff.md_run(int(step) - done)
        done = int(step)
        x, v = ff.md_state()
        assert st["settle_failures"] == 0
        assert np.abs(x - frame).max() <= 2e-9, (step, np.abs(x - frame).max())
    ff.md_run(md["nstlim"] - done)
    x, v = ff.md_state()
    ff.close()
    assert np.abs(x - md["final_pos"]).max() <= 2e-9
    assert np.abs(v - md["final_vel"]).max() <= 1e-8


def test_md_split_calls_bit_identical():
    """md_run(7) + md_run(13) == md_run(20) bit for bit (the rebuild cadence carries over)."""
    s = g.spc_water_system(500, box=g.box_for_waters(500), seed=32, rcutp=0.8, rcutl=1.0, nsnb=4)
    m = g.masses(s)
    v = g.maxwell_velocities(m, 300.0, 3)
    out = []
    for parts in ((20,), (7, 13)):
        ff = Forcefield(s)
        ff.upload_positions(s.pos)
        ff.md_init(m, v, dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
        for n in parts:
            ff.md_run(n)
        out.append(ff.md_state())
        ff.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_md_rollback_after_list_overflow():
    """A rebuild inside gr_md_run overflows its (deliberately tiny) lists: the period is rolled back,
    the lists grown and the steps run again -- the trajectory is the oracle's all the same."""
    s = g.spc_water_system(1200, box=g.box_for_waters(1200), seed=33, rcutp=0.8, rcutl=1.2, nsnb=3)
    m = g.masses(s)
    v = g.maxwell_velocities(m, 300.0, 8)
    ff = Forcefield(s)
    ff.apply(s.pos)                      # lists sized from the density, built synchronously
    ff.set_params(list_capacity=16)      # the next rebuild runs asynchronously with tiny lists
    ff.upload_positions(s.pos)
    ff.md_init(m, v, dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
    st = ff.md_run(12)
    x, vg = ff.md_state()
    ff.close()
    assert st["rollbacks"] >= 1
    xo, vo, so = ob.OracleForcefield(s).md_run(s.pos, v, m, 12, dist_oh=0.1, dist_hh=g.SPC_DHH)
    assert np.abs(x - xo).max() <= 1e-5
    assert np.sqrt(((vg - vo) ** 2).sum() / (vo ** 2).sum()) <= 1e-4


def test_md_rollback_mid_period_keeps_the_schedule():
    """A call that starts inside a pairlist period (md_run(2), then md_run(11) with NSNB 4) whose
    lists overflow at the period's next rebuild: the block goes back to the period start, replays
    the two steps and runs again with grown lists.  Rebuilds stay at steps 1, 5, 9, ... from
    gr_md_init, so the trajectory equals, bit for bit, the same calls on lists that never overflow."""
    s = g.spc_water_system(1200, box=g.box_for_waters(1200), seed=33, rcutp=0.8, rcutl=1.2, nsnb=4)
    m = g.masses(s)
    v = g.maxwell_velocities(m, 300.0, 8)
    out = []
    for tiny in (False, True):
        ff = Forcefield(s)
        ff.upload_positions(s.pos)
        ff.md_init(m, v, dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
        ff.md_run(2)
        if tiny:
            ff.set_params(list_capacity=16)  # only the capacity: the current lists and schedule stay
        st = ff.md_run(11)
        out.append((ff.md_state(), st))
        ff.close()
    (xa, va), sa = out[0]
    (xb, vb), sb = out[1]
    assert sa["rollbacks"] == 0 and sb["rollbacks"] >= 1
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_md_trajectory_files(tmp_path):
    """Device MD written as ENERTRJ / FREEFORCERED frames and read back unchanged."""
    from gromos_nb import gromos_io as io
    s = g.spc_water_system(500, box=g.box_for_waters(500), seed=41, rcutp=0.8, rcutl=1.2, nsnb=5)
    m = g.masses(s)
    ff = Forcefield(s)
    ff.upload_positions(s.pos)
    ff.md_init(m, g.maxwell_velocities(m, 300.0, 9), dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH,
               temperature=300.0, tau=0.1)
    dof = 3 * s.topo.n_atoms - (s.topo.n_atoms - s.topo.n_solute_atoms)
    pe, pf = str(tmp_path / "md.tre"), str(tmp_path / "md.trf")
    kept = []
    with io.EnergyWriter(pe, "device MD") as we, io.ForceWriter(pf, "device MD") as wf:
        for k in range(4):
            st = ff.md_run(5)              # statistics of this call; the step count is kept here
            step = 5 * (k + 1)
            fr = io.md_energy_frame(0.002 * step, st["e_kin"], st["e_lj"], st["e_crf"], dof,
                                    volume=float(np.prod(s.box)))
            f = ff.result()["forces"]
            we.write_frame(fr)
            wf.write_frame(step, 0.002 * step, f)
            kept.append((fr, f, step))
    ff.close()
    back = io.read_energy_trajectory(pe)
    assert len(back) == 4
    for (fr, f, step), b in zip(kept, back):
        np.testing.assert_allclose(b.values(), fr.values(), rtol=1e-12)
        assert 0.0 < b.temperature < 1e4 and np.isfinite(b.total)
        np.testing.assert_allclose(io.read_forces_step(pf, step), f, atol=1e-9)
