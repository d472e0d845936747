"""Berendsen MD against the oracle, and temperature replica exchange over a batch."""
import numpy as np
import pytest

import oracle_binding as ob
from gromos_nb import generators as g
from gromos_nb.nonbonded import Forcefield
from gromos_nb.remd import ReplicaExchange

pytestmark = pytest.mark.gpu


def test_berendsen_md_vs_oracle():
    s = g.spc_water_system(600, box=g.box_for_waters(600), seed=51, rcutp=0.8, rcutl=1.0, nsnb=5)
    m = g.masses(s)
    v = g.maxwell_velocities(m, 300.0, 9)
    ff = Forcefield(s)
    ff.upload_positions(s.pos)
    ff.md_init(m, v, dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH, temperature=280.0, tau=0.05)
    st = ff.md_run(15)
    x, vg = ff.md_state()
    ff.close()
    xo, vo, so = ob.OracleForcefield(s).md_run(s.pos, v, m, 15, dist_oh=0.1, dist_hh=g.SPC_DHH,
                                               temperature=280.0, tau=0.05)
    assert np.abs(x - xo).max() <= 1e-5
    assert np.sqrt(((vg - vo) ** 2).sum() / (vo ** 2).sum()) <= 1e-4
    assert abs(st["e_kin"] - so["e_kin"]) <= 1e-5 * so["e_kin"]


def replicas(n, T):
    s = g.spc_water_system(400, box=g.box_for_waters(400), seed=52, rcutp=0.8, rcutl=1.0, nsnb=5)
    m = g.masses(s)
    out = []
    for k in range(n):
        ff = Forcefield(s)
        ff.upload_positions(s.pos)
        ff.md_init(m, g.maxwell_velocities(m, T[k], 100 + k), dt=0.002, settle=True, dist_oh=0.1,
                   dist_hh=g.SPC_DHH, temperature=T[k], tau=0.1)
        out.append(ff)
    return out


def test_replica_exchange_reproducible_and_consistent():
    T = [300.0, 305.0, 310.0, 315.0]
    finals = []
    for rep in range(2):
        rs = replicas(4, T)
        rx = ReplicaExchange(rs, T, exchange_interval=5, seed=11)
        rx.run(40)
        st = rx.statistics()
        assert sorted(st["temperatures"]) == T                      # a permutation of the ladder
        assert sum(st["attempts"]) == 4 * 1 + 4 * 2                  # 8 rounds: odd (1 pair) and even (2 pairs) alternate
        assert all(0 <= a <= b for a, b in zip(st["accepts"], st["attempts"]))
        finals.append((st, [r.md_state()[0] for r in rs]))
        rx.close()
        for r in rs:
            r.close()
    assert finals[0][0] == finals[1][0]
    assert all(np.array_equal(a, b) for a, b in zip(finals[0][1], finals[1][1]))


def test_temperature_change_keeps_batch_graphs_and_matches_standalone():
    """The bath temperature is read from device memory by the MD step kernel, so an
    exchange (gr_md_set_temperature) between batch steps records no graph again (the
    members' own launch counters, which only recording advances, stay put) and the
    trajectories equal standalone runs with the same temperature change, bit for bit."""
    from gromos_nb.nonbonded import Batch

    T = [300.0, 330.0]
    rs = replicas(2, T)
    b = Batch()
    for r in rs:
        b.add(r)
    b.md_run(7)
    before = [r.launches() for r in rs]
    rs[0].md_set_temperature(330.0, rescale_velocities=False)
    rs[1].md_set_temperature(300.0, rescale_velocities=False)
    b.md_run(8)
    assert [r.launches() for r in rs] == before
    got = [r.md_state() for r in rs]
    b.close()
    for r in rs:
        r.close()
    alone = replicas(2, T)
    alone[0].md_run(7)
    alone[1].md_run(7)
    alone[0].md_set_temperature(330.0, rescale_velocities=False)
    alone[1].md_set_temperature(300.0, rescale_velocities=False)
    for r, (x, v) in zip(alone, got):
        r.md_run(8)
        xa, va = r.md_state()
        assert np.array_equal(x, xa) and np.array_equal(v, va)
        r.close()
