"""Batches: many systems stepped together must give each member exactly its
standalone results (bitwise: fixed-point sums, same kernels per member).

Covers uneven REMD-like members (water boxes of different sizes, one with a
solute), members that join and leave between calls (continuous batching),
FEP lambda windows evaluated together, and the batch against the oracle.
"""
import numpy as np
import pytest

import oracle_binding as ob
from gromos_nb import generators as g
from gromos_nb.nonbonded import Batch, Forcefield

pytestmark = pytest.mark.gpu


def member(s, seed, T=300.0):
    ff = Forcefield(s)
    ff.upload_positions(s.pos)
    m = g.masses(s)
    ff.md_init(m, g.maxwell_velocities(m, T, seed), dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
    return ff


def systems():
    return [
        g.spc_water_system(300, box=g.box_for_waters(300), seed=41, rcutp=0.8, rcutl=1.0, nsnb=5),
        g.spc_water_system(1100, box=g.box_for_waters(1100), seed=42, rcutp=0.8, rcutl=1.0, nsnb=5),
        g.solvated_solute_system(500, 40, seed=43, rc=1.0, nsnb=5),
        g.spc_water_system(700, box=g.box_for_waters(700), seed=44, rcutp=0.8, rcutl=1.0, nsnb=5),
    ]


def standalone(s, seed, n):
    ff = member(s, seed)
    ff.md_run(n)
    out = ff.md_state()
    ff.close()
    return out


def test_batch_md_bit_identical_to_standalone():
    sy = systems()
    b = Batch()
    ffs = [member(s, 100 + k) for k, s in enumerate(sy)]
    for ff in ffs:
        b.add(ff)
    b.md_run(5)
    b.md_run(8)
    for k, (s, ff) in enumerate(zip(sy, ffs)):
        x, v = ff.md_state()
        xr, vr = standalone(s, 100 + k, 13)
        assert np.array_equal(x, xr) and np.array_equal(v, vr), k
        assert ff.md_stats()["steps"] == 13
    b.close()
    for ff in ffs:
        ff.close()


def test_batch_members_join_and_leave():
    """Continuous batching: a member joins after 3 steps, another leaves after 7."""
    sy = systems()
    b = Batch()
    a, c, d = member(sy[0], 1), member(sy[1], 2), member(sy[2], 3)
    b.add(a)
    b.add(c)
    b.md_run(3)
    b.add(d)                 # joins at batch step 3 with its own rebuild phase
    b.md_run(4)
    b.remove(c)              # leaves after 7 steps
    b.md_run(5)
    xa, va = a.md_state()
    xc, vc = c.md_state()
    xd, vd = d.md_state()
    for (x, v), (s, seed, n) in zip([(xa, va), (xc, vc), (xd, vd)], [(sy[0], 1, 12), (sy[1], 2, 7), (sy[2], 3, 9)]):
        xr, vr = standalone(s, seed, n)
        assert np.array_equal(x, xr) and np.array_equal(v, vr)
    b.close()
    for ff in (a, c, d):
        ff.close()


def test_batch_fep_windows_eval():
    """lambda windows of one perturbed system evaluated together == one by one == oracle."""
    lams = [0.0, 0.25, 0.5, 0.75, 1.0]
    base = g.solvated_solute_system(600, 30, seed=1004, perturbed=True, rc=1.2)
    b = Batch()
    ffs = []
    for lam in lams:
        base.params.lam = lam
        ff = Forcefield(base)
        ff.upload_positions(base.pos)
        b.add(ff)
        ffs.append(ff)
    b.eval()
    for lam, ff in zip(lams, ffs):
        r = ff.result()
        base.params.lam = lam
        alone = Forcefield(base)
        a = alone.apply(base.pos)
        assert np.array_equal(r["forces"], a["forces"])
        assert r["e_lj"] == a["e_lj"] and r["e_crf"] == a["e_crf"] and r["dhdl"] == a["dhdl"]
        o = ob.OracleForcefield(base).apply(base.pos)
        assert abs(r["dhdl"] - o["dhdl"]) <= 1e-5 * max(abs(o["dhdl"]), 1.0)
        alone.close()
    b.close()
    for ff in ffs:
        ff.close()


def test_batch_launch_accounting():
    sy = systems()[:2]
    b = Batch()
    ffs = [member(s, 7 + k) for k, s in enumerate(sy)]
    for ff in ffs:
        b.add(ff)
    ms = b.md_run(10)
    assert ms > 0.0
    assert b.launches() >= 10 * 2 * 4   # at least prep/water/finalize/md per member and step
    b.close()
    for ff in ffs:
        ff.close()


def test_autotune_picks_a_variant_and_keeps_results():
    s = g.spc_water_system(2000, box=g.box_for_waters(2000), seed=45, rcutp=0.8, rcutl=1.2, nsnb=5)
    ff = Forcefield(s)
    ff.upload_positions(s.pos)
    r = ff.autotune(periods=1)
    assert (r["water_layout"], r["cluster_size"]) in [(2, 4), (2, 8), (1, 4), (3, 4)]
    assert all(c["ms_per_step"] > 0 for c in r["candidates"])
    a = ff.apply(s.pos)
    o = ob.OracleForcefield(s).apply(s.pos)
    d = a["forces"] - o["forces"]
    assert np.sqrt((d * d).sum() / (o["forces"] ** 2).sum()) <= 1e-5
    ff.close()
    b = Batch()
    ffs = [member(x, 50 + k) for k, x in enumerate(systems()[:3])]
    for f in ffs:
        b.add(f)
    rb = b.autotune(periods=1)
    assert len(rb["candidates"]) == 4
    b.md_run(6)
    for k, f in enumerate(ffs):
        x, v = f.md_state()
        xr, vr = standalone_variant(systems()[k], 50 + k, 6, rb["water_layout"], rb["cluster_size"])
        assert np.array_equal(x, xr) and np.array_equal(v, vr)
    b.close()
    for f in ffs:
        f.close()


def test_autotune_cache_reuses_the_choice(tmp_path):
    """A second autotune of the same system shape with the same cache file applies the stored
    variant without timing (no candidate times), and the forces still match the oracle."""
    cache = str(tmp_path / "tuning.json")
    s = g.spc_water_system(1500, box=g.box_for_waters(1500), seed=46, rcutp=0.8, rcutl=1.2, nsnb=5)
    ff = Forcefield(s)
    ff.upload_positions(s.pos)
    r1 = ff.autotune(periods=1, cache=cache)
    ff.close()
    s2 = g.spc_water_system(1500, box=g.box_for_waters(1500), seed=47, rcutp=0.8, rcutl=1.2, nsnb=5)
    ff = Forcefield(s2)
    ff.upload_positions(s2.pos)
    r2 = ff.autotune(periods=1, cache=cache)
    assert r1["cached"] is False and r2["cached"] is True
    assert (r2["water_layout"], r2["cluster_size"]) == (r1["water_layout"], r1["cluster_size"])
    a = ff.apply(s2.pos)
    o = ob.OracleForcefield(s2).apply(s2.pos)
    d = a["forces"] - o["forces"]
    assert np.sqrt((d * d).sum() / (o["forces"] ** 2).sum()) <= 1e-5
    ff.close()
    b = Batch()
    ffs = [member(x, 60 + k) for k, x in enumerate(systems()[:2])]
    for f in ffs:
        b.add(f)
    rb1 = b.autotune(periods=1, cache=cache)
    rb2 = b.autotune(periods=1, cache=cache)
    assert rb1["cached"] is False and rb2["cached"] is True
    b.md_run(5)
    for k, f in enumerate(ffs):
        x, v = f.md_state()
        xr, vr = standalone_variant(systems()[k], 60 + k, 5, rb2["water_layout"], rb2["cluster_size"])
        assert np.array_equal(x, xr) and np.array_equal(v, vr)
    b.close()
    for f in ffs:
        f.close()


def standalone_variant(s, seed, n, layout, width):
    ff = Forcefield(s, cluster_size=width, water_layout=layout)
    ff.upload_positions(s.pos)
    m = g.masses(s)
    ff.md_init(m, g.maxwell_velocities(m, 300.0, seed), dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
    ff.md_run(n)
    out = ff.md_state()
    ff.close()
    return out


def test_member_close_leaves_batch():
    """Closing a member removes it from its batch first; the C ABI refuses to destroy a member."""
    from gromos_nb import _lib
    sy = systems()[:2]
    b = Batch()
    a, c = member(sy[0], 1), member(sy[1], 2)
    b.add(a)
    b.add(c)
    assert _lib.lib().gr_ctx_destroy(a.handle) == _lib.GR_ERR_STATE
    a.close()                      # leaves the batch, then is destroyed
    assert len(b) == 1
    b.md_run(4)
    x, v = c.md_state()
    xr, vr = standalone(sy[1], 2, 4)
    assert np.array_equal(x, xr) and np.array_equal(v, vr)
    b.close()
    c.close()


def test_batch_graphs_across_joins_and_leaves():
    """Batch graphs replayed over several pairlist periods, then recorded again after a join (the new
    member mid-way through the others' periods) and after a leave; every member's trajectory is its
    standalone one, bit for bit."""
    sy = systems()
    b = Batch()
    a, c, d = member(sy[0], 11), member(sy[1], 12), member(sy[3], 13)
    b.add(a)
    b.add(c)
    b.md_run(12)
    b.add(d)                 # joins at batch step 12 with its own rebuild phase
    b.md_run(13)
    b.remove(a)
    b.md_run(3)
    for ff, (s, seed, n) in zip((a, c, d), [(sy[0], 11, 25), (sy[1], 12, 28), (sy[3], 13, 16)]):
        x, v = ff.md_state()
        xr, vr = standalone(s, seed, n)
        assert np.array_equal(x, xr) and np.array_equal(v, vr), seed
    b.close()
    for ff in (a, c, d):
        ff.close()


def test_batch_member_rollback_after_list_overflow():
    """A member's rebuild inside a batch step overflows its (deliberately tiny) lists: that member is
    rolled back to its period start and re-run alone with grown lists, the other members go on; its
    trajectory is the oracle's and the others' are their standalone ones."""
    s = g.spc_water_system(1200, box=g.box_for_waters(1200), seed=33, rcutp=0.8, rcutl=1.2, nsnb=5)
    m = g.masses(s)
    v = g.maxwell_velocities(m, 300.0, 8)
    small = Forcefield(s)
    small.apply(s.pos)                   # lists sized from the density, built synchronously
    small.set_params(list_capacity=16)   # later rebuilds run asynchronously with tiny lists
    small.upload_positions(s.pos)
    small.md_init(m, v, dt=0.002, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
    sy = systems()[:2]
    others = [member(x, 60 + k) for k, x in enumerate(sy)]
    b = Batch()
    for ff in [small] + others:
        b.add(ff)
    b.md_run(12)
    assert small.md_stats()["rollbacks"] >= 1
    x, vg = small.md_state()
    xo, vo, _ = ob.OracleForcefield(s).md_run(s.pos, v, m, 12, dist_oh=0.1, dist_hh=g.SPC_DHH)
    assert np.abs(x - xo).max() <= 1e-5
    assert np.sqrt(((vg - vo) ** 2).sum() / (vo ** 2).sum()) <= 1e-4
    for k, (sx, ff) in enumerate(zip(sy, others)):
        xx, vv = ff.md_state()
        xr, vr = standalone(sx, 60 + k, 12)
        assert np.array_equal(xx, xr) and np.array_equal(vv, vr), k
    b.close()
    for ff in [small] + others:
        ff.close()


def test_batch_phase_reports_the_members_period_step():
    """gr_batch_phase: members added together share a phase (their graphs are recorded once
    per distinct set of rebuilding members); a member added mid-period makes it -1, and both
    keep their standalone trajectories bit for bit."""
    sy = systems()[:2]
    b = Batch()
    assert b.phase()[0] == -1                      # empty
    a = member(sy[0], 201)
    b.add(a)
    assert b.phase() == (0, 5)
    b.md_run(3)
    assert b.phase() == (3, 5)
    assert b.record_stats()[0] == 2                # a rebuilds at one phase: two distinct step graphs
    c = member(sy[1], 202)
    b.add(c)
    assert b.phase() == (-1, 5)                    # a at step 3 of its period, c at step 0
    b.md_run(9)
    n_graphs, seconds = b.record_stats()
    assert n_graphs == 5 and seconds > 0.0         # + {c}, {a}, {} rebuilding: three more
    xa, va = a.md_state()
    xc, vc = c.md_state()
    b.close()
    for ff in (a, c):
        ff.close()
    for s, seed, n, (x, v) in ((sy[0], 201, 12, (xa, va)), (sy[1], 202, 9, (xc, vc))):
        xr, vr = standalone(s, seed, n)
        assert np.array_equal(x, xr) and np.array_equal(v, vr)
