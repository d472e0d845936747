"""Pins of the oracle's 1-4, perturbed-pair and MD terms to the gromosXX reference runs.

* 1-4 interactions (one_four_interaction_loop, excluded.rs:131-206): aladip_vacuum and
  butane_vacuum step-0 LJ / CRF totals include every INE14 pair (relative 1e-8, through
  test_oracle_golden.test_step0_energies); their step-0 forces include bonded terms, so the
  nonbonded forces are pinned as minus the gradient of the fixture-pinned energy.
* Perturbed 1-4 and PERTATOMPAIR corrections (perturbed.rs:517-707): aladip_vacuum_fep.
  gromos-rs's own harness ignores this fixture as a known FEP mismatch
  (crates/gromos-md/tests/test_gromosXX_references.rs:562).  One cause is the soft-core
  reaction-field constant of perturbed_lj_crf_interaction (perturbed.rs:186-187):
  crf_2cut3i / cut2soft^(3/2) divides by the cutoff cubed a second time (the excluded
  correction scales by (cut2 / cut2soft)^(3/2) instead, perturbed.rs:476-477), so the pair
  and 1-4 corrections of a charged perturbed atom do not vanish at lambda 0.  The oracle keeps
  the reference's formula; the tests pin it at lambda 0 against the unperturbed fixture plus
  that closed-form term, and at lambda 0.125 through the lambda derivative and the gradient.
* The PERTATOMPAIR correction adds its reaction-field change to the forces and to dH/dlambda
  but not to E_CRF (forcefield.rs:908-924 adds delta_e_lj only); the oracle does the same and
  the tests state the resulting offsets exactly.
* MD (leap-frog, leap_frog.rs:37-148, and SETTLE, constraints.rs:815-1010): every frame of
  the nacl_1water_settle trajectory (9-decimal output) to 1e-9 nm, the fixture's own position
  tolerance (its input.toml), and the final velocities to 1e-9 nm/ps.
"""
import copy

import numpy as np
import pytest

import oracle_binding as ob
from golden_loader import load_fixture


def _energy(s, pos=None):
    r = ob.OracleForcefield(s).apply(s.pos if pos is None else pos)
    return r["e_lj"] + r["e_crf"], r


def _numeric_gradient(s, h=1e-6):
    g = np.zeros_like(s.pos)
    for a in range(s.pos.shape[0]):
        for k in range(3):
            p = s.pos.copy()
            p[a, k] += h
            ep, _ = _energy(s, p)
            p[a, k] -= 2 * h
            em, _ = _energy(s, p)
            g[a, k] = (ep - em) / (2 * h)
    return g


@pytest.mark.parametrize("name", ["aladip_vacuum", "butane_vacuum"])
def test_one_four_fixtures_have_one_four_pairs(name):
    s, ex = load_fixture(name)
    t = s.topo.normalized()
    assert len(t.o14) > 0 and ex["reference_ignores"] is None


@pytest.mark.parametrize("name", ["aladip_vacuum", "butane_vacuum"])
def test_one_four_forces_are_the_energy_gradient(name):
    """Vacuum solute with exclusions and 1-4 pairs: F = -dE/dx for every atom (the energy is
    pinned to the fixture; no solvent, so every term's force is its energy's gradient)."""
    s, _ = load_fixture(name)
    _, r = _energy(s)
    g = _numeric_gradient(s)
    scale = np.abs(r["forces"]).max()
    assert np.abs(r["forces"] + g).max() <= 1e-6 * scale, np.abs(r["forces"] + g).max()


def _crf(s):
    c = ob.crf_params(s.params.rcutl, s.params.epsilon, s.params.epsrf, s.params.kappa)
    return {"crf_cut": c[0], "crf_2cut3i": c[1], "crf_cut3i": c[2], "cutoff_sq": c[3]}


def _corrected_pairs(s):
    """Pairs the reference's pair and 1-4 corrections visit: listed pairs whose first atom is
    perturbed (perturbed.rs:324-333), 1-4 pairs with a perturbed atom (perturbed.rs:531-538)."""
    t = s.topo.normalized()
    pert = np.asarray(t.pert_idx) >= 0
    out = []
    for lst in ob.pairlist(s):
        out += [(int(i), int(j)) for i, j in lst if pert[i]]
    for i in range(t.n_atoms):
        out += [(i, int(j)) for j in t.o14[t.o14_off[i]:t.o14_off[i + 1]] if j > i and (pert[i] or pert[j])]
    return out


def test_perturbed_fixture_at_lambda0_is_state_a_plus_the_reference_crf_term():
    """aladip_vacuum_fep at lambda 0 against the gromosXX aladip_vacuum energies (same topology and
    configuration, state A = the unperturbed topology): E_LJ equal to 1e-8; E_CRF offset by the
    reference's soft-core constant, sum over corrected pairs of q_i q_j f crf_2cut3i r^2 (1 - R^-3)."""
    s, ex = load_fixture("aladip_vacuum_fep")
    a, exa = load_fixture("aladip_vacuum")
    assert ex["reference_ignores"] and "test_gromosXX_references.rs" in ex["reference_ignores"]
    t = copy.deepcopy(s)
    t.params.lam = 0.0
    _, r = _energy(t)
    assert abs(r["e_lj"] - exa["e_lj"]) <= 1e-8 * abs(exa["e_lj"])
    c = _crf(t)
    R3 = c["cutoff_sq"] ** 1.5
    tn = t.topo.normalized()
    q, f = tn.charge, tn.four_pi_eps_i
    de = 0.0
    for i, j in _corrected_pairs(t):
        d = t.pos[i] - t.pos[j]
        de += q[i] * q[j] * f * c["crf_2cut3i"] * (d @ d) * (1.0 - 1.0 / R3)
    assert abs(de) > 1e-3                      # the term is there: charged perturbed atoms
    assert abs((r["e_crf"] - exa["e_crf"]) - de) <= 1e-8 * abs(exa["e_crf"]), (r["e_crf"] - exa["e_crf"], de)


def _pair_crf_reg(s):
    """Reaction-field energy and scalar force of each PERTATOMPAIR at the regular charges
    (perturbed.rs:664-666)."""
    t = s.topo.normalized()
    c = _crf(s)
    out = []
    for i, j in zip(t.pp_i, t.pp_j):
        d = s.pos[i] - s.pos[j]
        r2 = d @ d
        qp = t.charge[i] * t.charge[j] * t.four_pi_eps_i
        e = qp * (1.0 / np.sqrt(r2) - c["crf_2cut3i"] * r2 - c["crf_cut"])
        fs = qp * (1.0 / np.sqrt(r2) / r2 + c["crf_cut3i"])
        out.append((int(i), int(j), d, e, fs))
    return out


def _fep_fixture(variant):
    """aladip_vacuum_fep as converted, or with its PERTATOMPAIR's uncharged first atom (a CB,
    sequence number 7) given a charge of +0.15 e, so that the pair's reaction-field term is not
    zero (the fixture's pair has no reaction-field energy)."""
    s, ex = load_fixture("aladip_vacuum_fep")
    if variant == "charged_pair":
        i = int(s.topo.pp_i[0])
        assert s.topo.charge[i] == 0.0 and s.topo.pert_idx[i] < 0
        s.topo.charge = s.topo.charge.copy()
        s.topo.charge[i] = 0.15
    return s, ex


@pytest.mark.parametrize("variant", ["fixture", "charged_pair"])
@pytest.mark.parametrize("lam,nlam", [(0.125, 1), (0.125, 2), (0.6, 1)])
def test_perturbed_fixture_dhdl_is_the_lambda_derivative(variant, lam, nlam):
    """dH/dlambda of aladip_vacuum_fep (pair, self, excluded, 1-4 and PERTATOMPAIR corrections)
    equals d(E_LJ + E_CRF)/dlambda plus the PERTATOMPAIR reaction-field term the energy omits:
    -n (1-lambda)^(n-1) e_crf (state B of the pair is absent)."""
    s, _ = _fep_fixture(variant)
    s.params.nlam = nlam
    h = 1e-6
    e = []
    for l in (lam - h, lam + h):
        t = copy.deepcopy(s)
        t.params.lam = l
        e.append(_energy(t)[0])
    t = copy.deepcopy(s)
    t.params.lam = lam
    _, r = _energy(t)
    numeric = (e[1] - e[0]) / (2 * h)
    omitted = sum(-nlam * (1.0 - lam) ** (nlam - 1) * ec for _, _, _, ec, _ in _pair_crf_reg(t))
    assert (abs(omitted) > 1e-3) == (variant == "charged_pair")
    assert abs(r["dhdl"] - (numeric + omitted)) <= 1e-6 * max(abs(r["dhdl"]), 1.0), (r["dhdl"], numeric, omitted)


@pytest.mark.parametrize("variant", ["fixture", "charged_pair"])
def test_perturbed_fixture_forces_are_the_gradient_plus_the_pair_crf_term(variant):
    """At lambda 0.125 the oracle's forces equal -dE/dx except for the PERTATOMPAIR reaction-field
    change, r ((1-lambda)^n - 1) f_crf, which enters the forces but not E_CRF."""
    s, _ = _fep_fixture(variant)
    _, r = _energy(s)
    g = _numeric_gradient(s)
    lam, n = s.params.lam, s.params.nlam
    extra = np.zeros_like(s.pos)
    for i, j, d, _, fs in _pair_crf_reg(s):
        df = d * (((1.0 - lam) ** n - 1.0) * fs)
        extra[i] += df
        extra[j] -= df
    scale = np.abs(r["forces"]).max()
    assert (np.abs(extra).max() > 1e-3 * scale) == (variant == "charged_pair")
    assert np.abs(r["forces"] + g - extra).max() <= 1e-6 * scale


def test_settle_trajectory_matches_gromosxx():
    """nacl_1water_settle: leap-frog + SETTLE, no bath coupling (TAU -1), 10 steps of 2 fs.
    Every written frame to 1e-9 nm; after the last step, positions and velocities of
    expected/final.conf to 1e-9."""
    s, ex = load_fixture("nacl_1water_settle")
    md = ex["md"]
    assert md["bath_tau"] < 0
    cons = {(i, j): d for i, j, d in md["solvent_constraints"]}
    orc = ob.OracleForcefield(s)
    x, v = s.pos.copy(), md["vel"].copy()
    steps, frames = list(md["traj_steps"]), md["traj_pos"]
    assert steps[0] == 0 and np.abs(frames[0] - x).max() < 1e-9
    done = 0
    for k in range(1, len(steps)):
        x, v, st = orc.md_run(x, v, md["mass"], steps[k] - done, dt=md["dt"], dist_oh=cons[(0, 1)],
                              dist_hh=cons[(1, 2)], tau=-1.0)
        done = steps[k]
        assert st["settle_failures"] == 0
        assert np.abs(x - frames[k]).max() <= 1e-9, (steps[k], np.abs(x - frames[k]).max())
    x, v, st = orc.md_run(x, v, md["mass"], md["nstlim"] - done, dt=md["dt"], dist_oh=cons[(0, 1)],
                          dist_hh=cons[(1, 2)], tau=-1.0)
    orc.close()
    assert np.abs(x - md["final_pos"]).max() <= 1e-9
    assert np.abs(v - md["final_vel"]).max() <= 1e-9, np.abs(v - md["final_vel"]).max()
