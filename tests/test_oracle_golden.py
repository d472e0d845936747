"""Pins the FP64 oracle to the gromosXX reference runs shipped with gromos-rs.

Step-0 LJ and CRF energy totals must agree to the fixtures' 10 significant
digits (relative 1e-8, the tolerance the reference's own harness uses,
crates/gromos-md/tests/test_gromosXX_references.rs:22-25); step-0 forces must
agree to 1e-6 kJ/(mol nm) wherever the fixture has no covalent energy (then
FREEFORCERED is the pure nonbonded force); the per-energy-group nonbonded
block of ch4_water_fep pins the group attribution.
"""
import numpy as np
import pytest

import oracle_binding as ob
from golden_loader import FIXTURE_NAMES, load_fixture


@pytest.mark.parametrize("name", FIXTURE_NAMES)
def test_step0_energies(name):
    s, ex = load_fixture(name)
    if ex["reference_ignores"]:
        pytest.skip(ex["reference_ignores"])
    r = ob.OracleForcefield(s).apply()
    for key in ("e_lj", "e_crf"):
        want = ex[key]
        assert abs(r[key] - want) <= 1e-8 * max(abs(want), 1e-12) + 1e-12, (key, r[key], want)


@pytest.mark.parametrize("name", FIXTURE_NAMES)
def test_step0_forces(name):
    s, ex = load_fixture(name)
    if ex["e_covalent"] != 0.0:
        pytest.skip("fixture forces include bonded terms")
    if ex["reference_ignores"]:
        pytest.skip(ex["reference_ignores"])
    r = ob.OracleForcefield(s).apply()
    assert r["forces"].shape == ex["forces"].shape
    np.testing.assert_allclose(r["forces"], ex["forces"], atol=1e-6, rtol=0)


def test_energy_group_split_fep():
    s, ex = load_fixture("ch4_water_fep")
    r = ob.OracleForcefield(s).apply()
    g = ex["nonbonded_groups"]  # rows (1,1), (1,2), (2,2); columns LJ, CRF, ...
    got_lj = [r["egroup_lj"][0, 0], r["egroup_lj"][0, 1], r["egroup_lj"][1, 1]]
    got_crf = [r["egroup_crf"][0, 0], r["egroup_crf"][0, 1], r["egroup_crf"][1, 1]]
    np.testing.assert_allclose(got_lj, g[:, 0], rtol=1e-8, atol=1e-9)
    np.testing.assert_allclose(got_crf, g[:, 1], rtol=1e-8, atol=1e-9)
    assert abs(sum(got_lj) - r["e_lj"]) < 1e-8 * abs(r["e_lj"])


def test_lambda_params_known_answers():
    """perturbed.rs:715-745: λ = 0.5, n = 2."""
    import ctypes as C
    out = np.zeros(17)
    ob.lib().orc_lambda_params(0.5, 0.5, 0.5, 0.5, 1.0, 1.0, 1.0, 1.0, 2, out.ctypes.data_as(C.POINTER(C.c_double)))
    a_lj_n, b_lj_n, _, _, a_lj_n1, b_lj_n1 = out[:6]
    assert b_lj_n == 0.25 and a_lj_n == 0.25
    assert b_lj_n1 == 0.5 and a_lj_n1 == 0.5
    assert out[11] == 0.25 and out[10] == 0.25  # b_ljs2, a_ljs2


def test_crf_parameters():
    """CRFParameters::new(1.4, 1, 61, 0) closed form (params.rs:78-96)."""
    c = ob.crf_params(1.4, 1.0, 61.0, 0.0)
    crf = 2.0 * (1.0 - 61.0) / (1.0 + 2.0 * 61.0)
    assert np.isclose(c[2], crf / 1.4**3, rtol=1e-15)
    assert np.isclose(c[1], crf / 1.4**3 / 2, rtol=1e-15)
    assert np.isclose(c[0], (1 - crf / 2) / 1.4, rtol=1e-15)


@pytest.mark.parametrize("name", ["water_216_box", "water_1000_spc_gridcell", "ch4_water_fep", "nacl_water_box"])
def test_cell_list_matches_standard(name):
    """pairlist.rs:1121-1302: Standard and CellList give the same pair SET."""
    s, _ = load_fixture(name)
    a = ob.pairlist(s, algorithm=0)
    b = ob.pairlist(s, algorithm=2)
    for k in range(4):
        sa = set(map(tuple, np.sort(a[k], axis=1).tolist()))
        sb = set(map(tuple, np.sort(b[k], axis=1).tolist()))
        assert sa == sb, (k, len(sa), len(sb))


@pytest.mark.parametrize("case", ["spc1000_single_range", "solute_small_box", "twin_range_solute"])
def test_cell_list_matches_standard_synthetic(case):
    """The same set equality on the synthetic shapes the parity tests use: 2 cells per axis (the
    de-duplicated neighbour path), a box below twice the cutoff with a solute (per-atom images),
    and a twin-range solvated solute."""
    from gromos_nb import generators
    if case == "spc1000_single_range":
        s = generators.config1_spc1000()
    elif case == "solute_small_box":
        s = generators.solvated_solute_system(300, 40, seed=1003, rc=1.4)
    else:
        s = generators.solvated_solute_system(900, 60, seed=1005, rc=0.9)
        s.params.rcutp = 0.6
    a = ob.pairlist(s, algorithm=0)
    b = ob.pairlist(s, algorithm=2)
    for k in range(4):
        sa = set(map(tuple, np.sort(a[k], axis=1).tolist()))
        sb = set(map(tuple, np.sort(b[k], axis=1).tolist()))
        assert sa == sb, (case, k, len(sa), len(sb))
    assert sum(len(x) for x in a) > 0


@pytest.mark.parametrize("case,lam,nlam", [("ch4_water_fep", 0.2, 1), ("ch4_water_fep", 0.5, 1),
                                           ("ch4_water_fep", 0.8, 1), ("solute30", 0.1, 1),
                                           ("solute30", 0.7, 2), ("solute30_twin", 0.4, 3)])
def test_dhdl_is_the_lambda_derivative_of_the_energy(case, lam, nlam):
    """The fixtures hold no dH/dlambda, but they pin the energy at lambda 0.5.  The oracle's analytic
    dH/dlambda (perturbed.rs:123-266, 395-605) must equal the central difference of its own total
    nonbonded energy in lambda, for NLAM 1-3, single and twin range."""
    import copy
    from gromos_nb import generators
    if case == "ch4_water_fep":
        s, _ = load_fixture(case)
    else:
        s = generators.solvated_solute_system(300, 30, seed=1004, perturbed=True, lam=0.5, rc=1.2)
        if case == "solute30_twin":
            s.params.rcutp = 0.8
    s.params.nlam = nlam
    h = 1e-5
    res = []
    for l in (lam - h, lam, lam + h):
        t = copy.deepcopy(s)
        t.params.lam = l
        res.append(ob.OracleForcefield(t).apply(t.pos))
    numeric = ((res[2]["e_lj"] + res[2]["e_crf"]) - (res[0]["e_lj"] + res[0]["e_crf"])) / (2 * h)
    assert abs(res[1]["dhdl"] - numeric) <= 1e-6 * max(abs(numeric), 1.0), (res[1]["dhdl"], numeric)


def _strain_derivative(s, a, b, periodic, h=1e-6):
    """-dE/d(eps_ab) by central differences: positions x -> (I + eps) x, the box scaled with them."""
    import copy
    e = []
    for sign in (-1.0, 1.0):
        m = np.eye(3)
        m[a, b] += sign * h
        t = copy.deepcopy(s)
        t.pos = s.pos @ m.T
        if periodic:
            t.box = s.box * np.diag(m)
        r = ob.OracleForcefield(t).apply(t.pos)
        e.append(r["e_lj"] + r["e_crf"])
    return -(e[1] - e[0]) / (2 * h)


def test_virial_is_the_strain_derivative_in_vacuum():
    """No fixture holds a virial, but the energy is pinned.  For pair forces the virial
    sum r_a F_b (innerloops.rs:169-210, forcefield.rs:953-1000) is -dE/d(eps_ab) under a homogeneous
    strain; in vacuum every component can be strained.  Solute-only fixture (the solvent's
    intramolecular RF terms carry energy without force, excluded.rs:25-112)."""
    import dataclasses
    s, _ = load_fixture("water_216_box")
    s.params = dataclasses.replace(s.params, boundary=0)
    w = np.asarray(ob.OracleForcefield(s).apply(s.pos)["virial"]).reshape(3, 3)
    d = np.array([[_strain_derivative(s, a, b, periodic=False) for b in range(3)] for a in range(3)])
    assert np.abs(w - d).max() <= 1e-6 * np.abs(w).max(), (w, d)


@pytest.mark.parametrize("name", ["water_216_box", "water_1000_spc_gridcell"])
def test_virial_diagonal_is_the_box_strain_derivative(name):
    """Periodic solute-only fixtures (single and twin range): scaling one box edge with the
    positions gives the diagonal virial element."""
    s, _ = load_fixture(name)
    w = np.asarray(ob.OracleForcefield(s).apply(s.pos)["virial"]).reshape(3, 3)
    for a in range(3):
        d = _strain_derivative(s, a, a, periodic=True)
        assert abs(w[a, a] - d) <= 1e-6 * abs(w[a, a]), (a, w[a, a], d)
