"""GPU parity: the CUDA path through the C ABI against the FP64 oracle.

* Pairlist: the four reference lists (solute_short, solute_long,
  solvent_short, solvent_long) must be IDENTICAL as sorted atom-pair sets
  (bit-exact; the reference's own cell-list-vs-standard check,
  pairlist.rs:1121-1302, compares the same sets).
* Forces: RMS relative error sqrt(sum|dF|^2 / sum|F|^2) <= 1e-5 for the
  fixed-point kernel (the path's accuracy target), <= 1e-4 for the plain FP32 kernel;
  max relative error max|dF_i| / max(|F_i|, 1e-3 RMS|F|) <= 1e-3.
* Energies (per group and totals) and the virial: relative 1e-5 of the
  largest magnitude in the set (FP32 pair arithmetic).
* dH/dlambda: relative 1e-5 (FP64 perturbation kernels).
"""
import dataclasses

import numpy as np
import pytest

import oracle_binding as ob
from golden_loader import load_fixture
from gromos_nb import generators
from gromos_nb.nonbonded import Forcefield

pytestmark = pytest.mark.gpu

FIXTURES = ["water_216_box", "water_1000_spc_gridcell", "ch4_water_fep", "nacl_water_box",
            "water_3_box_twinrange", "water_10_box", "nacl_3water_box", "nacl_pair_box",
            "aladip_vacuum", "butane_vacuum", "aladip_vacuum_fep", "nacl_1water_settle"]


def sorted_pairs(a):
    a = np.asarray(a, dtype=np.int64).reshape(-1, 2)
    if a.size == 0:
        return a
    return a[np.lexsort((a[:, 1], a[:, 0]))]


def force_errors(f, ref):
    df = f - ref
    rms = float(np.sqrt((df * df).sum() / max((ref * ref).sum(), 1e-300)))
    mag = np.linalg.norm(ref, axis=1)
    floor = 1e-3 * np.sqrt((mag ** 2).mean())
    mx = float((np.linalg.norm(df, axis=1) / np.maximum(mag, floor)).max())
    return rms, mx


def rel(a, b, scale=None):
    s = scale if scale is not None else max(abs(b), 1e-12)
    return abs(a - b) / s


def check_pairlist(s):
    ff = Forcefield(s, kernel="fixed")
    ff.upload_positions(s.pos)
    ff.build_pairlist()
    got = ff.pairlist_lists()
    ref = ob.pairlist(s, algorithm=0 if s.topo.n_atoms < 4000 else 2)
    for k in range(4):
        g, r = sorted_pairs(got[k]), sorted_pairs(ref[k])
        assert g.shape == r.shape, (s.name, k, g.shape, r.shape)
        assert np.array_equal(g, r), (s.name, k)
    ff.close()


@pytest.mark.parametrize("name", FIXTURES)
def test_pairlist_bit_exact_fixtures(name):
    s, _ = load_fixture(name)
    check_pairlist(s)


def test_pairlist_bit_exact_spc1000():
    check_pairlist(generators.config1_spc1000())


def test_pairlist_bit_exact_solute_small_box():
    # box < 2 * cutoff: one cell per axis, per-atom images for solute pairs
    check_pairlist(generators.solvated_solute_system(500, 200, seed=1003, rc=1.4))


def test_pairlist_bit_exact_spc30000_twin_range():
    check_pairlist(generators.config2_spc30000())


def test_many_cells_sparse_box():
    """3000 waters in a 12 nm box with a 0.9 nm cutoff: 13^3 = 2197 cells, most nearly empty,
    so the cell and cluster scans take more than one pass of their block (2048 cells each)."""
    s = generators.spc_water_system(3000, 12.0, 7, rcutp=0.9, rcutl=0.9, epsrf=61.0, nsnb=5, name="sparse3000")
    assert int(12.0 / 0.9) ** 3 > 2048
    check_pairlist(s)
    compare_eval(s, steps=2, move=0.002)


def compare_eval(s, kernel="fixed", steps=1, tol_rms=1e-5, tol_e=1e-5, move=0.0, seed=0, cluster_size=0,
                 layout=0, list_capacity=0):
    ff = Forcefield(s, kernel=kernel, cluster_size=cluster_size, water_layout=layout, list_capacity=list_capacity)
    orc = ob.OracleForcefield(s)
    rng = np.random.default_rng(seed)
    pos = s.pos.copy()
    worst = 0.0
    for step in range(steps):
        r = ff.apply(pos)
        o = orc.apply(pos)
        rms, mx = force_errors(r["forces"], o["forces"])
        worst = max(worst, rms)
        assert rms <= tol_rms, (s.name, kernel, step, rms)
        assert mx <= 1e-3 if kernel == "fixed" else mx <= 1e-2, (s.name, kernel, step, mx)
        escale = max(abs(o["e_lj"]), abs(o["e_crf"]), 1e-9)
        assert rel(r["e_lj"], o["e_lj"], escale) <= tol_e, (s.name, step, r["e_lj"], o["e_lj"])
        assert rel(r["e_crf"], o["e_crf"], escale) <= tol_e, (s.name, step, r["e_crf"], o["e_crf"])
        vscale = max(np.abs(o["virial"]).max(), 1e-9)
        assert np.abs(r["virial"] - o["virial"]).max() <= tol_e * 10 * vscale, (s.name, step)
        if kernel == "fixed":
            gscale = max(np.abs(o["egroup_lj"]).max(), np.abs(o["egroup_crf"]).max(), 1e-9)
            assert np.abs(r["egroup_lj"] - o["egroup_lj"]).max() <= tol_e * gscale
            assert np.abs(r["egroup_crf"] - o["egroup_crf"]).max() <= tol_e * gscale
        if abs(o["dhdl"]) > 0:
            assert rel(r["dhdl"], o["dhdl"], max(abs(o["dhdl"]), 1.0)) <= 1e-5, (r["dhdl"], o["dhdl"])
        if move:
            pos = pos + rng.normal(0.0, move, size=pos.shape)
    ff.close()
    orc.close()
    return worst


@pytest.mark.parametrize("name", FIXTURES + ["pair_lj", "pair_lj_mixed", "nacl_pair"])
def test_forces_fixtures_fixed(name):
    s, _ = load_fixture(name)
    compare_eval(s, "fixed")


@pytest.mark.parametrize("name", ["water_216_box", "ch4_water_fep", "nacl_water_box"])
def test_forces_fixtures_plain(name):
    s, _ = load_fixture(name)
    compare_eval(s, "plain", tol_rms=1e-4, tol_e=1e-4)


def test_spc1000_fixed_and_plain():
    s = generators.config1_spc1000()
    compare_eval(s, "fixed")
    compare_eval(s, "plain", tol_rms=1e-4, tol_e=1e-4)


@pytest.mark.parametrize("variant", ["fixture", "charged_pair"])
@pytest.mark.parametrize("lam", [0.0, 0.125, 0.6, 1.0])
def test_fep_fixture_one_four_and_atom_pair(variant, lam):
    """aladip_vacuum_fep: perturbed 1-4 pairs (perturbed.rs:517-605) and the PERTATOMPAIR
    correction (perturbed.rs:624-707) on the device against the oracle, with the pair's first
    atom uncharged (as converted) or charged (+0.15 e, so the pair's reaction-field term counts)."""
    s, _ = load_fixture("aladip_vacuum_fep")
    assert s.topo.n_pert_pairs == 1 and len(s.topo.normalized().o14) > 0
    if variant == "charged_pair":
        s.topo.charge = s.topo.charge.copy()
        s.topo.charge[int(s.topo.pp_i[0])] = 0.15
    s.params.lam = lam
    compare_eval(s, "fixed")
    compare_eval(s, "plain", tol_rms=1e-4, tol_e=1e-4)


def test_spc30000_twin_range_forces_over_a_period():
    """The bench workload (30,000 SPC waters, 9.65 nm, 0.8/1.4 nm, NSNB 5) against the FP64 oracle
    over six steps with motion: a rebuild step with the long-range refresh, four short-range steps
    on the cached long-range forces (forcefield.rs:620-697), and the next rebuild.  Forces RMS
    <= 1e-5 relative, per-atom max <= 1e-3, energies, energy groups and virial as compare_eval."""
    s = generators.config2_spc30000()
    worst = compare_eval(s, "fixed", steps=6, move=0.001, seed=9)
    assert worst <= 1e-5


def test_twin_range_cache_over_steps():
    """Short range every step, long range refreshed every NSNB steps (forcefield.rs:620-697)."""
    s = generators.spc_water_system(2000, box=generators.box_for_waters(2000), seed=21, rcutp=0.8, rcutl=1.4,
                                    nsnb=3)
    compare_eval(s, "fixed", steps=7, move=0.002, seed=5)


def test_fep_synthetic_windows():
    for lam in (0.0, 0.35, 1.0):
        s = generators.solvated_solute_system(700, 30, seed=1004, perturbed=True, lam=lam, rc=1.4)
        s.params.lam = lam
        compare_eval(s, "fixed")


def test_solute_small_box_per_atom_images():
    s = generators.solvated_solute_system(500, 200, seed=1003, rc=1.4)
    compare_eval(s, "fixed", steps=3, move=0.002)


WATER_KERNELS = [(1, 4), (2, 4), (2, 8), (3, 4), (4, 4), (4, 8)]


@pytest.mark.parametrize("layout,width", WATER_KERNELS)
@pytest.mark.parametrize("name", ["ch4_water_fep", "water_216_box", "nacl_3water_box", "water_3_box_twinrange"])
def test_water_kernel_variants_fixtures(name, layout, width):
    """Every solvent kernel variant (shared-bit width 4, per-lane-bit width 4 and 8) against the oracle."""
    s, _ = load_fixture(name)
    compare_eval(s, "fixed", cluster_size=width, layout=layout)


@pytest.mark.parametrize("layout,width", WATER_KERNELS)
def test_water_kernel_variants_twin_range_steps(layout, width):
    s = generators.spc_water_system(1500, box=generators.box_for_waters(1500), seed=22, rcutp=0.8, rcutl=1.4,
                                    nsnb=2)
    compare_eval(s, "fixed", steps=4, move=0.002, seed=6, cluster_size=width, layout=layout)


def coincident_water_system():
    """512 SPC waters with one hydrogen placed exactly on another water's hydrogen: water b
    (water 0's nearest neighbour) is moved rigidly so that its atom 1 sits on water 0's atom 2."""
    s = generators.spc_water_system(512, box=generators.box_for_waters(512), seed=77, rcutp=0.8, rcutl=1.2,
                                    nsnb=5)
    pos = s.pos.copy()
    o = pos[0::3]
    d = o[1:] - o[0]
    d -= s.box * np.round(d / s.box)
    b = 1 + int(np.argmin((d * d).sum(1)))
    pos[3 * b:3 * b + 3] += pos[2] - pos[3 * b + 1]
    out = s.copy()
    out.pos = pos
    out.name = "spc512_coincident_h"
    return out


@pytest.mark.parametrize("layout,width", WATER_KERNELS)
def test_water_kernels_coincident_atoms(layout, width):
    """An atom pair at r^2 < 1e-10 contributes nothing, as lj_crf_interaction's guard
    (innerloops.rs:32) has it: every solvent kernel's slow path against the oracle."""
    compare_eval(coincident_water_system(), "fixed", cluster_size=width, layout=layout)


def vacuum_droplet():
    s = generators.spc_water_system(216, box=generators.box_for_waters(216), seed=91, rcutp=0.8, rcutl=1.2, nsnb=2)
    s.params = dataclasses.replace(s.params, boundary=0)
    s.name = "spc216_vacuum"
    return s


@pytest.mark.parametrize("layout,width", WATER_KERNELS)
def test_water_kernels_vacuum(layout, width):
    """Solvent without periodic boundaries (no images, the cell grid spans the molecules'
    extent): every solvent kernel over twin-range steps with motion against the oracle."""
    compare_eval(vacuum_droplet(), "fixed", steps=3, move=0.002, seed=5, cluster_size=width, layout=layout)


def test_plain_kernel_vacuum():
    compare_eval(vacuum_droplet(), "plain", tol_rms=1e-4, tol_e=1e-4)


def test_deterministic_bits():
    s = generators.config1_spc1000()
    ff = Forcefield(s, kernel="fixed")
    a = ff.apply(s.pos, force_rebuild=True)
    b = ff.apply(s.pos, force_rebuild=True)
    assert np.array_equal(a["forces"], b["forces"])
    assert a["e_lj"] == b["e_lj"] and a["e_crf"] == b["e_crf"]
    assert np.array_equal(a["virial"], b["virial"])
    ff.close()


def test_pair_counts_match_oracle_lists():
    s = generators.config1_spc1000()
    ff = Forcefield(s, kernel="fixed")
    r = ff.apply(s.pos)
    lists = ob.pairlist(s)
    n_expected = len(lists[0]) + len(lists[1]) + 9 * len(lists[2]) + len(lists[3])
    assert r["n_pairs_short"] + r["n_pairs_long"] == n_expected
    ff.close()


@pytest.mark.parametrize("entry", ["serial", "parallel"])
def test_innerloop_stub_replacement(entry):
    """gr_lj_crf_innerloop / gr_lj_crf_innerloop_parallel (ffi.rs:55-145 with a body) against an
    FP64 loop over the same FP32-rounded inputs: forces RMS <= 1e-5 relative; each energy within
    1e-5 of the sum of its per-pair magnitudes (the FP32 pair terms are summed in FP64); the
    parallel name returns the serial name's results (the kernel's FP32 force atomics may differ
    in order, so within 1e-6 RMS)."""
    from gromos_nb.nonbonded import CRFParameters, lj_crf_innerloop
    s, _ = load_fixture("nacl_water_box")
    lists = ob.pairlist(s, algorithm=0)
    pairs = np.concatenate([lists[0], lists[1], lists[3]])
    crf = CRFParameters.new(s.params.rcutl, 1.0, s.params.epsrf, 0.0)
    lj = s.topo.lj[:, :, :2].copy()
    f, elj, ecrf, vir = lj_crf_innerloop(s.pos, s.topo.charge, s.topo.iac, pairs, lj, crf, box=s.box,
                                         parallel=(entry == "parallel"))
    pos32 = s.pos.astype(np.float32).astype(np.float64)
    q32 = s.topo.charge.astype(np.float32).astype(np.float64)
    fpe = 138.9354
    ref = np.zeros_like(s.pos)
    e1 = e2 = a1 = a2 = 0.0
    for i, j in pairs:
        r = pos32[i] - pos32[j]
        r -= s.box * np.round(r / s.box)
        r2 = r @ r
        c6, c12 = s.topo.lj[s.topo.iac[i], s.topo.iac[j], :2]
        q = q32[i] * q32[j] * fpe
        ir2 = 1 / r2
        ir6 = ir2 ** 3
        el = (c12 * ir6 - c6) * ir6
        ec = q * (np.sqrt(ir2) - crf.crf_2cut3i * r2 - crf.crf_cut)
        e1, e2, a1, a2 = e1 + el, e2 + ec, a1 + abs(el), a2 + abs(ec)
        fs = (12 * c12 * ir6 - 6 * c6) * ir6 * ir2 + q * (np.sqrt(ir2) * ir2 + crf.crf_cut3i)
        ref[i] += r * fs
        ref[j] -= r * fs
    rms, _ = force_errors(f.astype(np.float64), ref)
    assert rms <= 1e-5, rms
    assert abs(elj - e1) <= 1e-5 * a1 and abs(ecrf - e2) <= 1e-5 * a2, (elj, e1, a1, ecrf, e2, a2)
    if entry == "parallel":
        g, gl, gc, gv = lj_crf_innerloop(s.pos, s.topo.charge, s.topo.iac, pairs, lj, crf, box=s.box)
        assert force_errors(f.astype(np.float64), g.astype(np.float64))[0] <= 1e-6
        assert abs(gl - elj) <= 1e-6 * a1 and abs(gc - ecrf) <= 1e-6 * a2


@pytest.mark.parametrize("kind", ["water", "solute_fep"])
def test_graph_replay_bit_identical(kind):
    """GR_EVAL_GRAPH (recorded step graphs) == the launch-by-launch path, bit for bit, over rebuilds."""
    if kind == "water":
        s = generators.spc_water_system(1500, box=generators.box_for_waters(1500), seed=23, rcutp=0.8, rcutl=1.2,
                                        nsnb=3)
    else:
        s = generators.solvated_solute_system(600, 30, seed=1006, perturbed=True, lam=0.4, rc=1.2, nsnb=3)
        s.params.lam = 0.4
    a, b = Forcefield(s), Forcefield(s)
    rng = np.random.default_rng(3)
    pos = s.pos.copy()
    for step in range(8):
        ra = a.apply(pos)
        rb = b.apply(pos, graph=True)
        assert np.array_equal(ra["forces"], rb["forces"]), step
        assert ra["e_lj"] == rb["e_lj"] and ra["e_crf"] == rb["e_crf"] and ra["dhdl"] == rb["dhdl"]
        assert np.array_equal(ra["virial"], rb["virial"])
        assert ra["rebuilt"] == rb["rebuilt"]
        pos = pos + rng.normal(0.0, 0.002, size=pos.shape)
    a.close()
    b.close()


def test_graph_replay_regrows_lists():
    """Graph replay whose rebuild overflows (denser positions than the lists were sized for): the
    lists are grown, the graphs recorded again, and forces equal the launch-by-launch path."""
    s = generators.spc_water_system(1500, box=generators.box_for_waters(1500), seed=25, rcutp=0.8, rcutl=1.2,
                                    nsnb=2)
    a, b = Forcefield(s), Forcefield(s, list_capacity=16)
    w = s.pos.reshape(-1, 3, 3)
    dense = (w + (0.7 * w[:, 0] - w[:, 0])[:, None, :]).reshape(-1, 3)   # rigid waters, centres pulled in
    for step, pos in enumerate([s.pos, s.pos, dense, dense, dense]):
        ra = a.apply(pos, force_rebuild=True)
        rb = b.apply(pos, force_rebuild=True, graph=True)
        assert np.all(np.isfinite(ra["forces"]))
        assert np.array_equal(ra["forces"], rb["forces"]), step
        assert ra["e_lj"] == rb["e_lj"] and ra["e_crf"] == rb["e_crf"]
    a.close()
    b.close()


def test_list_overflow_regrow():
    """Solvent lists far too small at the start: every overflow is grown and the step redone."""
    s = generators.spc_water_system(1500, box=generators.box_for_waters(1500), seed=24, rcutp=0.8, rcutl=1.2,
                                    nsnb=2)
    compare_eval(s, "fixed", steps=5, move=0.002, seed=7, list_capacity=16)


def _rel_errors(got, ref):
    d = got - ref
    rms = float(np.sqrt((d * d).sum() / max((ref * ref).sum(), 1e-300)))
    mx = float(np.abs(d).max() / max(np.abs(ref).max(), 1e-300))
    return rms, mx


@pytest.mark.parametrize("kernel", ["fixed", "plain"])
def test_accuracy_report(kernel):
    """RMS and max relative errors against the FP64 oracle for forces, energy groups, virial and
    dH/dlambda (1000 SPC waters at 1.4 nm; a solvated perturbed solute at lambda 0.5; the 30,000-water
    twin-range bench workload at its rebuild step), printed."""
    rows = []
    s1 = generators.config1_spc1000()
    s2 = generators.solvated_solute_system(700, 30, seed=1004, perturbed=True, lam=0.5, rc=1.4)
    s2.params.lam = 0.5
    s3 = generators.config2_spc30000()
    for name, s in (("spc1000", s1), ("fep_solute30_lambda0.5", s2), ("spc30000_twin_range", s3)):
        ff = Forcefield(s, kernel=kernel)
        r = ff.apply(s.pos)
        o = ob.OracleForcefield(s).apply(s.pos)
        ff.close()
        fr, fm = force_errors(r["forces"], o["forces"])
        lr, lm = _rel_errors(r["egroup_lj"], o["egroup_lj"]) if kernel == "fixed" else (float("nan"),) * 2
        cr, cm = _rel_errors(r["egroup_crf"], o["egroup_crf"]) if kernel == "fixed" else (float("nan"),) * 2
        vr, vm = _rel_errors(r["virial"], o["virial"])
        dh = abs(r["dhdl"] - o["dhdl"]) / max(abs(o["dhdl"]), 1e-12) if abs(o["dhdl"]) > 0 else 0.0
        rows.append((name, fr, fm, lr, lm, cr, cm, vr, vm, dh))
        tol = 1e-5 if kernel == "fixed" else 1e-4
        assert fr <= tol and vr <= 10 * tol
    print(f"\naccuracy vs FP64 oracle, {kernel} kernel: name | forces rms, max | LJ groups rms, max | "
          f"CRF groups rms, max | virial rms, max | dH/dlambda rel")
    for row in rows:
        print(" | ".join([row[0]] + [f"{v:.2e}" for v in row[1:]]))


def test_null_output_arguments_are_rejected():
    """Entry points given a null output or input array return GR_ERR_INVALID instead of dereferencing it."""
    from gromos_nb import _lib
    s = generators.spc_water_system(216, box=generators.box_for_waters(216), seed=3, rcutp=0.8, rcutl=0.9)
    ff = Forcefield(s)
    ff.apply(s.pos)
    L = _lib.lib()
    for name in ("gr_set_box", "gr_pairlist_counts", "gr_last_timings", "gr_ctx_launches", "gr_forces_device"):
        assert getattr(L, name)(ff.handle, None) == _lib.GR_ERR_INVALID, name
    r = ff.apply(s.pos)                          # the context is still usable
    assert np.isfinite(r["e_lj"])
    ff.close()
