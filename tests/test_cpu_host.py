"""CPU-only checks of the host side: the C-ABI library loads and exports every
declared entry point, calls fail cleanly without a GPU, and the host helpers
(GROMOS readers, generators, CRF parameters) agree with the oracle."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle_binding as ob
from gromos_nb import _lib, generators
from gromos_nb.nonbonded import CRFParameters


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="module")
def libnb():
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    return _lib.lib()


def test_library_exports_every_declared_symbol(libnb):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    declared = _lib.declared_symbols()
    assert declared, "no declarations found"
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


def test_build_targets_sm100a():
    assert "arch=compute_100a,code=sm_100a" in _lib.NVCC_FLAGS


@pytest.mark.skipif(_have_gpu(), reason="checks the no-device error path")
def test_no_device_is_an_error(libnb):
    h = C.c_void_p()
    st = libnb.gr_ctx_create(0, C.byref(h))
    assert st == _lib.GR_ERR_NO_DEVICE
    assert b"no CUDA device" in libnb.gr_last_error()


def test_null_context_is_rejected(libnb):
    assert libnb.gr_set_box(None, None) == _lib.GR_ERR_INVALID
    assert libnb.gr_forces_eval(None, 0, None) == _lib.GR_ERR_INVALID


def test_crf_parameters_match_oracle():
    for rc, eps_rf, kappa in [(1.4, 61.0, 0.0), (0.9, 62.0, 0.0), (1.4, 78.5, 0.0), (1.2, 66.0, 0.5)]:
        py = CRFParameters.new(rc, 1.0, eps_rf, kappa)
        orc = ob.crf_params(rc, 1.0, eps_rf, kappa)
        assert (py.crf_cut, py.crf_2cut3i, py.crf_cut3i, py.cutoff_sq) == tuple(orc)


def test_spc_generator_geometry_and_contacts():
    s = generators.config1_spc1000()
    pos = s.pos.reshape(-1, 3, 3)
    oh = np.linalg.norm(pos[:, 1] - pos[:, 0], axis=1)
    assert np.allclose(oh, 0.1, atol=1e-12)
    ang = np.degrees(np.arccos(np.einsum("ij,ij->i", pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0]) / 0.01))
    assert np.allclose(ang, 109.47, atol=1e-9)
    from scipy.spatial import cKDTree
    t = cKDTree(np.mod(s.pos, 3.104), boxsize=3.104)
    pairs = t.query_pairs(0.15, output_type="ndarray")
    mol = np.repeat(np.arange(1000), 3)
    assert not np.any(mol[pairs[:, 0]] != mol[pairs[:, 1]])
    # seeded: same seed, same positions
    assert np.array_equal(s.pos, generators.config1_spc1000().pos)


def test_solute_generator_neutral_charge_groups():
    s = generators.solvated_solute_system(400, 60, seed=3, perturbed=True)
    t = s.topo
    for c in range(t.n_solute_cg):
        a, b = t.cg_offsets[c], t.cg_offsets[c + 1]
        assert 3 <= b - a <= 5
        assert abs(t.charge[a:b].sum()) < 1e-12
        assert abs(t.pert_b_q[a:b].sum()) < 1e-12
    assert t.n_atoms == 60 + 3 * 400


def test_gromos_reader_roundtrip_fixture():
    from golden_loader import load_fixture
    s, ex = load_fixture("ch4_water_fep")
    assert s.topo.n_atoms == 2998 and s.topo.n_solute_cg == 1 and s.topo.n_egroups == 2
    assert s.params.rcutp == 0.8 and s.params.rcutl == 1.4 and s.params.nsnb == 1
    assert s.topo.pert_idx[0] == 0 and s.topo.pert_alpha_lj[0] == 0.25  # 0.5 * ALPHLJ 0.5


def test_oracle_md_settle_constraints_and_cadence():
    """Oracle MD: SETTLE keeps the rigid SPC triangle; split runs equal one run."""
    import oracle_binding as ob
    from gromos_nb import generators as g
    s = g.spc_water_system(216, box=g.box_for_waters(216), seed=5, rcutp=0.8, rcutl=0.8)
    m = g.masses(s)
    v = g.maxwell_velocities(m, 300.0, 7)
    o1 = ob.OracleForcefield(s)
    x, vv, st = o1.md_run(s.pos, v, m, 10, dist_oh=0.1, dist_hh=g.SPC_DHH)
    assert st["settle_failures"] == 0
    w = x.reshape(-1, 3, 3)
    assert np.abs(np.linalg.norm(w[:, 1] - w[:, 0], axis=1) - 0.1).max() < 1e-12
    assert np.abs(np.linalg.norm(w[:, 2] - w[:, 1], axis=1) - g.SPC_DHH).max() < 1e-12
    o2 = ob.OracleForcefield(s)
    x2, v2, _ = o2.md_run(s.pos, v, m, 4, dist_oh=0.1, dist_hh=g.SPC_DHH)
    x2, v2, _ = o2.md_run(x2, v2, m, 6, dist_oh=0.1, dist_hh=g.SPC_DHH)
    assert np.array_equal(x, x2) and np.array_equal(vv, v2)


def test_md_entry_points_reject_bad_input_without_device():
    from gromos_nb import _lib
    import ctypes as C
    L = _lib.lib()
    mp = _lib.GrMdParams(0.002, 1, 0.1, 0.1633, 300.0, -1.0)
    assert L.gr_md_init(None, None, None, C.byref(mp)) == _lib.GR_ERR_INVALID
    assert L.gr_md_run(None, 1, None) == _lib.GR_ERR_INVALID


def test_batch_entry_points_without_device():
    from gromos_nb import _lib
    import ctypes as C
    L = _lib.lib()
    h = C.c_void_p()
    assert L.gr_batch_create(0, C.byref(h)) == _lib.GR_ERR_NO_DEVICE
    assert L.gr_batch_md_run(None, 1) == _lib.GR_ERR_INVALID
    assert L.gr_batch_add(None, None) == _lib.GR_ERR_INVALID


def test_server_entry_points_without_device():
    from gromos_nb import _lib
    import ctypes as C
    L = _lib.lib()
    h = C.c_void_p()
    assert L.gr_server_create(0, 1 << 30, 5, C.byref(h)) == _lib.GR_ERR_NO_DEVICE
    assert L.gr_server_create(0, 0, 5, C.byref(h)) == _lib.GR_ERR_INVALID
    assert L.gr_server_create(0, 1 << 30, 0, C.byref(h)) == _lib.GR_ERR_INVALID
    n = C.c_int32(0)
    assert L.gr_server_step(None, C.byref(n)) == _lib.GR_ERR_INVALID
    assert L.gr_server_submit(None, None, None) == _lib.GR_ERR_INVALID
    assert L.gr_server_release(None, 0) == _lib.GR_ERR_INVALID
    assert L.gr_server_destroy(None) == _lib.GR_OK


def test_energy_params_mirror_reference_defaults():
    """EnergyParams::default (crates/gromos-forces/src/energy.rs:52-66) and the single-cutoff list setup."""
    from gromos_nb.energy import EnergyParams, SinglePointEnergy, _nonbonded_params
    p = EnergyParams()
    assert (p.cutoff, p.epsilon, p.rf_epsilon, p.rf_kappa, p.pairlist_freq, p.atoms_per_solvent) == \
        (1.4, 1.0, 78.5, 0.0, 1, 3)
    assert p.ntf == (True, True, True, True) and p.quartic_bonds
    nb = _nonbonded_params(EnergyParams(cutoff=0.9, rf_epsilon=62.0), np.array([3.0, 3.0, 3.0]))
    assert (nb.rcutp, nb.rcutl, nb.skin, nb.nsnb, nb.boundary, nb.epsrf) == (0.9, 0.9, 0.0, 1, 1, 62.0)
    assert _nonbonded_params(EnergyParams(), np.zeros(3)).boundary == 0   # vacuum (energy.rs:108-117)
    assert SinglePointEnergy().potential == 0.0


def test_energy_frames_entry_rejects_null_context():
    from gromos_nb import _lib
    L = _lib.lib()
    assert L.gr_energy_frames(None, 1, None, None, None, None, None, None) == _lib.GR_ERR_INVALID


def test_single_atom_solute_generator():
    """Serving jobs use single-atom solute CGs: neutral, at least 0.35 nm apart; the default keeps 3-5 atom CGs."""
    from gromos_nb import generators as gen
    s = gen.solvated_solute_system(400, 60, seed=11, single_atom_cgs=True)
    t = s.topo
    assert t.n_solute_cg == t.n_solute_atoms == 60
    assert abs(t.charge[:60].sum()) < 1e-12 and np.abs(t.charge[:60]).max() > 0.1
    d = s.pos[:60, None, :] - s.pos[None, :60, :]
    d -= s.box * np.round(d / s.box)
    r = np.sqrt((d * d).sum(-1)) + np.eye(60) * 9
    assert r.min() >= 0.35 - 1e-9
    m = gen.solvated_solute_system(400, 60, seed=11)
    sizes = np.diff(m.topo.cg_offsets[:m.topo.n_solute_cg + 1])
    assert sizes.min() >= 3 and sizes.max() <= 5


def test_trajectory_writers_round_trip(tmp_path):
    """ENERTRJ and FREEFORCERED files in the reference writers' layout, read back."""
    from gromos_nb import gromos_io as io
    assert io.rust_exp(123.456) == "    1.234560000000e2"
    assert io.rust_exp(-0.001) == "  -1.000000000000e-3"
    assert io.rust_exp(0.0) == "    0.000000000000e0"
    frames = [io.md_energy_frame(0.002 * k, 1000.0 + k, -5000.0 - 3.5 * k, -20000.25 + k, 600.0, volume=27.0)
              for k in range(3)]
    p = str(tmp_path / "e.tre")
    with io.EnergyWriter(p, "device MD") as w:
        for f in frames:
            w.write_frame(f)
    text = open(p, encoding="utf-8").read().splitlines()
    assert text[:4] == ["TITLE", "  device MD", "END", "ENERTRJ"] and text[-1] == "END"
    assert text[5] == "#   0 = Time (ps)"
    back = io.read_energy_trajectory(p)
    assert len(back) == 3
    for a, b in zip(frames, back):
        np.testing.assert_allclose(b.values(), a.values(), rtol=1e-12, atol=1e-300)
    assert back[1].lj == -5003.5 and back[1].potential == back[1].lj + back[1].coul_real
    forces = np.random.default_rng(1).normal(0.0, 300.0, size=(23, 3))
    q = str(tmp_path / "f.trf")
    with io.ForceWriter(q, "forces", constraint_forces=True) as w:
        w.write_frame(0, 0.0, forces)
        w.write_frame(5, 0.01, -forces)
    lines = open(q, encoding="utf-8").read().splitlines()
    assert lines[4] == "              0    0.000000000"
    assert lines[7] == f"{forces[0, 0]:18.9f}{forces[0, 1]:18.9f}{forces[0, 2]:18.9f}"
    assert "#        10" in lines and "CONSFORCERED" in lines
    np.testing.assert_allclose(io.read_forces_step(q, 0), forces, atol=1e-9)
    np.testing.assert_allclose(io.read_forces_step(q, 5), -forces, atol=1e-9)


def test_single_atom_solute_md_stays_stable():
    """A serving-style system (single-atom solute CGs, Berendsen bath) runs 800 FP64 oracle MD steps
    with no SETTLE failure; unbonded multi-atom CGs drifted apart within that many steps."""
    from gromos_nb import generators as gen
    s = gen.solvated_solute_system(500, 60, seed=77, rc=1.0, nsnb=5, single_atom_cgs=True)
    m = gen.masses(s)
    o = ob.OracleForcefield(s)
    x, v, st = o.md_run(s.pos, gen.maxwell_velocities(m, 300.0, 5), m, 800, dist_oh=0.1, dist_hh=gen.SPC_DHH,
                        temperature=300.0, tau=0.1)
    assert st["settle_failures"] == 0
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))


def test_reference_arm_json_line_and_nonzero_ranks():
    """`bench.py --impl reference` (the CPU reference arm) prints one JSON line with the bench
    contract's keys; under torchrun a rank other than 0 exits 0 without work or output."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cmd = [sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "3"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["config"]["workload"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["kind"] == "port"
    other = subprocess.run(cmd, capture_output=True, text=True, timeout=120, check=True,
                           env=dict(env, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1"))
    assert other.stdout.strip() == ""
