"""Readers and writers for the GROMOS file subset the nonbonded path needs.

Topology (.topo/.top), configuration (.conf/.cnf), input parameters (.in/.imd)
and perturbation topology (.ptp) are read; energy (.tre, ENERTRJ) and force
(.trf, FREEFORCERED) trajectories are read and written in the layout of
gromos-rs's EnergyWriter / ForceWriter, so trajectories of the device MD can be
diffed against the reference's output.  The topology is assembled the way
gromos-rs's ``build_topology`` + ``Topology::solvate`` do it
(crates/gromos-io/src/topology.rs:1040-1298, crates/gromos-core/src/topology.rs:1204-1262):

* IAC and atom numbers are 1-based in the files and stored 0-based;
* a solute CG ends at every atom with CGC == 1;
* solute exclusions = INE lists + bonds (BOND, BONDH) + angle end atoms
  (BONDANGLE, BONDANGLEH), made symmetric, sorted and de-duplicated;
* 1-4 pairs = INE14 lists, kept separate from the exclusions;
* every solvent molecule is one CG whose atoms all exclude each other;
* the LJ matrix covers every type the LJPARAMETERS table names.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, TextIO, Tuple

import numpy as np

from .system import NonbondedParams, System, Topology, csr_from_lists


def read_blocks(path: str) -> Dict[str, List[str]]:
    """Split a GROMOS file into {BLOCKNAME: [non-comment lines]} (first occurrence)."""
    blocks: Dict[str, List[str]] = {}
    cur: Optional[str] = None
    buf: List[str] = []
    with open(path) as fh:
        for raw in fh:
            line = raw.rstrip("\n")
            s = line.strip()
            if cur is None:
                if s and not s.startswith("#"):
                    cur, buf = s.split()[0], []
                continue
            if s == "END":
                blocks.setdefault(cur, buf)
                cur = None
                continue
            if s.startswith("#") or not s:
                continue
            buf.append(line)
    return blocks


def _tokens(lines: List[str]) -> List[str]:
    out: List[str] = []
    for ln in lines:
        out.extend(ln.split())
    return out


def _read_topology_blocks(blocks):
    fpe = 138.9354
    if "PHYSICALCONSTANTS" in blocks:
        fpe = float(_tokens(blocks["PHYSICALCONSTANTS"])[0])
    sol_iac, sol_q, sol_cgc, sol_excl, sol_14 = [], [], [], [], []
    if "SOLUTEATOM" in blocks:
        lines = blocks["SOLUTEATOM"]
        nrp = int(lines[0].split()[0])
        k = 1
        for _ in range(nrp):
            parts = lines[k].split()
            k += 1
            sol_iac.append(int(parts[3]) - 1)
            sol_q.append(float(parts[5]))
            sol_cgc.append(int(parts[6]))
            ine = int(parts[7])
            ex = [int(x) - 1 for x in parts[8:8 + ine]]
            while len(ex) < ine:  # continuation lines
                more = lines[k].split()
                k += 1
                ex += [int(x) - 1 for x in more]
            sol_excl.append(ex)
            p14 = lines[k].split()
            k += 1
            n14 = int(p14[0])
            l14 = [int(x) - 1 for x in p14[1:1 + n14]]
            while len(l14) < n14:
                more = lines[k].split()
                k += 1
                l14 += [int(x) - 1 for x in more]
            sol_14.append(l14)
    bonds: List[Tuple[int, int]] = []
    for name in ("BONDH", "BOND"):
        if name in blocks and blocks[name]:
            ls = blocks[name]
            for ln in ls[1:1 + int(ls[0].split()[0])]:
                p = ln.split()
                bonds.append((int(p[0]) - 1, int(p[1]) - 1))
    angles: List[Tuple[int, int]] = []
    for name in ("BONDANGLEH", "BONDANGLE"):
        if name in blocks and blocks[name]:
            ls = blocks[name]
            for ln in ls[1:1 + int(ls[0].split()[0])]:
                p = ln.split()
                angles.append((int(p[0]) - 1, int(p[2]) - 1))
    ljtab: Dict[Tuple[int, int], Tuple[float, float, float, float]] = {}
    if "LJPARAMETERS" in blocks:
        ls = blocks["LJPARAMETERS"]
        for ln in ls[1:]:
            p = ln.split()
            if len(p) < 4:
                continue
            i, j = int(p[0]) - 1, int(p[1]) - 1
            c12, c6 = float(p[2]), float(p[3])
            cs12 = float(p[4]) if len(p) > 4 else c12
            cs6 = float(p[5]) if len(p) > 5 else c6
            ljtab[(i, j)] = (c6, c12, cs6, cs12)
    solv = []
    if "SOLVENTATOM" in blocks:
        ls = blocks["SOLVENTATOM"]
        nram = int(ls[0].split()[0])
        for ln in ls[1:1 + nram]:
            p = ln.split()
            solv.append((int(p[2]) - 1, float(p[4])))
    return fpe, sol_iac, sol_q, sol_cgc, sol_excl, sol_14, bonds, angles, ljtab, solv


def read_topology(path: str, nsm: int) -> Topology:
    """Build the nonbonded topology from a GROMOS topology plus NSM solvent molecules."""
    blocks = read_blocks(path)
    fpe, sol_iac, sol_q, sol_cgc, sol_excl, sol_14, bonds, angles, ljtab, solv = _read_topology_blocks(blocks)
    nsol = len(sol_iac)
    aps = len(solv)
    nat = nsol + aps * nsm
    charge = np.zeros(nat)
    iac = np.zeros(nat, dtype=np.int32)
    charge[:nsol] = sol_q
    iac[:nsol] = sol_iac
    for m in range(nsm):
        for a, (t, q) in enumerate(solv):
            iac[nsol + m * aps + a] = t
            charge[nsol + m * aps + a] = q
    # solute CGs from CGC codes (gromos-io topology.rs:1094-1127)
    cg_off = [0]
    for i in range(nsol):
        if sol_cgc[i] == 1:
            cg_off.append(i + 1)
    if cg_off[-1] != nsol:
        cg_off.append(nsol)
    n_solute_cg = len(cg_off) - 1
    for m in range(nsm):
        cg_off.append(nsol + (m + 1) * aps)
    excl: List[set] = [set() for _ in range(nat)]
    for i, lst in enumerate(sol_excl):
        for j in lst:
            excl[i].add(j)
            if j < nsol:
                excl[j].add(i)
    for i, j in bonds + angles:
        excl[i].add(j)
        excl[j].add(i)
    for m in range(nsm):
        b = nsol + m * aps
        for x in range(aps):
            for y in range(x + 1, aps):
                excl[b + x].add(b + y)
                excl[b + y].add(b + x)
    excl_off, excl_flat = csr_from_lists([sorted(s) for s in excl], nat)
    o14 = [list(l) for l in sol_14] + [[] for _ in range(nat - nsol)]
    o14_off, o14_flat = csr_from_lists(o14, nat)
    max_t = max([max(k) for k in ljtab] + [int(iac.max()) if nat else 0])
    nt = max_t + 1
    lj = np.zeros((nt, nt, 4))
    for (i, j), v in ljtab.items():
        lj[i, j] = v
        lj[j, i] = v
    return Topology(charge=charge, iac=iac, lj=lj, cg_offsets=np.asarray(cg_off, dtype=np.int32),
                    n_solute_atoms=nsol, n_solute_cg=n_solute_cg, excl_off=excl_off, excl=excl_flat,
                    o14_off=o14_off, o14=o14_flat, atoms_per_solvent=aps if aps else 3,
                    four_pi_eps_i=fpe)


def read_configuration(path: str):
    """POSITION/POSITIONRED + GENBOX/BOX -> (pos (N,3), box (3,))."""
    blocks = read_blocks(path)
    pos = None
    if "POSITION" in blocks:
        rows = []
        for ln in blocks["POSITION"]:
            rows.append([float(x) for x in ln[24:].split()[:3]])
        pos = np.asarray(rows, dtype=np.float64)
    elif "POSITIONRED" in blocks:
        pos = np.asarray([[float(x) for x in ln.split()[:3]] for ln in blocks["POSITIONRED"]])
    box = np.zeros(3)
    if "GENBOX" in blocks:
        t = _tokens(blocks["GENBOX"])
        box = np.asarray([float(x) for x in t[1:4]])
    elif "BOX" in blocks:
        box = np.asarray([float(x) for x in _tokens(blocks["BOX"])[:3]])
    return pos, box


def read_imd(path: str) -> dict:
    """Fields of the IMD blocks used here."""
    b = read_blocks(path)
    out: dict = {}
    t = _tokens(b["SYSTEM"])
    out["npm"], out["nsm"] = int(t[0]), int(t[1])
    t = _tokens(b["PAIRLIST"])
    alg = t[0].lower()
    out["algorithm"] = {"standard": 0, "grid": 1, "grid_cell": 2}.get(alg, int(alg) if alg.isdigit() else 0)
    out["nsnb"], out["rcutp"], out["rcutl"] = int(t[1]), float(t[2]), float(t[3])
    t = _tokens(b["NONBONDED"])
    out["nlrele"], out["appak"], out["rcrf"], out["epsrf"] = int(t[0]), float(t[1]), float(t[2]), float(t[3])
    t = _tokens(b.get("BOUNDCOND", ["1 0"]))
    out["ntb"] = int(t[0])
    t = _tokens(b["FORCE"])
    negr = int(t[6])
    out["energy_groups_last"] = [int(x) for x in t[7:7 + negr]]
    if "STEP" in b:
        t = _tokens(b["STEP"])
        out["nstlim"], out["dt"] = int(t[0]), float(t[2])
    if "MULTIBATH" in b:
        # weak-coupling, NBATHS, then (TEMP0, TAU) of the first bath
        t = _tokens(b["MULTIBATH"])
        out["bath_temp0"], out["bath_tau"] = float(t[2]), float(t[3])
    if "PERTURBATION" in b:
        t = _tokens(b["PERTURBATION"])
        out["ntg"], out["rlam"] = int(t[0]), float(t[2])
        out["alphlj"], out["alphc"], out["nlam"] = float(t[4]), float(t[5]), int(t[6])
    else:
        out["ntg"] = 0
    return out


def read_ptp(path: str):
    """PERTATOMPARAM + PERTATOMPAIR (gromos-io ptp.rs), 0-based indices.

    Returns (atoms, pairs): atoms = [(seq, a_iac, a_q, b_iac, b_q, alj, acrf)],
    pairs = [(i, j, a_type, b_type or -1)].
    """
    b = read_blocks(path)
    atoms = []
    ls = b.get("PERTATOMPARAM", ["0"])
    n = int(ls[0].split()[0])
    for ln in ls[1:1 + n]:
        p = ln.split()
        atoms.append((int(p[0]) - 1, int(p[3]) - 1, float(p[5]), int(p[6]) - 1, float(p[8]),
                      float(p[9]), float(p[10])))
    pairs = []
    ls = b.get("PERTATOMPAIR", ["0"])
    n = int(ls[0].split()[0])
    for ln in ls[1:1 + n]:
        p = ln.split()
        bt = int(p[3])
        pairs.append((int(p[0]) - 1, int(p[1]) - 1, int(p[2]) - 1, bt - 1 if bt > 0 else -1))
    return atoms, pairs


def apply_perturbation(topo: Topology, atoms, pairs, alphlj: float, alphc: float) -> Topology:
    """Attach PertAtomInfo with alphas scaled by ALPHLJ/ALPHC (forcefield.rs:146-170)."""
    n = topo.n_atoms
    idx = -np.ones(n, dtype=np.int32)
    a_iac, b_iac, a_q, b_q, alj, acrf = [], [], [], [], [], []
    for k, (seq, ai, aq, bi, bq, lj_soft, crf_soft) in enumerate(atoms):
        idx[seq] = k
        a_iac.append(ai)
        b_iac.append(bi)
        a_q.append(aq)
        b_q.append(bq)
        alj.append(lj_soft * alphlj)
        acrf.append(crf_soft * alphc)
    topo.pert_idx = idx
    topo.pert_a_iac = np.asarray(a_iac, dtype=np.int32)
    topo.pert_b_iac = np.asarray(b_iac, dtype=np.int32)
    topo.pert_a_q = np.asarray(a_q)
    topo.pert_b_q = np.asarray(b_q)
    topo.pert_alpha_lj = np.asarray(alj)
    topo.pert_alpha_crf = np.asarray(acrf)
    topo.pp_i = np.asarray([p[0] for p in pairs], dtype=np.int32)
    topo.pp_j = np.asarray([p[1] for p in pairs], dtype=np.int32)
    topo.pp_a_type = np.asarray([p[2] for p in pairs], dtype=np.int32)
    topo.pp_b_type = np.asarray([p[3] for p in pairs], dtype=np.int32)
    return topo


def energy_groups_from_last(last_atoms: List[int], n_atoms: int) -> np.ndarray:
    """FORCE block NRE(k) = last atom (1-based) of group k -> per-atom group ids."""
    g = np.zeros(n_atoms, dtype=np.int32)
    start = 0
    for k, last in enumerate(last_atoms):
        g[start:last] = k
        start = last
    return g


def load_system(topo_path: str, conf_path: str, imd_path: str, ptp_path: Optional[str] = None,
                name: str = "") -> System:
    imd = read_imd(imd_path)
    topo = read_topology(topo_path, imd["nsm"])
    pos, box = read_configuration(conf_path)
    if pos.shape[0] != topo.n_atoms:
        raise ValueError(f"{conf_path}: {pos.shape[0]} positions for {topo.n_atoms} atoms")
    groups = imd["energy_groups_last"]
    topo.egroup = energy_groups_from_last(groups, topo.n_atoms)
    topo.n_egroups = len(groups)
    p = NonbondedParams(rcutp=imd["rcutp"], rcutl=imd["rcutl"], skin=0.0, epsilon=1.0,
                        epsrf=imd["epsrf"], kappa=imd["appak"], nsnb=imd["nsnb"],
                        algorithm=imd["algorithm"], boundary=1 if imd["ntb"] != 0 else 0)
    if imd["ntg"] != 0 and ptp_path:
        atoms, pairs = read_ptp(ptp_path)
        apply_perturbation(topo, atoms, pairs, imd["alphlj"], imd["alphc"])
        p.lam, p.nlam, p.alphlj, p.alphc = imd["rlam"], imd["nlam"], imd["alphlj"], imd["alphc"]
    return System(topo=topo, pos=pos, box=box, params=p, name=name)


def read_energy03_step(path: str, step: int = 0) -> dict:
    """ENERGY03 totals (LJ = line 11, CRF = line 12 of '# totals') and the
    '# nonbonded' group block of one frame of an energy trajectory (.tre)."""
    lines = open(path).read().splitlines()
    i = 0
    while i < len(lines):
        if lines[i].strip() == "TIMESTEP":
            st = int(lines[i + 1].split()[0])
            if st == step:
                break
        i += 1
    j = i
    while lines[j].strip() != "ENERGY03":
        j += 1
    tot: List[float] = []
    groups: List[List[float]] = []
    mode = None
    for ln in lines[j + 1:]:
        s = ln.strip()
        if s == "END":
            break
        if s.startswith("#"):
            mode = s[1:].strip()
            continue
        if mode == "totals":
            tot.append(float(s))
        elif mode == "nonbonded":
            groups.append([float(x) for x in s.split()])
    return {"totals": tot, "e_lj": tot[10], "e_crf": tot[11], "nonbonded": groups}


def read_forces_step(path: str, step: int = 0) -> np.ndarray:
    """FREEFORCERED block of one frame of a force trajectory (.trf)."""
    lines = open(path).read().splitlines()
    cur = None
    i = 0
    while i < len(lines):
        s = lines[i].strip()
        if s == "TIMESTEP":
            cur = int(lines[i + 1].split()[0])
            i += 2
            continue
        if s == "FREEFORCERED" and cur == step:
            rows = []
            i += 1
            while lines[i].strip() != "END":
                t = lines[i].strip()
                if t and not t.startswith("#"):
                    rows.append([float(x) for x in t.split()[:3]])
                i += 1
            return np.asarray(rows)
        i += 1
    raise KeyError(f"step {step} not found in {path}")


def read_masses(path: str, nsm: int) -> np.ndarray:
    """Atom masses: SOLUTEATOM MASS column, then SOLVENTATOM MASS for each of the
    NSM solvent molecules (gromos-io topology.rs build order)."""
    blocks = read_blocks(path)
    masses: List[float] = []
    if "SOLUTEATOM" in blocks:
        lines = blocks["SOLUTEATOM"]
        nrp = int(lines[0].split()[0])
        k = 1
        for _ in range(nrp):
            parts = lines[k].split()
            k += 1
            masses.append(float(parts[4]))
            ine = int(parts[7])
            seen = len(parts) - 8
            while seen < ine:
                seen += len(lines[k].split())
                k += 1
            p14 = lines[k].split()
            k += 1
            n14, seen = int(p14[0]), len(p14) - 1
            while seen < n14:
                seen += len(lines[k].split())
                k += 1
    solv: List[float] = []
    if "SOLVENTATOM" in blocks:
        ls = blocks["SOLVENTATOM"]
        for ln in ls[1:1 + int(ls[0].split()[0])]:
            solv.append(float(ln.split()[3]))
    return np.asarray(masses + solv * nsm, dtype=np.float64)


def read_solvent_constraints(path: str) -> List[Tuple[int, int, float]]:
    """SOLVENTCONSTR: (i, j, length) with 0-based solvent atom indices."""
    blocks = read_blocks(path)
    out: List[Tuple[int, int, float]] = []
    if "SOLVENTCONSTR" in blocks:
        ls = blocks["SOLVENTCONSTR"]
        for ln in ls[1:1 + int(ls[0].split()[0])]:
            p = ln.split()
            out.append((int(p[0]) - 1, int(p[1]) - 1, float(p[2])))
    return out


def read_velocities(path: str) -> np.ndarray:
    """VELOCITY (24 ignored characters per line) or VELOCITYRED block of a configuration."""
    blocks = read_blocks(path)
    if "VELOCITY" in blocks:
        return np.asarray([[float(x) for x in ln[24:].split()[:3]] for ln in blocks["VELOCITY"]])
    if "VELOCITYRED" in blocks:
        return np.asarray([[float(x) for x in ln.split()[:3]] for ln in blocks["VELOCITYRED"]])
    raise KeyError(f"{path}: no VELOCITY block")


def read_position_trajectory(path: str) -> Tuple[List[int], List[np.ndarray]]:
    """(steps, positions) of every TIMESTEP / POSITIONRED frame of a .trc file."""
    lines = open(path).read().splitlines()
    steps: List[int] = []
    frames: List[np.ndarray] = []
    cur = None
    i = 0
    while i < len(lines):
        s = lines[i].strip()
        if s == "TIMESTEP":
            cur = int(lines[i + 1].split()[0])
            i += 2
            continue
        if s == "POSITIONRED":
            rows = []
            i += 1
            while lines[i].strip() != "END":
                t = lines[i].strip()
                if t and not t.startswith("#"):
                    rows.append([float(x) for x in t.split()[:3]])
                i += 1
            steps.append(cur)
            frames.append(np.asarray(rows))
        i += 1
    return steps, frames



# ---- trajectory writers ------------------------------------------------------
#
# Number formats follow the Rust formatting the reference's writers use:
# ``{:20.12e}`` (mantissa with 12 decimals, exponent without sign padding:
# ``1.234560000000e2``, ``-1.000000000000e-3``) for energies and ``{:>18.9}``
# / ``{:>15.9}`` fixed-point fields for forces and times.


def rust_exp(x: float, prec: int = 12, width: int = 20) -> str:
    """``format!("{:width.prec e}", x)`` as Rust prints an f64."""
    x = float(x)
    if math.isnan(x):
        t = "NaN"
    elif math.isinf(x):
        t = "inf" if x > 0 else "-inf"
    else:
        mant, exp = f"{x:.{prec}e}".split("e")
        t = f"{mant}e{int(exp)}"
    return t.rjust(width)


@dataclasses.dataclass
class EnergyFrame:
    """One energy-trajectory row (crates/gromos-io/src/energy.rs:97-121), kJ/mol, K, nm^3, ps."""

    time: float = 0.0
    kinetic: float = 0.0
    potential: float = 0.0
    total: float = 0.0
    temperature: float = 0.0
    volume: float = 0.0
    pressure: float = 0.0
    bond: float = 0.0
    angle: float = 0.0
    improper: float = 0.0
    dihedral: float = 0.0
    lj: float = 0.0
    coul_real: float = 0.0
    coul_recip: float = 0.0
    coul_self: float = 0.0
    shake: float = 0.0
    restraint: float = 0.0

    def values(self) -> List[float]:
        return [getattr(self, f.name) for f in dataclasses.fields(self)]


_ENE_HEADER = ["Time (ps)", "Kinetic energy (kJ/mol)", "Potential energy (kJ/mol)", "Total energy (kJ/mol)",
               "Temperature (K)", "Volume (nm\u00b3)", "Pressure (bar)", "Bond energy", "Angle energy",
               "Improper dihedral", "Proper dihedral", "Lennard-Jones", "Coulomb (real)", "Coulomb (reciprocal)",
               "Coulomb (self)", "SHAKE constraint", "Distance restraint"]


def md_energy_frame(time: float, e_kin: float, e_lj: float, e_crf: float, n_dof: float,
                    volume: float = 0.0, e_bonded: float = 0.0) -> EnergyFrame:
    """An ENERTRJ row from device MD statistics: nonbonded LJ and reaction-field
    energies (Coulomb, real space), kinetic energy and the temperature
    2 E_kin / (n_dof k_B); bonded terms, if the caller has them, in ``e_bonded``."""
    boltz = 0.00831446261815324
    pot = e_lj + e_crf + e_bonded
    denom = n_dof * boltz
    return EnergyFrame(time=time, kinetic=e_kin, potential=pot, total=e_kin + pot,
                       temperature=2.0 * e_kin / denom if denom > 0.0 else 0.0, volume=volume,
                       bond=e_bonded, lj=e_lj, coul_real=e_crf)


class EnergyWriter:
    """ENERTRJ energy trajectory: TITLE, then one row of 17 values per frame
    (EnergyWriter, crates/gromos-io/src/energy.rs:181-316); ``close`` ends the block."""

    def __init__(self, path: str, title: str):
        self._f: TextIO = open(path, "w", encoding="utf-8")
        self._f.write(f"TITLE\n  {title}\nEND\nENERTRJ\n")
        self._header = True
        self.frames = 0

    def write_frame(self, frame: EnergyFrame) -> None:
        if self._header:
            self._f.write("# Block definitions (ENE format):\n")
            for k, name in enumerate(_ENE_HEADER):
                self._f.write(f"# {k:>3} = {name}\n")
            self._header = False
        self._f.write(" ".join(rust_exp(v) for v in frame.values()) + "\n")
        self.frames += 1

    def close(self) -> None:
        if self._f:
            self._f.write("END\n")
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_energy_trajectory(path: str) -> List[EnergyFrame]:
    """Frames of an ENERTRJ file (rows of at least 17 numbers; comments skipped)."""
    frames = []
    inside = False
    for ln in open(path, encoding="utf-8"):
        t = ln.strip()
        if t == "ENERTRJ":
            inside = True
            continue
        if not inside or not t or t.startswith("#"):
            continue
        if t == "END":
            break
        vals = [float(v) for v in t.split()]
        if len(vals) < 17:
            raise ValueError(f"{path}: energy row with {len(vals)} values, expected at least 17")
        frames.append(EnergyFrame(*vals[:17]))
    return frames


class ForceWriter:
    """Force trajectory: TITLE, then per frame TIMESTEP (``%15d%15.9f``) and
    FREEFORCERED (three ``%18.9f`` fields per atom, a ``#`` count line every 10
    atoms), optionally CONSFORCERED (ForceWriter, crates/gromos-io/src/force.rs:44-153)."""

    def __init__(self, path: str, title: str, constraint_forces: bool = False):
        self._f: TextIO = open(path, "w", encoding="utf-8")
        self._f.write(f"TITLE\n  {title}\nEND\n")
        self._cons = constraint_forces
        self.frames = 0

    def _block(self, name: str, f: np.ndarray) -> None:
        out = [name]
        for i, (x, y, z) in enumerate(np.asarray(f, dtype=np.float64).reshape(-1, 3)):
            out.append(f"{x:18.9f}{y:18.9f}{z:18.9f}")
            if (i + 1) % 10 == 0:
                out.append(f"#{i + 1:>10}")
        out.append("END")
        self._f.write("\n".join(out) + "\n")

    def write_frame(self, step: int, time: float, forces: np.ndarray,
                    constraint_forces: Optional[np.ndarray] = None) -> None:
        self._f.write(f"TIMESTEP\n{step:>15}{time:15.9f}\nEND\n")
        self._block("FREEFORCERED", forces)
        if self._cons:
            cf = np.zeros_like(np.asarray(forces, dtype=np.float64)) if constraint_forces is None else constraint_forces
            self._block("CONSFORCERED", cf)
        self.frames += 1

    def close(self) -> None:
        if self._f:
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
