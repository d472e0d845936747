"""ctypes binding of the FP64 oracle (oracle/libgromos_oracle.so).

TEST INFRASTRUCTURE ONLY: the oracle is the checker that the CUDA library is
compared against.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg load it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "lib", "libgromos_oracle.so")

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class OrcTopology(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32), ("n_solute_atoms", C.c_int32), ("n_cg", C.c_int32),
        ("n_solute_cg", C.c_int32), ("cg_offsets", _i32p), ("charge", _f64p), ("iac", _i32p),
        ("n_types", C.c_int32), ("lj", _f64p), ("excl_off", _i32p), ("excl", _i32p),
        ("o14_off", _i32p), ("o14", _i32p), ("egroup", _i32p), ("n_egroups", C.c_int32),
        ("pert_idx", _i32p), ("pert_a_iac", _i32p), ("pert_b_iac", _i32p), ("pert_a_q", _f64p),
        ("pert_b_q", _f64p), ("pert_alpha_lj", _f64p), ("pert_alpha_crf", _f64p),
        ("n_pert", C.c_int32), ("n_pert_pairs", C.c_int32), ("pp_i", _i32p), ("pp_j", _i32p),
        ("pp_a_type", _i32p), ("pp_b_type", _i32p), ("atoms_per_solvent", C.c_int32),
    ]


class OrcParams(C.Structure):
    _fields_ = [
        ("rcutp", C.c_double), ("rcutl", C.c_double), ("skin", C.c_double),
        ("epsilon", C.c_double), ("epsrf", C.c_double), ("kappa", C.c_double),
        ("four_pi_eps_i", C.c_double), ("nsnb", C.c_int32), ("boundary", C.c_int32),
        ("box", C.c_double * 3), ("algorithm", C.c_int32), ("virial", C.c_int32),
        ("lam", C.c_double), ("nlam", C.c_int32), ("nthreads", C.c_int32),
    ]


class OrcResult(C.Structure):
    _fields_ = [
        ("e_lj", C.c_double), ("e_crf", C.c_double), ("dhdl", C.c_double),
        ("virial", C.c_double * 9), ("forces", _f64p), ("egroup_lj", _f64p), ("egroup_crf", _f64p),
    ]


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_oracle()
        L = C.CDLL(LIB_PATH)
        L.orc_pairlist_build.restype = C.c_void_p
        L.orc_pairlist_build.argtypes = [C.POINTER(OrcTopology), C.POINTER(OrcParams), _f64p]
        L.orc_pairlist_size.restype = C.c_int64
        L.orc_pairlist_size.argtypes = [C.c_void_p, C.c_int]
        L.orc_pairlist_get.argtypes = [C.c_void_p, C.c_int, _i32p]
        L.orc_pairlist_free.argtypes = [C.c_void_p]
        L.orc_ff_create.restype = C.c_void_p
        L.orc_ff_create.argtypes = [C.POINTER(OrcTopology), C.POINTER(OrcParams), _f64p]
        L.orc_ff_apply.argtypes = [C.c_void_p, _f64p, C.POINTER(OrcResult)]
        L.orc_ff_apply.restype = C.c_int
        L.orc_ff_destroy.argtypes = [C.c_void_p]
        L.orc_ff_set_box.argtypes = [C.c_void_p, _f64p]
        L.orc_crf_params.argtypes = [C.c_double] * 4 + [_f64p]
        L.orc_lambda_params.argtypes = [C.c_double] * 8 + [C.c_int, _f64p]
        L.orc_perturbed_pair.argtypes = [_f64p] + [C.c_double] * 8 + [_f64p, _f64p, C.c_double, _f64p]
        L.orc_md_run.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, C.POINTER(OrcMdParams), C.c_int, _f64p, _f64p]
        L.orc_md_run.restype = C.c_int
        _lib = L
    return _lib


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


class _Keep:
    """Holds the NumPy arrays a ctypes struct points into."""

    def __init__(self, topo):
        self.t = topo.normalized()


def make_topology(topo):
    k = _Keep(topo)
    t = k.t
    s = OrcTopology()
    s.n_atoms, s.n_solute_atoms = t.n_atoms, t.n_solute_atoms
    s.n_cg, s.n_solute_cg = t.n_cg, t.n_solute_cg
    s.cg_offsets, s.charge, s.iac = _p(t.cg_offsets, C.c_int32), _p(t.charge, C.c_double), _p(t.iac, C.c_int32)
    s.n_types, s.lj = t.n_types, _p(t.lj, C.c_double)
    s.excl_off, s.excl = _p(t.excl_off, C.c_int32), _p(t.excl, C.c_int32)
    s.o14_off, s.o14 = _p(t.o14_off, C.c_int32), _p(t.o14, C.c_int32)
    s.egroup, s.n_egroups = _p(t.egroup, C.c_int32), int(t.n_egroups)
    s.pert_idx = _p(t.pert_idx, C.c_int32)
    s.pert_a_iac, s.pert_b_iac = _p(t.pert_a_iac, C.c_int32), _p(t.pert_b_iac, C.c_int32)
    s.pert_a_q, s.pert_b_q = _p(t.pert_a_q, C.c_double), _p(t.pert_b_q, C.c_double)
    s.pert_alpha_lj, s.pert_alpha_crf = _p(t.pert_alpha_lj, C.c_double), _p(t.pert_alpha_crf, C.c_double)
    s.n_pert, s.n_pert_pairs = t.n_pert, t.n_pert_pairs
    s.pp_i, s.pp_j = _p(t.pp_i, C.c_int32), _p(t.pp_j, C.c_int32)
    s.pp_a_type, s.pp_b_type = _p(t.pp_a_type, C.c_int32), _p(t.pp_b_type, C.c_int32)
    s.atoms_per_solvent = t.atoms_per_solvent
    return s, k


def make_params(sysm, virial=True, nthreads=0):
    p = sysm.params
    q = OrcParams()
    q.rcutp, q.rcutl, q.skin = p.rcutp, p.rcutl, p.skin
    q.epsilon, q.epsrf, q.kappa = p.epsilon, p.epsrf, p.kappa
    q.four_pi_eps_i = sysm.topo.four_pi_eps_i
    q.nsnb, q.boundary = p.nsnb, p.boundary
    for k in range(3):
        q.box[k] = float(sysm.box[k])
    q.algorithm, q.virial = p.algorithm, 1 if virial else 0
    q.lam, q.nlam, q.nthreads = p.lam, p.nlam, nthreads
    return q


def crf_params(cutoff, eps, epsrf, kappa):
    out = np.zeros(4)
    lib().orc_crf_params(cutoff, eps, epsrf, kappa, _p(out, C.c_double))
    return out


def pairlist(sysm, algorithm=None, nthreads=0):
    """The four reference lists [(i, j)] as int32 arrays (n, 2)."""
    t, keep = make_topology(sysm.topo)
    q = make_params(sysm, nthreads=nthreads)
    if algorithm is not None:
        q.algorithm = algorithm
    pos = np.ascontiguousarray(sysm.pos, dtype=np.float64)
    h = lib().orc_pairlist_build(C.byref(t), C.byref(q), _p(pos, C.c_double))
    out = []
    for w in range(4):
        n = lib().orc_pairlist_size(h, w)
        a = np.zeros((n, 2), dtype=np.int32)
        if n:
            lib().orc_pairlist_get(h, w, _p(a, C.c_int32))
        out.append(a)
    lib().orc_pairlist_free(h)
    del keep
    return out


class OrcMdParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("settle", C.c_int32), ("dist_oh", C.c_double), ("dist_hh", C.c_double),
                ("temperature", C.c_double), ("tau", C.c_double)]


class OracleForcefield:
    """Forcefield::apply restated in FP64 (nonbonded only); one apply() per MD step."""

    def __init__(self, sysm, virial=True, nthreads=0):
        self.sys = sysm
        self.t, self.keep = make_topology(sysm.topo)
        self.q = make_params(sysm, virial=virial, nthreads=nthreads)
        pos = np.ascontiguousarray(sysm.pos, dtype=np.float64)
        self.h = lib().orc_ff_create(C.byref(self.t), C.byref(self.q), _p(pos, C.c_double))
        self.G = max(1, int(sysm.topo.n_egroups))

    def apply(self, pos=None):
        pos = np.ascontiguousarray(self.sys.pos if pos is None else pos, dtype=np.float64)
        n = pos.shape[0]
        f = np.zeros((n, 3))
        glj = np.zeros((self.G, self.G))
        gcrf = np.zeros((self.G, self.G))
        r = OrcResult()
        r.forces, r.egroup_lj, r.egroup_crf = _p(f, C.c_double), _p(glj, C.c_double), _p(gcrf, C.c_double)
        rc = lib().orc_ff_apply(self.h, _p(pos, C.c_double), C.byref(r))
        assert rc == 0
        return {"forces": f, "e_lj": r.e_lj, "e_crf": r.e_crf, "dhdl": r.dhdl,
                "virial": np.asarray(list(r.virial)).reshape(3, 3), "egroup_lj": glj, "egroup_crf": gcrf}

    def md_run(self, pos, vel, mass, n_steps, dt=0.002, settle=True, dist_oh=0.1, dist_hh=0.1633,
               temperature=300.0, tau=-1.0):
        """n_steps MD steps (leap-frog + Berendsen + SETTLE) in FP64; returns (pos, vel, stats)."""
        x = np.ascontiguousarray(pos, dtype=np.float64).copy()
        v = np.ascontiguousarray(vel, dtype=np.float64).copy()
        m = np.ascontiguousarray(mass, dtype=np.float64)
        mp = OrcMdParams(dt, 1 if settle else 0, dist_oh, dist_hh, temperature, tau)
        ke = C.c_double(0.0)
        e = np.zeros(2)
        fails = lib().orc_md_run(self.h, _p(x, C.c_double), _p(v, C.c_double), _p(m, C.c_double), C.byref(mp),
                                 int(n_steps), C.byref(ke), _p(e, C.c_double))
        return x, v, {"e_kin": ke.value, "e_lj": e[0], "e_crf": e[1], "settle_failures": fails}

    def close(self):
        if self.h:
            lib().orc_ff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
