"""Host-side mirror of gromos-rs's nonbonded interface, backed by the CUDA library.

Names follow the reference so that callers and tests read the same:

* :class:`CRFParameters` -- ``CRFParameters::new``
  (crates/gromos-forces/src/nonbonded/params.rs:61-97)
* :class:`PairlistContainer` -- cutoffs, skin and NSNB
  (crates/gromos-core/src/pairlist.rs:59-126)
* :class:`Forcefield` -- ``Forcefield::apply``'s nonbonded part
  (crates/gromos-integrators/src/algorithms/forcefield.rs:226-1020): one
  :meth:`Forcefield.apply` per MD step, pairlist rebuilt every NSNB calls,
  twin-range long-range forces cached between rebuilds.
* :func:`lj_crf_innerloop` -- the C-ABI stub ``rust_lj_crf_innerloop``
  (crates/gromos-core/src/ffi.rs:55-103) with a body.

Every evaluation runs on the GPU through include/gromos_nb.h; errors from the
library raise :class:`GromosNbError`.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import GromosNbError, check  # noqa: F401  (re-exported)
from .system import NonbondedParams, System, Topology

KERNELS = {"fixed": _lib.GR_KERNEL_FIXED, "plain": _lib.GR_KERNEL_PLAIN}


@dataclasses.dataclass
class CRFParameters:
    crf_cut: float
    crf_2cut3i: float
    crf_cut3i: float
    cutoff_sq: float

    @staticmethod
    def new(cutoff: float, epsilon: float, rf_epsilon: float, rf_kappa: float) -> "CRFParameters":
        kc = rf_kappa * cutoff
        kc2 = kc * kc
        crf = (2.0 * (epsilon - rf_epsilon) * (1.0 + kc) - rf_epsilon * kc2) / (
            (epsilon + 2.0 * rf_epsilon) * (1.0 + kc) + rf_epsilon * kc2)
        crf_cut3i = crf * (1.0 / (cutoff * cutoff * cutoff))
        return CRFParameters((1.0 - crf / 2.0) / cutoff, crf_cut3i / 2.0, crf_cut3i, cutoff * cutoff)


@dataclasses.dataclass
class PairlistContainer:
    short_range_cutoff: float
    long_range_cutoff: float
    skin: float = 0.0
    update_frequency: int = 5


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


class _TopologyStruct:
    """gr_topology plus the arrays it points into (kept alive here)."""

    def __init__(self, topo: Topology):
        t = topo.normalized()
        self.t = t
        s = _lib.GrTopology()
        s.n_atoms, s.n_solute_atoms = t.n_atoms, t.n_solute_atoms
        s.n_chargegroups, s.n_solute_chargegroups = t.n_cg, t.n_solute_cg
        s.cg_offsets, s.charge, s.iac = _p(t.cg_offsets, C.c_int32), _p(t.charge, C.c_double), _p(t.iac, C.c_int32)
        s.n_types, s.lj = t.n_types, _p(t.lj, C.c_double)
        s.excl_offsets, s.excl = _p(t.excl_off, C.c_int32), _p(t.excl, C.c_int32)
        s.o14_offsets, s.o14 = _p(t.o14_off, C.c_int32), _p(t.o14, C.c_int32)
        s.energy_group = _p(t.egroup, C.c_int32)
        s.n_energy_groups = int(t.n_egroups)
        s.atoms_per_solvent = t.atoms_per_solvent
        s.four_pi_eps_i = t.four_pi_eps_i
        self.pert = None
        self.pairs = None
        if t.pert_idx is not None and t.n_pert > 0:
            atoms = np.nonzero(t.pert_idx >= 0)[0]
            arr = (_lib.GrPerturbedAtom * len(atoms))()
            for n, a in enumerate(atoms):
                k = int(t.pert_idx[a])
                arr[n] = _lib.GrPerturbedAtom(int(a), int(t.pert_a_iac[k]), int(t.pert_b_iac[k]),
                                              float(t.pert_a_q[k]), float(t.pert_b_q[k]),
                                              float(t.pert_alpha_lj[k]), float(t.pert_alpha_crf[k]))
            self.pert = arr
            s.n_perturbed = len(atoms)
            s.perturbed = C.cast(arr, C.POINTER(_lib.GrPerturbedAtom))
        if t.pp_i is not None and t.n_pert_pairs > 0:
            arr = (_lib.GrPerturbedPair * t.n_pert_pairs)()
            for n in range(t.n_pert_pairs):
                arr[n] = _lib.GrPerturbedPair(int(t.pp_i[n]), int(t.pp_j[n]), int(t.pp_a_type[n]), int(t.pp_b_type[n]))
            self.pairs = arr
            s.n_perturbed_pairs = t.n_pert_pairs
            s.perturbed_pairs = C.cast(arr, C.POINTER(_lib.GrPerturbedPair))
        self.struct = s


def make_params(p: NonbondedParams, kernel: str = "fixed", cluster_size: int = 0,
                water_layout: int = 0, list_capacity: int = 0) -> _lib.GrNbParams:
    q = _lib.GrNbParams()
    q.rcutp, q.rcutl, q.skin = p.rcutp, p.rcutl, p.skin
    q.epsilon, q.epsrf, q.kappa = p.epsilon, p.epsrf, p.kappa
    q.nsnb, q.boundary, q.lam, q.nlam = p.nsnb, p.boundary, p.lam, p.nlam
    q.kernel = KERNELS[kernel]
    q.cluster_size = cluster_size
    q.water_layout = water_layout
    q.list_capacity = list_capacity
    return q


class Forcefield:
    """Nonbonded ``Forcefield`` on one GPU.

    ``Forcefield(system)`` uploads the topology, parameters and box; the first
    :meth:`apply` builds the pairlist (md.rs:864-867 builds it before the
    first step), later calls rebuild it every ``nsnb`` calls.
    """

    def __init__(self, system: System, kernel: str = "fixed", device: int = 0, cluster_size: int = 0,
                 water_layout: int = 0, list_capacity: int = 0):
        L = _lib.lib()
        self._L = L
        self.system = system
        self.kernel = kernel
        self.device = device
        h = C.c_void_p()
        check(L.gr_ctx_create(device, C.byref(h)))
        self._h = h
        self._topo = _TopologyStruct(system.topo)
        check(L.gr_system_upload(h, C.byref(self._topo.struct)))
        self._params = make_params(system.params, kernel, cluster_size, water_layout, list_capacity)
        check(L.gr_set_params(h, C.byref(self._params)))
        self.set_box(system.box)
        self.n_atoms = system.topo.n_atoms
        self.G = max(1, int(system.topo.n_egroups))
        self.crf = CRFParameters.new(system.params.rcutl, system.params.epsilon, system.params.epsrf,
                                     system.params.kappa)
        self.pairlist = PairlistContainer(system.params.rcutp, system.params.rcutl, system.params.skin,
                                          system.params.nsnb)

    # ---- set-up
    def set_params(self, **changes) -> None:
        """Change parameters (e.g. ``list_capacity``, ``water_layout``); the next step rebuilds,
        except when only ``list_capacity`` changes (then the new size applies from the next rebuild)."""
        for k, v in changes.items():
            setattr(self._params, k, v)
        check(self._L.gr_set_params(self._h, C.byref(self._params)))

    def set_box(self, box) -> None:
        b = np.ascontiguousarray(box, dtype=np.float64)
        check(self._L.gr_set_box(self._h, _p(b, C.c_double)))

    def upload_positions(self, pos) -> None:
        x = np.ascontiguousarray(pos, dtype=np.float64)
        if x.shape != (self.n_atoms, 3):
            raise ValueError(f"positions must be ({self.n_atoms}, 3)")
        check(self._L.gr_positions_upload(self._h, _p(x, C.c_double)))

    # ---- evaluation
    def apply(self, pos=None, virial: bool = True, force_rebuild: bool = False, count_pairs: bool = True,
              download_forces: bool = True, out: Optional[np.ndarray] = None, graph: bool = False) -> Dict:
        """One Forcefield::apply.  ``out`` (n_atoms, 3) float64, ideally in
        pinned memory, receives the forces without a per-call allocation;
        ``graph`` replays the step from a recorded CUDA graph."""
        if pos is not None:
            self.upload_positions(pos)
        flags = (_lib.GR_EVAL_VIRIAL if virial else 0) | (_lib.GR_EVAL_FORCE_REBUILD if force_rebuild else 0)
        if graph:
            flags |= _lib.GR_EVAL_GRAPH
        if out is not None:
            if out.shape != (self.n_atoms, 3) or out.dtype != np.float64 or not out.flags.c_contiguous:
                raise ValueError("out must be a C-contiguous float64 (n_atoms, 3) array")
            f = out
        else:
            f = np.zeros((self.n_atoms, 3)) if download_forces else None
        glj = np.zeros((self.G, self.G))
        gcrf = np.zeros((self.G, self.G))
        r = _lib.GrResult()
        r.forces = _p(f, C.c_double)
        r.egroup_lj, r.egroup_crf = _p(glj, C.c_double), _p(gcrf, C.c_double)
        r.n_pairs_short = 0 if count_pairs else -1
        check(self._L.gr_forces_eval(self._h, flags, C.byref(r)))
        return {"forces": f, "e_lj": r.e_lj, "e_crf": r.e_crf, "dhdl": r.dhdl,
                "virial": np.asarray(list(r.virial)).reshape(3, 3), "egroup_lj": glj, "egroup_crf": gcrf,
                "n_pairs_short": r.n_pairs_short, "n_pairs_long": r.n_pairs_long, "rebuilt": bool(r.rebuilt)}

    def eval_async(self, force_rebuild: bool = False, graph: bool = False) -> None:
        """Evaluate without reading results back (device-resident pipelines)."""
        flags = _lib.GR_EVAL_VIRIAL | _lib.GR_EVAL_NO_DOWNLOAD | (_lib.GR_EVAL_FORCE_REBUILD if force_rebuild else 0)
        if graph:
            flags |= _lib.GR_EVAL_GRAPH
        check(self._L.gr_forces_eval(self._h, flags, None))

    def energy_frames(self, frames: np.ndarray, boxes: Optional[np.ndarray] = None, groups: bool = False) -> dict:
        """LJ and CRF energies of every configuration in ``frames`` (n_frames, n_atoms, 3), each with
        a fresh pairlist (``gr_energy_frames``); ``boxes`` (n_frames, 3) or None for the current box.
        With ``groups`` the (n_frames, G, G) energy-group matrices are returned too."""
        n = self.system.topo.n_atoms
        fr = np.ascontiguousarray(frames, dtype=np.float64).reshape(-1, n, 3)
        nf = fr.shape[0]
        bx = None if boxes is None else np.ascontiguousarray(boxes, dtype=np.float64).reshape(nf, 3)
        e_lj, e_crf = np.zeros(nf), np.zeros(nf)
        G = int(self.system.topo.n_egroups)
        glj = np.zeros((nf, G, G)) if groups else None
        gcrf = np.zeros((nf, G, G)) if groups else None
        f64 = C.POINTER(C.c_double)
        ptr = lambda a: None if a is None else a.ctypes.data_as(f64)
        check(self._L.gr_energy_frames(self._h, nf, ptr(fr), ptr(bx), ptr(e_lj), ptr(e_crf), ptr(glj), ptr(gcrf)))
        out = {"e_lj": e_lj, "e_crf": e_crf}
        if groups:
            out["egroup_lj"], out["egroup_crf"] = glj, gcrf
        return out

    def timings(self) -> List[float]:
        ms = (C.c_float * 5)()
        check(self._L.gr_last_timings(self._h, ms))
        return list(ms)

    def kernel_timings(self) -> List[float]:
        """[water prep, short-range water kernel, long-range water kernel] in ms of the last
        kernel-by-kernel evaluation (-1 where a kernel did not run)."""
        ms = (C.c_float * 3)()
        check(self._L.gr_last_kernel_timings(self._h, ms))
        return list(ms)

    def launches(self) -> int:
        n = C.c_int64(0)
        check(self._L.gr_ctx_launches(self._h, C.byref(n)))
        return int(n.value)

    def stream(self) -> int:
        return int(self._L.gr_ctx_stream(self._h) or 0)

    def positions_device_ptr(self) -> int:
        p = C.c_void_p()
        check(self._L.gr_positions_device(self._h, C.byref(p)))
        return int(p.value)

    def forces_device_ptr(self) -> int:
        p = C.c_void_p()
        check(self._L.gr_forces_device(self._h, C.byref(p)))
        return int(p.value)

    # ---- MD (leap-frog + SETTLE around the force call, device resident)
    def md_init(self, mass, vel=None, dt: float = 0.002, settle: bool = True, dist_oh: float = 0.1,
                dist_hh: float = 0.1633, temperature: float = 300.0, tau: float = -1.0) -> None:
        """Positions are those of the last upload; ``vel`` are v(-dt/2) (None = zero).
        ``tau`` >= 0 couples to a Berendsen bath at ``temperature`` (tau < 0: NVE)."""
        m = np.ascontiguousarray(mass, dtype=np.float64)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        if m.shape != (self.n_atoms,) or (v is not None and v.shape != (self.n_atoms, 3)):
            raise ValueError("mass must be (n_atoms,), vel (n_atoms, 3)")
        self._md_mass, self._md_vel = m, v
        mp = _lib.GrMdParams(dt, 1 if settle else 0, dist_oh, dist_hh, temperature, tau)
        self.temperature = temperature
        check(self._L.gr_md_init(self._h, _p(m, C.c_double), _p(v, C.c_double), C.byref(mp)))

    def md_set_temperature(self, t0: float, rescale_velocities: bool = True) -> None:
        check(self._L.gr_md_set_temperature(self._h, float(t0), 1 if rescale_velocities else 0))
        self.temperature = t0

    def md_run(self, n_steps: int) -> Dict:
        st = _lib.GrMdStats()
        check(self._L.gr_md_run(self._h, int(n_steps), C.byref(st)))
        return {"steps": st.steps, "e_lj": st.e_lj, "e_crf": st.e_crf, "e_kin": st.e_kin,
                "settle_failures": st.settle_failures, "rollbacks": st.rollbacks}

    def md_run_async(self, n_steps: int) -> None:
        check(self._L.gr_md_run(self._h, int(n_steps), None))

    def md_stats(self) -> Dict:
        st = _lib.GrMdStats()
        check(self._L.gr_md_stats_get(self._h, C.byref(st)))
        return {"steps": st.steps, "e_lj": st.e_lj, "e_crf": st.e_crf, "e_kin": st.e_kin,
                "settle_failures": st.settle_failures, "rollbacks": st.rollbacks}

    def result(self) -> Dict:
        """Results of the last evaluation (e.g. after a batch evaluation), without evaluating."""
        f = np.zeros((self.n_atoms, 3))
        glj = np.zeros((self.G, self.G))
        gcrf = np.zeros((self.G, self.G))
        r = _lib.GrResult()
        r.forces = _p(f, C.c_double)
        r.egroup_lj, r.egroup_crf = _p(glj, C.c_double), _p(gcrf, C.c_double)
        check(self._L.gr_result_download(self._h, C.byref(r)))
        return {"forces": f, "e_lj": r.e_lj, "e_crf": r.e_crf, "dhdl": r.dhdl,
                "virial": np.asarray(list(r.virial)).reshape(3, 3), "egroup_lj": glj, "egroup_crf": gcrf}

    def autotune(self, periods: int = 2, cache: Optional[str] = None) -> Dict:
        """Pick the fastest solvent kernel variant by timing pairlist periods (forces only).
        With ``cache`` (a JSON file path) a choice made earlier for the same system shape on the
        same kind of GPU is applied without timing, and a new choice is stored."""
        from . import tuning

        def tune():
            r = _lib.GrAutotuneResult()
            check(self._L.gr_autotune(self._h, int(periods), C.byref(r)))
            return _autotune_dict(r)

        if cache is None:
            return dict(tune(), cached=False)
        key = tuning.cache_key(tuning.device_signature(self.device), [tuning.system_signature(self.system)])
        return tuning.tune_cached(tuning.TuningCache(cache), key, tune,
                                  lambda layout, width: self.set_params(water_layout=layout, cluster_size=width))

    def device_bytes(self) -> int:
        n = C.c_int64(0)
        check(self._L.gr_ctx_device_bytes(self._h, C.byref(n)))
        return int(n.value)

    @property
    def handle(self):
        return self._h

    def md_state(self):
        x = np.zeros((self.n_atoms, 3))
        v = np.zeros((self.n_atoms, 3))
        check(self._L.gr_md_download(self._h, _p(x, C.c_double), _p(v, C.c_double)))
        return x, v

    # ---- pairlist
    def build_pairlist(self) -> None:
        check(self._L.gr_pairlist_build(self._h))

    def pairlist_lists(self) -> List[np.ndarray]:
        """solute_short, solute_long, solvent_short, solvent_long as sorted (n, 2) int32."""
        counts = (C.c_int64 * 4)()
        check(self._L.gr_pairlist_counts(self._h, counts))
        out = [np.zeros((int(counts[k]), 2), dtype=np.int32) for k in range(4)]
        check(self._L.gr_pairlist_download(self._h, *[_p(a, C.c_int32) for a in out]))
        return out

    def cg_pairs(self) -> np.ndarray:
        n = C.c_int64(0)
        check(self._L.gr_pairlist_cg_pairs(self._h, None, C.byref(n)))
        out = np.zeros((n.value, 3), dtype=np.int32)
        n2 = C.c_int64(n.value)
        check(self._L.gr_pairlist_cg_pairs(self._h, _p(out, C.c_int32), C.byref(n2)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            batch = getattr(self, "_batch", None)
            if batch is not None:  # a batch member leaves its batch first
                batch.remove(self)
            check(self._L.gr_ctx_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _autotune_dict(r) -> Dict:
    cands = [{"water_layout": r.cand_layout[k], "cluster_size": r.cand_cluster_size[k],
              "ms_per_step": float(r.cand_ms_per_step[k])} for k in range(r.n_candidates)]
    return {"water_layout": r.water_layout, "cluster_size": r.cluster_size, "candidates": cands}


class Batch:
    """Members (Forcefield objects) stepped together: one CUDA graph launch per MD step.

    Replaces stepping REMD replicas / FEP windows one after the other
    (replica.rs:163, :315; remd.rs:168).  Members stay owned by the caller;
    each member's results are bit-identical to its standalone run.
    """

    def __init__(self, device: int = 0):
        self._L = _lib.lib()
        self.device = device
        h = C.c_void_p()
        check(self._L.gr_batch_create(device, C.byref(h)))
        self._h = h
        self.members: List["Forcefield"] = []

    def add(self, ff: "Forcefield") -> None:
        check(self._L.gr_batch_add(self._h, ff.handle))
        self.members.append(ff)
        ff._batch = self

    def remove(self, ff: "Forcefield") -> None:
        check(self._L.gr_batch_remove(self._h, ff.handle))
        self.members.remove(ff)
        ff._batch = None

    def __len__(self) -> int:
        return len(self.members)

    def md_run(self, n_steps: int) -> float:
        """MD steps of every member; returns the device time in ms."""
        check(self._L.gr_batch_md_run(self._h, int(n_steps)))
        return self.last_ms()

    def eval(self, virial: bool = True) -> float:
        """One force evaluation of every member (results: ``member.result()``); device ms."""
        check(self._L.gr_batch_eval(self._h, _lib.GR_EVAL_VIRIAL if virial else 0))
        return self.last_ms()

    def autotune(self, periods: int = 2, cache: Optional[str] = None) -> Dict:
        """gr_batch_autotune over the members; ``cache`` as in Forcefield.autotune, keyed by the
        members' system shapes in order."""
        from . import tuning

        def tune():
            r = _lib.GrAutotuneResult()
            check(self._L.gr_batch_autotune(self._h, int(periods), C.byref(r)))
            return _autotune_dict(r)

        if cache is None:
            return dict(tune(), cached=False)
        key = tuning.cache_key(tuning.device_signature(self.device),
                               [tuning.system_signature(m.system) for m in self.members])
        return tuning.tune_cached(tuning.TuningCache(cache), key, tune,
                                  lambda layout, width: check(self._L.gr_batch_set_variant(self._h, layout, width)))

    def last_ms(self) -> float:
        ms = C.c_float(0.0)
        check(self._L.gr_batch_last_ms(self._h, C.byref(ms)))
        return float(ms.value)

    def launches(self) -> int:
        n = C.c_int64(0)
        check(self._L.gr_batch_launches(self._h, C.byref(n)))
        return int(n.value)

    def record_stats(self) -> Tuple[int, float]:
        """(step graphs recorded so far, host seconds spent recording them)."""
        n, sec = C.c_int64(0), C.c_double(0.0)
        check(self._L.gr_batch_record_stats(self._h, C.byref(n), C.byref(sec)))
        return int(n.value), float(sec.value)

    def phase(self) -> Tuple[int, int]:
        """(phase, period): the step of their pairlist period (NSNB = period) the members
        take at the next batch step, 0 when every member rebuilds there, -1 when the batch
        is empty or its members stand at different steps (``gr_batch_phase``)."""
        ph, per = C.c_int32(0), C.c_int32(0)
        check(self._L.gr_batch_phase(self._h, C.byref(ph), C.byref(per)))
        return int(ph.value), int(per.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.gr_batch_destroy(self._h)
            self._h = None
            for ff in self.members:
                ff._batch = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ffma_peak(device: int = 0) -> float:
    """Measured FP32 FMA operations per second of the device (one FFMA = one op)."""
    v = C.c_double(0.0)
    check(_lib.lib().gr_ffma_peak(device, C.byref(v)))
    return float(v.value)


def lj_crf_innerloop(positions, charges, iac, pairlist, lj_params, crf: CRFParameters, box=None,
                     parallel: bool = False):
    """``lj_crf_innerloop`` over an explicit atom-pair list, on the GPU.

    Same arguments as the reference C-ABI stub (ffi.rs:55-103): FP32
    positions/charges, (c6, c12) per type pair, per-atom nearest image
    (box=None -> vacuum).  ``parallel`` calls the ``rust_lj_crf_innerloop_parallel``
    replacement (ffi.rs:105-145) instead.  Returns (forces (N,3) float32, e_lj,
    e_crf, virial 3x3).
    """
    L = _lib.lib()
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    q = np.ascontiguousarray(charges, dtype=np.float32)
    ia = np.ascontiguousarray(iac, dtype=np.uint32)
    pl = np.ascontiguousarray(pairlist, dtype=np.uint32)
    lj = np.ascontiguousarray(lj_params, dtype=np.float64)
    n_types = int(round(np.sqrt(lj.size // 2)))
    n = pos.shape[0]
    f = np.zeros((n, 3), dtype=np.float32)
    e = np.zeros(2)
    v = np.zeros(9)
    bx = np.ascontiguousarray(box if box is not None else np.zeros(3), dtype=np.float64)
    fn = L.gr_lj_crf_innerloop_parallel if parallel else L.gr_lj_crf_innerloop
    fn.restype = C.c_int32
    u32 = C.POINTER(C.c_uint32)
    fn.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), u32, C.c_uint32, u32, C.c_uint32,
                   C.POINTER(C.c_double), C.c_uint32, C.POINTER(C.c_double), C.c_uint32, C.c_double, C.c_double,
                   C.c_double, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    check(fn(_p(pos, C.c_float), _p(q, C.c_float), _p(ia, C.c_uint32), n, _p(pl, C.c_uint32), pl.shape[0],
             _p(lj, C.c_double), n_types, _p(bx, C.c_double), 0 if box is None else 1, crf.crf_cut,
             crf.crf_2cut3i, crf.crf_cut3i, _p(f, C.c_float), _p(e, C.c_double), _p(v, C.c_double)))
    return f, e[0], e[1], v.reshape(3, 3)
