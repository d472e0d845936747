"""ctypes binding of libgromos_nb.so (include/gromos_nb.h).

The CUDA library is the only implementation of the nonbonded path in this
package: if it is missing or no GPU is present, every call raises.  There is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
SRC_DIR = os.path.join(os.path.dirname(PKG_DIR), "csrc")
LIB_DIR = os.path.join(PKG_DIR, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libgromos_nb.so")
REPO_ROOT = os.path.dirname(os.path.dirname(PKG_DIR))
HEADER = os.path.join(REPO_ROOT, "include", "gromos_nb.h")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "--shared", "-Xcompiler", "-fPIC"]

GR_OK, GR_ERR_INVALID, GR_ERR_CUDA, GR_ERR_OOM, GR_ERR_STATE = 0, 1, 2, 3, 4
GR_ERR_UNSUPPORTED, GR_ERR_OVERFLOW, GR_ERR_TIMEOUT, GR_ERR_NO_DEVICE = 5, 6, 7, 8
GR_KERNEL_FIXED, GR_KERNEL_PLAIN = 0, 1
GR_EVAL_VIRIAL, GR_EVAL_FORCE_REBUILD, GR_EVAL_NO_DOWNLOAD, GR_EVAL_GRAPH = 1, 2, 4, 8

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class GromosNbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gromos_nb error {status}: {message}")
        self.status = status


class GrPerturbedAtom(C.Structure):
    _fields_ = [("atom", C.c_int32), ("a_iac", C.c_int32), ("b_iac", C.c_int32),
                ("a_charge", C.c_double), ("b_charge", C.c_double),
                ("alpha_lj", C.c_double), ("alpha_crf", C.c_double)]


class GrPerturbedPair(C.Structure):
    _fields_ = [("i", C.c_int32), ("j", C.c_int32), ("a_type", C.c_int32), ("b_type", C.c_int32)]


class GrTopology(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32), ("n_solute_atoms", C.c_int32), ("n_chargegroups", C.c_int32),
        ("n_solute_chargegroups", C.c_int32), ("cg_offsets", _i32p), ("charge", _f64p), ("iac", _i32p),
        ("n_types", C.c_int32), ("lj", _f64p), ("excl_offsets", _i32p), ("excl", _i32p),
        ("o14_offsets", _i32p), ("o14", _i32p), ("energy_group", _i32p), ("n_energy_groups", C.c_int32),
        ("atoms_per_solvent", C.c_int32), ("n_perturbed", C.c_int32),
        ("perturbed", C.POINTER(GrPerturbedAtom)), ("n_perturbed_pairs", C.c_int32),
        ("perturbed_pairs", C.POINTER(GrPerturbedPair)), ("four_pi_eps_i", C.c_double),
    ]


class GrNbParams(C.Structure):
    _fields_ = [
        ("rcutp", C.c_double), ("rcutl", C.c_double), ("skin", C.c_double),
        ("epsilon", C.c_double), ("epsrf", C.c_double), ("kappa", C.c_double),
        ("nsnb", C.c_int32), ("boundary", C.c_int32), ("lam", C.c_double), ("nlam", C.c_int32),
        ("kernel", C.c_int32), ("cluster_size", C.c_int32), ("water_layout", C.c_int32),
        ("list_capacity", C.c_int32),
    ]


class GrResult(C.Structure):
    _fields_ = [
        ("forces", _f64p), ("e_lj", C.c_double), ("e_crf", C.c_double), ("dhdl", C.c_double),
        ("virial", C.c_double * 9), ("egroup_lj", _f64p), ("egroup_crf", _f64p),
        ("n_pairs_short", C.c_int64), ("n_pairs_long", C.c_int64), ("rebuilt", C.c_int32),
    ]


class GrMdParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("settle", C.c_int32), ("dist_oh", C.c_double), ("dist_hh", C.c_double),
                ("temperature", C.c_double), ("tau", C.c_double)]


class GrMdStats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("e_lj", C.c_double), ("e_crf", C.c_double), ("e_kin", C.c_double),
                ("settle_failures", C.c_int32), ("rollbacks", C.c_int32)]


class GrAutotuneResult(C.Structure):
    _fields_ = [("water_layout", C.c_int32), ("cluster_size", C.c_int32), ("n_candidates", C.c_int32),
                ("cand_layout", C.c_int32 * 4), ("cand_cluster_size", C.c_int32 * 4),
                ("cand_ms_per_step", C.c_float * 4)]


class GrJobDesc(C.Structure):
    _fields_ = [("topo", C.POINTER(GrTopology)), ("params", C.POINTER(GrNbParams)), ("box", _f64p),
                ("pos", _f64p), ("mass", _f64p), ("vel", _f64p), ("md", C.POINTER(GrMdParams)),
                ("n_steps", C.c_int64)]


class GrJobStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("steps_done", C.c_int64), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double), ("device_bytes", C.c_int64),
                ("stats", GrMdStats), ("error", C.c_int32), ("message", C.c_char * 160)]


class GrServerStats(C.Structure):
    _fields_ = [("jobs_done", C.c_int64), ("jobs_queued", C.c_int64), ("jobs_running", C.c_int64),
                ("latency_p50_s", C.c_double), ("latency_p99_s", C.c_double), ("resident_bytes", C.c_int64),
                ("max_resident_bytes", C.c_int64), ("max_resident_jobs", C.c_int32), ("batch_steps", C.c_int64),
                ("jobs_failed", C.c_int64), ("jobs_cancelled", C.c_int64), ("jobs_joined_running", C.c_int64)]


GR_JOB_QUEUED, GR_JOB_RUNNING, GR_JOB_DONE, GR_JOB_FAILED, GR_JOB_CANCELLED = 0, 1, 2, 3, 4


# symbol -> (restype, argtypes)
_SIGNATURES = {
    "gr_ctx_create": (C.c_int32, [C.c_int, C.POINTER(C.c_void_p)]),
    "gr_ctx_destroy": (C.c_int32, [C.c_void_p]),
    "gr_last_error": (C.c_char_p, []),
    "gr_ctx_stream": (C.c_void_p, [C.c_void_p]),
    "gr_system_upload": (C.c_int32, [C.c_void_p, C.POINTER(GrTopology)]),
    "gr_set_params": (C.c_int32, [C.c_void_p, C.POINTER(GrNbParams)]),
    "gr_set_box": (C.c_int32, [C.c_void_p, _f64p]),
    "gr_positions_upload": (C.c_int32, [C.c_void_p, _f64p]),
    "gr_positions_device": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "gr_pairlist_build": (C.c_int32, [C.c_void_p]),
    "gr_pairlist_counts": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "gr_pairlist_download": (C.c_int32, [C.c_void_p, _i32p, _i32p, _i32p, _i32p]),
    "gr_pairlist_cg_pairs": (C.c_int32, [C.c_void_p, _i32p, C.POINTER(C.c_int64)]),
    "gr_forces_eval": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(GrResult)]),
    "gr_forces_device": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "gr_result_download": (C.c_int32, [C.c_void_p, C.POINTER(GrResult)]),
    "gr_last_timings": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float)]),
    "gr_last_kernel_timings": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float)]),
    "gr_ctx_launches": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "gr_ffma_peak": (C.c_int32, [C.c_int, C.POINTER(C.c_double)]),
    "gr_md_init": (C.c_int32, [C.c_void_p, _f64p, _f64p, C.POINTER(GrMdParams)]),
    "gr_md_run": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(GrMdStats)]),
    "gr_md_download": (C.c_int32, [C.c_void_p, _f64p, _f64p]),
    "gr_md_stats_get": (C.c_int32, [C.c_void_p, C.POINTER(GrMdStats)]),
    "gr_md_set_temperature": (C.c_int32, [C.c_void_p, C.c_double, C.c_int32]),
    "gr_batch_create": (C.c_int32, [C.c_int, C.POINTER(C.c_void_p)]),
    "gr_batch_destroy": (C.c_int32, [C.c_void_p]),
    "gr_batch_add": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "gr_batch_remove": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "gr_batch_size": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32)]),
    "gr_batch_md_run": (C.c_int32, [C.c_void_p, C.c_int32]),
    "gr_batch_eval": (C.c_int32, [C.c_void_p, C.c_int32]),
    "gr_batch_last_ms": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float)]),
    "gr_batch_launches": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "gr_batch_phase": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "gr_batch_record_stats": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "gr_ctx_device_bytes": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "gr_autotune": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(GrAutotuneResult)]),
    "gr_energy_frames": (C.c_int32, [C.c_void_p, C.c_int32, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]),
    "gr_server_create": (C.c_int32, [C.c_int, C.c_int64, C.c_int32, C.POINTER(C.c_void_p)]),
    "gr_server_destroy": (C.c_int32, [C.c_void_p]),
    "gr_server_submit": (C.c_int32, [C.c_void_p, C.POINTER(GrJobDesc), C.POINTER(C.c_int64)]),
    "gr_server_step": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32)]),
    "gr_server_job": (C.c_int32, [C.c_void_p, C.c_int64, C.POINTER(GrJobStatus), _f64p, _f64p]),
    "gr_server_cancel": (C.c_int32, [C.c_void_p, C.c_int64]),
    "gr_server_release": (C.c_int32, [C.c_void_p, C.c_int64]),
    "gr_server_stats": (C.c_int32, [C.c_void_p, C.POINTER(GrServerStats)]),
    "gr_batch_autotune": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(GrAutotuneResult)]),
    "gr_batch_set_variant": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32]),
    "gr_lj_crf_innerloop_noalloc": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                                C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                                C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_void_p]),
}


def build(verbose: bool = False) -> str:
    """Compile libgromos_nb.so for sm_100a in-tree (nvcc cross-compiles without a GPU)."""
    os.makedirs(LIB_DIR, exist_ok=True)
    src = os.path.join(SRC_DIR, "gromos_nb_all.cu")
    cmd = ["nvcc", *NVCC_FLAGS, "-o", LIB_PATH, src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-4000:])
    if verbose:
        print(" ".join(cmd))
    return LIB_PATH


_lib = None


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != GR_OK:
        msg = lib().gr_last_error()
        raise GromosNbError(status, msg.decode() if msg else "")


def declared_symbols() -> list:
    """Entry points declared in include/gromos_nb.h."""
    import re
    txt = open(HEADER).read()
    pat = r"^\s*(?:gr_status|const char\s*\*|void\s*\*)\s*(gr_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(pat, txt, flags=re.M)))
