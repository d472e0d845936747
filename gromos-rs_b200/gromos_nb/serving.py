"""Continuous-batching MD job server on one GPU.

Jobs (a system, a number of MD steps, initial velocities) arrive over time.
The server keeps every admitted job resident on the device -- coordinates,
velocities, pairlists, force caches -- and steps all resident jobs together
through one :class:`~gromos_nb.nonbonded.Batch` (one CUDA graph launch per MD
step for all of them).  Between chunks of steps it admits queued jobs while
their device memory fits the HBM budget, and retires finished jobs, whose
memory is freed at once.  A job that arrives while others run joins the
running batch at the next chunk boundary: that is continuous batching, not a
queue in front of a single-job runner.

Admission: a job is admitted when the resident bytes plus its estimated
bytes stay within ``hbm_budget``.  The estimate is ``n_atoms`` times the
largest device-bytes-per-atom ratio seen so far (``bytes_per_atom`` until the
first job has been measured); after admission the job is accounted with its
measured bytes (``gr_ctx_device_bytes``).  A job whose measured bytes would
exceed the budget is released again and waits.

Every job's trajectory is bit-identical to a standalone run of the same job
(fixed-point force sums, the same kernels per member), whatever else runs
beside it.
"""
from __future__ import annotations

import dataclasses
import time
from collections import deque
from typing import Deque, Dict, List, Optional

import numpy as np

import ctypes as C

from . import _lib, generators
from .nonbonded import Batch, Forcefield, _TopologyStruct, make_params
from .system import System


@dataclasses.dataclass
class Job:
    job_id: int
    system: System
    n_steps: int
    mass: np.ndarray
    vel: np.ndarray
    dt: float = 0.002
    temperature: float = 300.0        # Berendsen bath (K)
    tau: float = 0.1                  # bath coupling time (ps); < 0 runs NVE
    arrival: float = 0.0              # seconds since the server started
    # filled in by the server
    admitted: Optional[float] = None
    finished: Optional[float] = None
    steps_done: int = 0
    result_pos: Optional[np.ndarray] = None
    result_vel: Optional[np.ndarray] = None
    stats: Optional[Dict] = None
    device_bytes: int = 0
    pairs_per_step: float = 0.0

    @property
    def latency(self) -> float:
        return (self.finished - self.arrival) if self.finished is not None else float("nan")


class Server:
    """One GPU, one batch of resident jobs, admission by device memory."""

    def __init__(self, hbm_budget: int, device: int = 0, chunk_steps: int = 5, bytes_per_atom: float = 8192.0,
                 count_pairs: bool = False):
        self.budget = int(hbm_budget)
        self.device = device
        self.chunk = max(1, int(chunk_steps))
        self.bytes_per_atom = float(bytes_per_atom)
        self.count_pairs = count_pairs
        self.batch = Batch(device)
        self.queue: Deque[Job] = deque()
        self.resident: Dict[int, tuple] = {}   # job_id -> (job, Forcefield)
        self.done: List[Job] = []
        self.resident_bytes = 0
        self.t0 = time.perf_counter()
        self.gpu_ms = 0.0
        self.steps_run = 0                     # batch steps
        self.pair_steps = 0.0                  # atom-pair interactions evaluated (when counted)
        self.sim_ps = 0.0                      # simulated time summed over jobs
        self.max_resident_jobs = 0
        self.max_resident_bytes = 0
        self.joined_running = 0                # jobs admitted into a batch that was already stepping
        # host time split of the serving loop (wall-clock seconds)
        self.setup_s = 0.0                     # job contexts: upload, first pairlist, MD set-up
        self.step_s = 0.0                      # batch steps, graph recording included
        self.retire_s = 0.0                    # results read back, contexts released

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, job: Job) -> None:
        self.queue.append(job)

    # ---- admission / retirement
    def _admit(self) -> None:
        t0 = time.perf_counter()
        try:
            self._admit_jobs()
        finally:
            self.setup_s += time.perf_counter() - t0

    def _admit_jobs(self) -> None:
        while self.queue:
            job = self.queue[0]
            est = int(job.system.topo.n_atoms * self.bytes_per_atom)
            if self.resident and self.resident_bytes + est > self.budget:
                return
            ff = Forcefield(job.system, device=self.device)
            ff.upload_positions(job.system.pos)
            if self.count_pairs:
                r = ff.apply(job.system.pos, count_pairs=True, download_forces=False)
                nsnb = max(1, job.system.params.nsnb)
                job.pairs_per_step = r["n_pairs_short"] + r["n_pairs_long"] / nsnb
                ff.upload_positions(job.system.pos)
            ff.md_init(job.mass, job.vel, dt=job.dt, settle=True, dist_oh=0.1, dist_hh=generators.SPC_DHH,
                       temperature=job.temperature, tau=job.tau)
            nbytes = ff.device_bytes()
            self.bytes_per_atom = max(self.bytes_per_atom if self.resident or self.done else 0.0,
                                      nbytes / max(1, job.system.topo.n_atoms))
            if self.resident and self.resident_bytes + nbytes > self.budget:
                ff.close()                   # does not fit after all: wait for memory
                return
            self.queue.popleft()
            if self.resident and self.steps_run > 0:
                self.joined_running += 1
            self.batch.add(ff)
            job.admitted = self.now()
            job.device_bytes = nbytes
            self.resident[job.job_id] = (job, ff)
            self.resident_bytes += nbytes
            self.max_resident_jobs = max(self.max_resident_jobs, len(self.resident))
            self.max_resident_bytes = max(self.max_resident_bytes, self.resident_bytes)

    def _retire(self) -> None:
        t0 = time.perf_counter()
        try:
            self._retire_jobs()
        finally:
            self.retire_s += time.perf_counter() - t0

    def _retire_jobs(self) -> None:
        for jid in [j for j, (job, _) in self.resident.items() if job.steps_done >= job.n_steps]:
            job, ff = self.resident.pop(jid)
            self.batch.remove(ff)
            job.result_pos, job.result_vel = ff.md_state()
            job.stats = ff.md_stats()
            job.finished = self.now()
            ff.close()
            self.resident_bytes -= job.device_bytes
            self.done.append(job)

    # ---- one scheduling round
    def step(self) -> int:
        """Admit, run one chunk of MD steps for every resident job, retire. Returns steps run."""
        self._admit()
        if not self.resident:
            return 0
        n = min(self.chunk, min(job.n_steps - job.steps_done for job, _ in self.resident.values()))
        t0 = time.perf_counter()
        self.gpu_ms += self.batch.md_run(n)
        self.step_s += time.perf_counter() - t0
        self.steps_run += n
        for job, _ in self.resident.values():
            job.steps_done += n
            self.pair_steps += job.pairs_per_step * n
            self.sim_ps += job.dt * n
        self._retire()
        return n

    def run(self, jobs: List[Job], timeout: float = 600.0) -> None:
        """Serve ``jobs`` arriving at their ``arrival`` times (seconds from now)."""
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        self.t0 = time.perf_counter()
        while pending or self.queue or self.resident:
            t = self.now()
            if t > timeout:
                raise TimeoutError("serving run exceeded its time limit")
            while pending and pending[0].arrival <= t:
                self.submit(pending.popleft())
            if self.step() == 0 and pending and not self.queue:
                time.sleep(max(0.0, min(pending[0].arrival - self.now(), 0.01)))

    # ---- report
    def report(self) -> Dict:
        records, record_s = self.batch.record_stats()
        lat = np.array([j.latency for j in self.done])
        wall = max((j.finished for j in self.done), default=0.0)
        return {
            "jobs": len(self.done),
            "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "wall_s": wall,
            "gpu_ms": self.gpu_ms,
            "batch_steps": self.steps_run,
            "pair_int_per_s": self.pair_steps / wall if wall > 0 and self.count_pairs else None,
            "ns_per_day_aggregate": self.sim_ps * 1e-3 / wall * 86400.0 if wall > 0 else None,
            "launches": self.batch.launches(),
            "max_resident_jobs": self.max_resident_jobs,
            "joined_running": self.joined_running,
            "max_resident_bytes": self.max_resident_bytes,
            # where the wall time goes: job set-up, batch steps (device time plus the step
            # graphs recorded on membership changes), retirement; the rest is waiting for arrivals
            "host_setup_s": self.setup_s,
            "host_step_s": self.step_s,
            "host_retire_s": self.retire_s,
            "graph_records": records,
            "graph_record_s": record_s,
        }

    def close(self) -> None:
        for job, ff in self.resident.values():
            self.batch.remove(ff)
            ff.close()
        self.resident.clear()
        self.batch.close()


def poisson_jobs(n_jobs: int, rate: float, seed: int, waters=(300, 20000), steps=(100, 2000),
                 solute_prob: float = 0.5, solute_atoms=(50, 500), rc: float = 1.4, nsnb: int = 5,
                 T: float = 300.0, tau: float = 0.1) -> List[Job]:
    """Seeded Poisson arrival stream of MD jobs: uniform water counts and
    lengths, an optional seeded solute (as in the batched REMD replicas),
    each coupled to a Berendsen bath at ``T`` with coupling time ``tau`` ps
    (the synthetic starting structures release potential energy; without a
    bath a job heats far above ``T`` within a picosecond).  The solutes are
    single-atom charge groups, which stay consistent with the charge-group
    cutoff over the jobs' up to 2,000 steps (see solvated_solute_system)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for k in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        nw = int(rng.integers(waters[0], waters[1] + 1))
        ns = int(rng.integers(solute_atoms[0], solute_atoms[1] + 1)) if rng.random() < solute_prob else 0
        sseed = seed * 1000 + k
        if ns >= 3:
            s = generators.solvated_solute_system(nw, ns, seed=sseed, rc=rc, nsnb=nsnb, single_atom_cgs=True)
        else:
            s = generators.spc_water_system(nw, box=generators.box_for_waters(nw), seed=sseed, rcutp=rc,
                                            rcutl=rc, nsnb=nsnb)
        m = generators.masses(s)
        v = generators.maxwell_velocities(m, T, sseed + 7)
        jobs.append(Job(job_id=k, system=s, n_steps=int(rng.integers(steps[0], steps[1] + 1)), mass=m, vel=v,
                        temperature=T, tau=tau, arrival=t))
    return jobs


class NativeServer:
    """The same continuous-batching server in the library (``gr_server_*``).

    Jobs are handed to the C ABI with all their inputs; admission, batching
    and retirement run in C++.  ``run`` serves jobs arriving at their
    ``arrival`` times like :meth:`Server.run`.
    """

    def __init__(self, hbm_budget: int, device: int = 0, chunk_steps: int = 5):
        self._L = _lib.lib()
        h = C.c_void_p()
        _lib.check(self._L.gr_server_create(device, int(hbm_budget), int(chunk_steps), C.byref(h)))
        self._h = h
        self.ids: Dict[int, int] = {}       # Job.job_id -> server job id
        self.jobs: Dict[int, Job] = {}

    def submit(self, job: Job, params=None) -> int:
        """Queue ``job``; ``params`` overrides the system's nonbonded parameters (a gr_nb_params)."""
        s = job.system
        topo = _TopologyStruct(s.topo)
        params = make_params(s.params, "fixed") if params is None else params
        box = np.ascontiguousarray(s.box, dtype=np.float64)
        pos = np.ascontiguousarray(s.pos, dtype=np.float64)
        mass = np.ascontiguousarray(job.mass, dtype=np.float64)
        vel = np.ascontiguousarray(job.vel, dtype=np.float64)
        md = _lib.GrMdParams(job.dt, 1, 0.1, generators.SPC_DHH, job.temperature, job.tau)
        f64 = C.POINTER(C.c_double)
        desc = _lib.GrJobDesc(C.pointer(topo.struct), C.pointer(params), box.ctypes.data_as(f64),
                              pos.ctypes.data_as(f64), mass.ctypes.data_as(f64), vel.ctypes.data_as(f64),
                              C.pointer(md), int(job.n_steps))
        jid = C.c_int64(0)
        _lib.check(self._L.gr_server_submit(self._h, C.byref(desc), C.byref(jid)))
        self.ids[job.job_id] = int(jid.value)
        self.jobs[job.job_id] = job
        return int(jid.value)

    def step(self) -> int:
        n = C.c_int32(0)
        _lib.check(self._L.gr_server_step(self._h, C.byref(n)))
        return int(n.value)

    def status(self, job: Job, fetch: bool = False) -> Dict:
        st = _lib.GrJobStatus()
        n3 = job.system.topo.n_atoms * 3
        pos = np.zeros(n3) if fetch else None
        vel = np.zeros(n3) if fetch else None
        f64 = C.POINTER(C.c_double)
        _lib.check(self._L.gr_server_job(self._h, self.ids[job.job_id], C.byref(st),
                                         None if pos is None else pos.ctypes.data_as(f64),
                                         None if vel is None else vel.ctypes.data_as(f64)))
        out = {"state": st.state, "steps_done": st.steps_done, "t_submit": st.t_submit, "t_admit": st.t_admit,
               "t_done": st.t_done, "device_bytes": st.device_bytes, "error": st.error,
               "message": st.message.decode(errors="replace")}
        if fetch:
            out["pos"], out["vel"] = pos.reshape(-1, 3), vel.reshape(-1, 3)
        return out

    def cancel(self, job: Job) -> None:
        _lib.check(self._L.gr_server_cancel(self._h, self.ids[job.job_id]))

    def stats(self) -> Dict:
        st = _lib.GrServerStats()
        _lib.check(self._L.gr_server_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def run(self, jobs: List[Job], timeout: float = 600.0) -> None:
        """Serve ``jobs`` arriving at their ``arrival`` times (seconds from now); finished jobs get
        ``result_pos`` / ``result_vel`` / ``steps_done`` filled in."""
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        t0 = time.perf_counter()
        open_jobs = []
        while True:
            t = time.perf_counter() - t0
            if t > timeout:
                raise TimeoutError("serving run exceeded its time limit")
            while pending and pending[0].arrival <= t:
                j = pending.popleft()
                self.submit(j)
                open_jobs.append(j)
            running = self.step()
            for j in list(open_jobs):
                st = self.status(j)
                if st["state"] in (_lib.GR_JOB_FAILED, _lib.GR_JOB_CANCELLED):
                    j.finished = t0 + st["t_done"]
                    open_jobs.remove(j)
                elif st["state"] == _lib.GR_JOB_DONE:
                    full = self.status(j, fetch=True)
                    j.result_pos, j.result_vel, j.steps_done = full["pos"], full["vel"], full["steps_done"]
                    j.finished = t0 + full["t_done"]
                    open_jobs.remove(j)
            if not pending and not open_jobs:
                return
            if running == 0 and pending and not open_jobs:
                time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.01)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.gr_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
