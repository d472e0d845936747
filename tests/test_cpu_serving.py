"""Job-server scheduling on CPU (no GPU): the device context and the batch
are replaced by fakes that record what the server asks of them.

Covers admission by HBM budget (estimate from the largest bytes-per-atom
seen, re-check with the measured bytes, release and wait when a job does not
fit), first-come-first-served order, chunks that never run a job past its
step count, retirement with the job's final state, and the latency report.
"""
from types import SimpleNamespace

import numpy as np
import pytest

from gromos_nb import serving
from gromos_nb.serving import Job, Server


class FakeForcefield:
    created = []

    def __init__(self, system, device=0):
        self.system = system
        self.n_atoms = system.topo.n_atoms
        self.closed = False
        self.md_inited = False
        FakeForcefield.created.append(self)

    def upload_positions(self, pos):
        pass

    def apply(self, pos, **kw):
        return {"n_pairs_short": 10 * self.n_atoms, "n_pairs_long": 50 * self.n_atoms}

    def md_init(self, mass, vel, **kw):
        self.md_inited = True

    def device_bytes(self):
        return int(self.n_atoms * self.system.bytes_per_atom)

    def md_state(self):
        return np.full((self.n_atoms, 3), float(self.system.tag)), np.zeros((self.n_atoms, 3))

    def md_stats(self):
        return {"steps": 0, "settle_failures": 0, "rollbacks": 0}

    def close(self):
        self.closed = True


class FakeBatch:
    def __init__(self, device=0):
        self.members = []
        self.runs = []          # (steps, tags of the members stepped)

    def add(self, ff):
        assert ff not in self.members
        self.members.append(ff)

    def remove(self, ff):
        self.members.remove(ff)

    def md_run(self, n):
        assert n > 0
        self.runs.append((n, [m.system.tag for m in self.members]))
        return 0.5 * n

    def launches(self):
        return 0

    def record_stats(self):
        return 0, 0.0

    def close(self):
        pass


@pytest.fixture(autouse=True)
def fakes(monkeypatch):
    FakeForcefield.created = []
    monkeypatch.setattr(serving, "Forcefield", FakeForcefield)
    monkeypatch.setattr(serving, "Batch", FakeBatch)


def job(tag, n_atoms, n_steps, bytes_per_atom=1000.0, arrival=0.0):
    system = SimpleNamespace(topo=SimpleNamespace(n_atoms=n_atoms), params=SimpleNamespace(nsnb=5),
                             pos=np.zeros((n_atoms, 3)), tag=tag, bytes_per_atom=bytes_per_atom)
    return Job(job_id=tag, system=system, n_steps=n_steps, mass=np.ones(n_atoms), vel=np.zeros((n_atoms, 3)),
               arrival=arrival)


def drain(srv, limit=100):
    for _ in range(limit):
        if not (srv.queue or srv.resident):
            return
        srv.step()
    raise AssertionError("server did not drain")


def test_budget_admission_and_fifo():
    srv = Server(hbm_budget=2_500_000, chunk_steps=5)
    jobs = [job(0, 1000, 10), job(1, 1000, 20), job(2, 1000, 5)]
    for j in jobs:
        srv.submit(j)
    srv.step()
    assert sorted(srv.resident) == [0, 1]          # 3 x 1 MB would exceed 2.5 MB: job 2 waits
    assert [j.job_id for j in srv.queue] == [2]
    drain(srv)
    assert [j.job_id for j in srv.done] == [0, 2, 1]
    assert srv.max_resident_jobs == 2 and srv.max_resident_bytes <= 2_500_000
    runs = srv.batch.runs
    assert runs[0] == (5, [0, 1]) and runs[1] == (5, [0, 1])
    assert runs[2] == (5, [1, 2])                   # job 2 joins the running batch once job 0 left
    assert sum(n for n, members in runs if 1 in members) == 20
    assert all(ff.closed for ff in FakeForcefield.created)


def test_chunks_stop_at_the_shortest_remaining_job():
    srv = Server(hbm_budget=10**9, chunk_steps=5)
    srv.submit(job(0, 300, 7))
    srv.submit(job(1, 300, 12))
    drain(srv)
    assert [n for n, _ in srv.batch.runs] == [5, 2, 5]
    assert [j.steps_done for j in srv.done] == [7, 12]
    assert srv.steps_run == 12


def test_measured_bytes_above_estimate_release_and_wait():
    srv = Server(hbm_budget=2_500_000, chunk_steps=5)
    srv.submit(job(0, 1000, 10, bytes_per_atom=1000.0))
    srv.submit(job(1, 1000, 5, bytes_per_atom=3000.0))    # estimated 1 MB, measures 3 MB
    srv.step()
    assert list(srv.resident) == [0]
    assert [j.job_id for j in srv.queue] == [1]
    first_try = [ff for ff in FakeForcefield.created if ff.system.tag == 1]
    assert len(first_try) == 1 and first_try[0].closed   # its device memory was released at once
    assert srv.bytes_per_atom == 3000.0                  # later estimates use the larger ratio
    drain(srv)
    assert [j.job_id for j in srv.done] == [0, 1]        # admitted alone once job 0 retired
    assert srv.batch.runs == [(5, [0]), (5, [0]), (5, [1])]


def test_results_latency_and_report():
    srv = Server(hbm_budget=10**9, chunk_steps=4, count_pairs=True)
    jobs = [job(k, 200 + 100 * k, 4 * (k + 1), arrival=0.0) for k in range(3)]
    srv.run(jobs, timeout=30.0)
    rep = srv.report()
    assert rep["jobs"] == 3 and rep["batch_steps"] == 12
    assert 0 < rep["latency_p50_s"] <= rep["latency_p99_s"]
    assert rep["pair_int_per_s"] > 0
    # the wall-time split: set-up, batch steps and retirement are timed, graph recording is the batch's
    assert all(rep[k] >= 0.0 for k in ("host_setup_s", "host_step_s", "host_retire_s", "graph_record_s"))
    assert rep["host_setup_s"] + rep["host_step_s"] + rep["host_retire_s"] <= rep["wall_s"] + 0.05
    assert rep["graph_records"] == 0                      # the fake batch records nothing
    for j in jobs:
        assert j.finished >= j.admitted >= 0.0
        assert np.all(j.result_pos == float(j.job_id))   # each job gets its own final state back
        assert j.pairs_per_step == pytest.approx(10 * j.system.topo.n_atoms + 50 * j.system.topo.n_atoms / 5)
    srv.close()
