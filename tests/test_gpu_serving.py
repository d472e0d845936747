"""Serving: continuous batching of MD jobs with HBM-budget admission.

Each job's final state must equal its standalone run bit for bit, whether it
ran alone or beside others that joined and left during its lifetime.
"""
import numpy as np
import pytest

from gromos_nb import generators as g
from gromos_nb.nonbonded import Forcefield
from gromos_nb.serving import NativeServer, Server, poisson_jobs

pytestmark = pytest.mark.gpu


def standalone(job):
    ff = Forcefield(job.system)
    ff.upload_positions(job.system.pos)
    ff.md_init(job.mass, job.vel, dt=job.dt, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH,
               temperature=job.temperature, tau=job.tau)
    ff.md_run(job.n_steps)
    x, v = ff.md_state()
    ff.close()
    return x, v


def small_jobs():
    jobs = poisson_jobs(5, rate=40.0, seed=9, waters=(300, 900), steps=(60, 120), solute_prob=0.4,
                        solute_atoms=(20, 40), rc=1.0, nsnb=5)
    # two jobs at once, the others while those run
    for j, t in zip(jobs, (0.0, 0.0, 0.004, 0.008, 0.03)):
        j.arrival = t
    return jobs


def test_serving_results_equal_standalone():
    jobs = small_jobs()
    srv = Server(hbm_budget=150 * 2 ** 30, chunk_steps=5, count_pairs=True)
    srv.run(jobs, timeout=300)
    rep = srv.report()
    srv.close()
    assert rep["jobs"] == len(jobs)
    assert rep["max_resident_jobs"] >= 2        # jobs overlapped on the device
    assert rep["joined_running"] >= 1           # at least one joined a batch that was already stepping
    assert 0 < rep["latency_p50_s"] <= rep["latency_p99_s"]
    for job in jobs:
        x, v = standalone(job)
        assert job.steps_done == job.n_steps
        assert np.array_equal(job.result_pos, x) and np.array_equal(job.result_vel, v), job.job_id


def test_serving_respects_small_budget():
    jobs = small_jobs()
    for j in jobs:
        j.arrival = 0.0                          # all at once: admission alone limits residency
    probe = Forcefield(jobs[0].system)
    probe.upload_positions(jobs[0].system.pos)
    probe.md_init(jobs[0].mass, jobs[0].vel)
    per_atom = probe.device_bytes() / jobs[0].system.topo.n_atoms
    probe.close()
    budget = int(per_atom * 2.2 * max(j.system.topo.n_atoms for j in jobs))
    srv = Server(hbm_budget=budget, chunk_steps=5)
    srv.run(jobs, timeout=300)
    rep = srv.report()
    srv.close()
    assert rep["jobs"] == len(jobs)
    assert rep["max_resident_bytes"] <= budget or rep["max_resident_jobs"] == 1
    assert rep["max_resident_jobs"] < len(jobs)
    for job in jobs[:2]:
        x, v = standalone(job)
        assert np.array_equal(job.result_pos, x) and np.array_equal(job.result_vel, v)


def test_native_server_results_equal_standalone():
    """gr_server_*: continuous batching in the library; each job equals its standalone run."""
    jobs = small_jobs()
    srv = NativeServer(hbm_budget=150 * 2 ** 30, chunk_steps=5)
    srv.run(jobs, timeout=300)
    st = srv.stats()
    srv.close()
    assert st["jobs_done"] == len(jobs)
    assert st["max_resident_jobs"] >= 2
    assert st["jobs_joined_running"] >= 1       # at least one joined a batch that was already stepping
    assert 0 < st["latency_p50_s"] <= st["latency_p99_s"]
    for job in jobs:
        x, v = standalone(job)
        assert job.steps_done == job.n_steps
        assert np.array_equal(job.result_pos, x) and np.array_equal(job.result_vel, v), job.job_id


def test_native_server_respects_small_budget():
    jobs = small_jobs()
    for j in jobs:
        j.arrival = 0.0
    srv = NativeServer(hbm_budget=2 ** 30, chunk_steps=5)   # measure the footprint of one job first
    srv.submit(jobs[0])
    srv.step()
    per_job = srv.status(jobs[0])["device_bytes"]
    srv.close()
    budget = int(per_job * 2.5)
    srv = NativeServer(hbm_budget=budget, chunk_steps=5)
    srv.run(jobs, timeout=300)
    st = srv.stats()
    srv.close()
    assert st["jobs_done"] == len(jobs)
    assert st["max_resident_jobs"] < len(jobs)
    assert st["max_resident_bytes"] <= budget


def test_native_server_bad_job_fails_alone():
    """A job with invalid parameters and one above the whole budget fail; the others finish unchanged."""
    from gromos_nb import _lib
    from gromos_nb.nonbonded import make_params
    jobs = small_jobs()
    for j in jobs:
        j.arrival = 0.0
    srv = NativeServer(hbm_budget=150 * 2 ** 30, chunk_steps=5)
    bad = make_params(jobs[1].system.params, "fixed")
    bad.rcutl = 0.5 * bad.rcutp                      # rcutl < rcutp: rejected by gr_set_params
    for k, j in enumerate(jobs):
        srv.submit(j, params=bad if k == 1 else None)
    while srv.step() or srv.stats()["jobs_queued"]:
        pass
    st = srv.stats()
    assert st["jobs_failed"] == 1 and st["jobs_done"] == len(jobs) - 1
    s1 = srv.status(jobs[1])
    assert s1["state"] == _lib.GR_JOB_FAILED and s1["error"] == _lib.GR_ERR_INVALID and "rcut" in s1["message"]
    for k, job in enumerate(jobs):
        if k == 1:
            continue
        full = srv.status(job, fetch=True)
        x, v = standalone(job)
        assert full["state"] == _lib.GR_JOB_DONE
        assert np.array_equal(full["pos"], x) and np.array_equal(full["vel"], v), job.job_id
    srv.close()
    tiny = NativeServer(hbm_budget=1 << 20, chunk_steps=5)   # 1 MiB: no job fits
    tiny.submit(jobs[0])
    assert tiny.step() == 0
    s0 = tiny.status(jobs[0])
    assert s0["state"] == _lib.GR_JOB_FAILED and s0["error"] == _lib.GR_ERR_OOM
    tiny.close()


def test_native_server_cancel():
    """Cancelling a running and a queued job frees them; the rest equal their standalone runs."""
    from gromos_nb import _lib
    jobs = small_jobs()
    srv = NativeServer(hbm_budget=150 * 2 ** 30, chunk_steps=5)
    for j in jobs[:3]:
        srv.submit(j)
    srv.step()                                       # all three resident
    assert srv.stats()["jobs_running"] == 3
    srv.submit(jobs[3])
    srv.cancel(jobs[0])                              # running
    srv.cancel(jobs[3])                              # still queued
    with pytest.raises(RuntimeError):
        srv.cancel(jobs[3])                          # already ended
    while srv.step() or srv.stats()["jobs_queued"]:
        pass
    st = srv.stats()
    assert st["jobs_cancelled"] == 2 and st["jobs_done"] == 2 and st["resident_bytes"] == 0
    assert srv.status(jobs[0])["state"] == _lib.GR_JOB_CANCELLED and srv.status(jobs[0])["steps_done"] == 5
    for job in jobs[1:3]:
        full = srv.status(job, fetch=True)
        x, v = standalone(job)
        assert np.array_equal(full["pos"], x) and np.array_equal(full["vel"], v), job.job_id
    srv.close()
