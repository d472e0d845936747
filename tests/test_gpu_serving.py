"""Serving: continuous batching of MD jobs with HBM-budget admission.

Each job's final state must equal its standalone run bit for bit, whether it
ran alone or beside others that joined and left during its lifetime.
"""
import numpy as np
import pytest

from gromos_nb import generators as g
from gromos_nb.nonbonded import Forcefield
from gromos_nb.serving import Job, Server, poisson_jobs

pytestmark = pytest.mark.gpu


def standalone(job):
    ff = Forcefield(job.system)
    ff.upload_positions(job.system.pos)
    ff.md_init(job.mass, job.vel, dt=job.dt, settle=True, dist_oh=0.1, dist_hh=g.SPC_DHH)
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
