"""Replica-exchange controller host logic on CPU (no GPU): fake replicas
report fixed potential energies and record the temperatures they are given.

Covers the Metropolis test delta = (beta_1 - beta_2)(E_2 - E_1), accepted
when a uniform number is below min(1, exp(-delta)) (remd.rs:259-308), the
odd-even pairing (remd.rs:211-226), the ladder bookkeeping of swapped
temperatures and the velocity-rescale flag of accepted exchanges
(replica.rs:355-371), and the same exchanges with the replicas sharded over
two gloo ranks.
"""
import numpy as np
import pytest

from gromos_nb.remd import KB, ReplicaExchange


class FakeReplica:
    def __init__(self, energy, n_atoms=3):
        self.energy = float(energy)
        self.n_atoms = n_atoms
        self.set_calls = []

    def md_stats(self):
        return {"e_lj": self.energy, "e_crf": 0.0}

    def md_set_temperature(self, t, rescale_velocities=True):
        self.set_calls.append((float(t), bool(rescale_velocities)))


class FakeBatch:
    def __init__(self):
        self.steps = 0

    def md_run(self, n):
        self.steps += n
        return 0.0


class FixedDraws:
    """Stands in for the seeded generator: returns the given uniform numbers in order."""

    def __init__(self, draws):
        self.draws = list(draws)

    def random(self):
        return self.draws.pop(0)


def test_initial_ladder_assignment_without_rescale():
    reps = [FakeReplica(0.0) for _ in range(3)]
    rx = ReplicaExchange(reps, [400.0, 300.0, 350.0], exchange_interval=10, batch=FakeBatch())
    assert [rx.temperature_of(r) for r in range(3)] == [400.0, 300.0, 350.0]
    assert [r.set_calls for r in reps] == [[(400.0, False)], [(300.0, False)], [(350.0, False)]]
    assert rx.replica_at(0) == 1 and rx.replica_at(2) == 0


def test_metropolis_threshold_is_exp_minus_delta():
    t0, t1 = 300.0, 310.0
    b0, b1 = 1.0 / (KB * t0), 1.0 / (KB * t1)
    delta = 0.5
    reps = [FakeReplica(0.0), FakeReplica(delta / (b0 - b1))]   # E_1 - E_0 gives exactly delta
    rx = ReplicaExchange(reps, [t0, t1], exchange_interval=5, scheme="sequential", batch=FakeBatch())
    p = np.exp(-delta)
    rx.rng = FixedDraws([p + 1e-6, p - 1e-6])
    rx.run(5)                                   # draw just above the acceptance probability
    assert rx.accepts.tolist() == [0] and rx.attempts.tolist() == [1]
    assert [rx.temperature_of(r) for r in range(2)] == [t0, t1]
    rx.run(5)                                   # just below: accepted, temperatures swapped
    assert rx.accepts.tolist() == [1] and rx.attempts.tolist() == [2]
    assert [rx.temperature_of(r) for r in range(2)] == [t1, t0]
    assert reps[0].set_calls[-1] == (t1, True) and reps[1].set_calls[-1] == (t0, True)


def test_downhill_exchanges_accepted_and_odd_even_alternates():
    temps = [300.0, 350.0, 400.0]
    # colder replicas hold higher energies, so the first two attempts are downhill (delta < 0)
    reps = [FakeReplica(-100.0), FakeReplica(-200.0), FakeReplica(-300.0)]
    b = FakeBatch()
    rx = ReplicaExchange(reps, temps, exchange_interval=10, batch=b, seed=3)
    rx.run(20)
    assert b.steps == 20
    assert rx.attempts.tolist() == [1, 1]       # pair (1,2) first, then (0,1)
    assert rx.accepts.tolist() == [1, 1]
    # (1,2) swaps replicas 1 and 2; (0,1) then swaps replica 0 with replica 2
    assert [rx.temperature_of(r) for r in range(3)] == [350.0, 400.0, 300.0]
    assert rx.statistics()["acceptance"] == [1.0, 1.0]


def test_uphill_exchanges_never_accepted():
    temps = [300.0, 330.0, 360.0, 390.0]
    reps = [FakeReplica(1e6 * k) for k in range(4)]   # hotter replicas far higher in energy
    rx = ReplicaExchange(reps, temps, exchange_interval=4, batch=FakeBatch(), seed=9)
    rx.run(40)
    assert rx.accepts.tolist() == [0, 0, 0]
    assert rx.attempts.tolist() == [5, 5, 5]
    assert [rx.temperature_of(r) for r in range(4)] == temps


def test_equilibration_steps_skip_attempts():
    reps = [FakeReplica(-10.0), FakeReplica(-20.0)]
    rx = ReplicaExchange(reps, [300.0, 320.0], exchange_interval=5, scheme="sequential", batch=FakeBatch(),
                         equilibration_steps=10)
    rx.run(20)                                  # attempts at steps 10, 15, 20; not at 5
    assert rx.attempts.tolist() == [3]


def test_bad_arguments_are_rejected():
    with pytest.raises(ValueError):
        ReplicaExchange([FakeReplica(0.0)], [300.0], batch=FakeBatch())
    with pytest.raises(ValueError):
        ReplicaExchange([FakeReplica(0.0), FakeReplica(0.0, n_atoms=6)], [300.0, 310.0], batch=FakeBatch())
    with pytest.raises(ValueError):
        ReplicaExchange([FakeReplica(0.0), FakeReplica(0.0)], [300.0, 310.0], scheme="random", batch=FakeBatch())


ENERGIES = [-100.0, -300.0, -50.0, -400.0, -500.0, -20.0]
LADDER = [300.0, 320.0, 340.0, 360.0, 380.0, 400.0]


def _single_process_run():
    reps = [FakeReplica(e) for e in ENERGIES]
    rx = ReplicaExchange(reps, LADDER, exchange_interval=10, batch=FakeBatch(), seed=5)
    rx.run(80)
    return rx.statistics(), {g: r.set_calls for g, r in enumerate(reps)}


def _rank_worker(rank, world, port, q):
    import datetime
    import os

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = [g for g in range(len(ENERGIES)) if g % world == rank]     # non-contiguous shards
        reps = [FakeReplica(ENERGIES[g]) for g in mine]
        rx = ReplicaExchange(reps, LADDER, exchange_interval=10, batch=FakeBatch(), seed=5, global_ids=mine)
        rx.run(80)
        q.put((rank, rx.statistics(), {g: r.set_calls for g, r in zip(mine, reps)}))
    finally:
        dist.destroy_process_group()


def test_exchange_across_ranks_matches_one_process():
    """Replicas sharded over two gloo ranks: the energies are summed over the ranks at each attempt,
    every rank takes the same decisions, and each replica receives the temperatures it would get with
    all replicas in one process."""
    import socket

    import torch.multiprocessing as mp
    want_stats, want_calls = _single_process_run()
    assert 0 < sum(want_stats["accepts"]) < sum(want_stats["attempts"])   # both outcomes occur
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    calls = {}
    for _, stats, c in out:
        assert stats == want_stats
        calls.update(c)
    assert calls == want_calls
