"""Multi-rank host logic on CPU: world size 2 over gloo (no GPU).

The GPU path is replicas only; what spans ranks is bookkeeping -- the
max-over-ranks time, the summed work and the deterministic assignment of
whole systems to ranks -- and that is what these tests exercise.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gromos_nb.replicas import shard_by_work


def test_shard_by_work_balanced_and_complete():
    work = [8000, 500, 7000, 3000, 3000, 1200, 6500, 900, 4000]
    shards = shard_by_work(work, 3)
    assert sorted(i for s in shards for i in s) == list(range(len(work)))
    loads = [sum(work[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(work)            # LPT bound
    assert shard_by_work(work, 3) == shards                # deterministic on every rank
    assert shard_by_work(work, 1) == [list(range(len(work)))]
    with pytest.raises(ValueError):
        shard_by_work(work, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from gromos_nb.replicas import aggregate, shard_by_work

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        work = [5.0, 1.0, 3.0, 2.0, 4.0]
        mine = shard_by_work(work, world)[rank]
        local_units = sum(work[i] for i in mine)
        local_ms = 10.0 + rank                               # rank 1 is the slow one
        q.put((rank, mine, aggregate(local_ms, local_units, device="cpu")))
    finally:
        dist.destroy_process_group()


def test_aggregate_max_time_sum_work_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert sorted(out[0][1] + out[1][1]) == [0, 1, 2, 3, 4]
    for _, _, (ms, units) in out:
        assert ms == 11.0 and units == 15.0
