"""World-size-2 gloo tests on CPU of the multi-rank plumbing: independent
systems are assigned to ranks with no data-path collective; the timing is
the max over ranks; summaries are gathered at rank 0."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from psblas3_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, work, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = shard.assign(work, world)[rank]
    local = sum(work[i] for i in mine)  # stands in for this rank's solve time
    tmax = shard.max_over_ranks(local, world)
    total = shard.sum_over_ranks(len(mine), world)
    got = shard.gather_to_root(sorted(mine), world, rank)
    if rank == 0:
        q.put((tmax, total, got))
    dist.barrier()
    dist.destroy_process_group()


def test_assign_is_balanced_and_complete():
    work = [5, 1, 1, 1, 4, 2, 2, 3, 8, 1]
    parts = shard.assign(work, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(work)))
    loads = [sum(work[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(work)
    assert shard.assign(work, 3) == parts  # deterministic: every rank agrees


def test_two_rank_gloo_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    work = [float(w) for w in (9, 7, 5, 3, 2, 2, 1)]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, work, q)) for r in range(2)]
    for p in procs:
        p.start()
    tmax, total, got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = shard.assign(work, 2)
    assert tmax == max(sum(work[i] for i in p) for p in parts)
    assert total == len(work)
    assert sorted(i for g in got for i in g) == list(range(len(work)))
