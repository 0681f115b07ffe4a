"""Multi-rank host logic on CPU (gloo, world size 2).

The scene split is complete, disjoint, balanced and identical on every rank
without any communication; the timed region takes the maximum over ranks, as
bench.py reduces it; a rank that never joins makes the others fail within the
process-group timeout instead of waiting for ever.
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _split_worker(rank, world, port, work, q):
    import torch
    import torch.distributed as dist

    from snow_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    mine = shard.shard(work, world, rank)
    lists = [None] * world
    dist.all_gather_object(lists, mine)
    local = [shard.shard(work, world, r) for r in range(world)]
    t = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, lists, local, float(t.item())))


def _requests():
    """Small independent scenes with their own step counts (requests of a stream)."""
    from snow_b200 import scenes

    scs = scenes.batch_scenes(count=6, lo=300, hi=2500, seed=21, grounded=True)
    return [(sc, 2 + (3 * i) % 5) for i, sc in enumerate(scs)]


def _shard_step_worker(rank, world, port, q):
    """One rank: steps its shard of the requests with the oracle (the CPU
    stand-in for a rank-local batch) and gathers (index, records) on rank 0."""
    import torch.distributed as dist

    from oracle_lib import Oracle
    from snow_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    reqs = _requests()
    mine = shard.shard([sc.n * n for sc, n in reqs], world, rank)
    o = Oracle()
    done = []
    for i in mine:
        sc, n = reqs[i]
        rec = o.setup(sc.particles, sc.dx)
        out, _ = o.step(rec, sc.params(), sc.plane_array(), n)
        done.append((i, out))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(done, gathered, dst=0)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, gathered if rank == 0 else len(done)))


def _lonely_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=3))
        dist.all_reduce(torch.zeros(1))
        q.put((rank, "joined"))
    except Exception as e:  # the rendezvous or the collective times out
        q.put((rank, type(e).__name__))


def _run(target, args, nprocs, limit_s=90):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=target, args=(r,) + args + (q,)) for r in range(nprocs)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in procs:
            item = q.get(timeout=limit_s)
            out[item[0]] = item[1:]
    finally:
        for p in procs:
            p.join(timeout=10)
            if p.is_alive():
                p.kill()
    return out


def test_scene_split_two_ranks():
    from snow_b200 import scenes

    work = [s.n for s in scenes.batch_scenes(count=64, lo=1000, hi=64000, seed=3)]
    out = _run(_split_worker, (2, _free_port(), work), 2)
    (lists0, local0, tmax0), (lists1, local1, tmax1) = out[0], out[1]
    assert lists0 == lists1 == local0 == local1
    assert sorted(i for lst in lists0 for i in lst) == list(range(len(work)))
    loads = [sum(work[i] for i in lst) for lst in lists0]
    assert max(loads) - min(loads) <= max(work)
    assert tmax0 == tmax1 == 11.0


def test_split_edge_cases():
    from snow_b200 import shard

    assert shard.shard([], 2, 0) == [] and shard.shard([], 2, 1) == []
    assert shard.shard([5], 3, 0) == [0] and shard.shard([5], 3, 2) == []
    w = [7, 7, 7, 7]
    assert sorted(shard.shard(w, 2, 0) + shard.shard(w, 2, 1)) == [0, 1, 2, 3]
    assert shard.imbalance([1.0] * 8, 4) == 1.0
    with pytest.raises(ValueError):
        shard.shard(w, 2, 2)
    assert shard.footprint_bytes(10000, 1) < shard.footprint_bytes(10000, 0)


def test_missing_rank_fails_fast():
    # world size 2, only rank 0 starts
    out = _run(_lonely_worker, (2, _free_port()), 1)
    assert out[0][0] != "joined"


def test_sharded_requests_equal_single_rank(oracle):
    """Each of two ranks steps its share of a request stream (work = particles x
    steps); the union gathered on rank 0 is the single-rank result, record for
    record (no data crosses ranks, so nothing may change)."""
    reqs = _requests()
    out = _run(_shard_step_worker, (2, _free_port()), 2, limit_s=120)
    gathered = out[0][0]
    got = dict(item for part in gathered for item in part)
    assert sorted(got) == list(range(len(reqs)))
    assert out[1][0] > 0, "both ranks hold work"
    for i, (sc, n) in enumerate(reqs):
        rec = oracle.setup(sc.particles, sc.dx)
        want, _ = oracle.step(rec, sc.params(), sc.plane_array(), n)
        assert np.array_equal(got[i], want), i
