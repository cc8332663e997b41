"""Multi-GPU plumbing on CPU: jobs shard across ranks with no data exchange,
every rank computes the same plan, and timings reduce by max (gloo, 2 ranks)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch

    from par2rust_b200 import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        jobs = W.batch_256(n_jobs=48)
        mine = W.shard_jobs(jobs, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = torch.tensor([float(sum(W.job_cost(jobs[i]) for i in mine))], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, gathered, float(t.item()), [W.job_cost(j) for j in jobs]))
    finally:
        dist.destroy_process_group()


def test_jobs_shard_disjoint_and_balanced():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    gathered = res[0][1]
    assert gathered == res[1][1], "ranks disagree on the plan"
    allj = sorted(i for part in gathered for i in part)
    costs = res[0][3]
    assert allj == list(range(len(costs))), "every job exactly once"
    loads = [sum(costs[i] for i in part) for part in gathered]
    assert res[0][2] == res[1][2] == float(max(loads))
    assert max(loads) <= 1.05 * sum(loads) / world + max(costs)


def test_single_rank_takes_everything():
    from par2rust_b200 import workloads as W

    jobs = W.batch_256(n_jobs=16)
    assert W.shard_jobs(jobs, 0, 1) == list(range(len(jobs)))
