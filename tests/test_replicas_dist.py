"""Multi-process replica sharding on CPU (gloo, world_size 2): every replica is
owned by exactly one rank, costs are balanced, and the end-of-run gather
returns every replica's result in order.  No GPU work: the sharded path has no
data-path collective, so the host logic is the whole multi-GPU contract."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ph_brush_b200.replicas import gather_results, partition, replica_cost


def test_partition_covers_every_replica_once():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 10, 96)
    for world in (1, 2, 3, 4, 8):
        b = partition(costs, world)
        assert len(b) == world
        owned = [i for s, e in b for i in range(s, e)]
        assert owned == list(range(96))
        if world > 1:
            loads = [costs[s:e].sum() for s, e in b]
            assert max(loads) <= costs.sum() / world + costs.max() + 1e-9


def test_partition_more_ranks_than_replicas():
    b = partition([1.0, 2.0], 4)
    assert [i for s, e in b for i in range(s, e)] == [0, 1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, costs, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s, e = partition(costs, world)[rank]
    local = [{"replica": i, "rank": rank, "alpha": 0.5 + 0.001 * i} for i in range(s, e)]
    allr = gather_results(local, world)
    if rank == 0:
        out_q.put(allr)
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_gather():
    costs = [replica_cost(n, (32, 32, 96)) for n in np.linspace(1500, 20000, 11).astype(int)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r["replica"] for r in res] == list(range(11))
    assert {r["rank"] for r in res} == {0, 1}
