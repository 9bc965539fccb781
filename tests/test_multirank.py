"""Multi-process paths on CPU (gloo, world_size 2).

The hot path does not shard within an instance; bench.py runs one replica
per GPU, each contracting its own seeded batch, and reports the max time
over ranks.  These tests cover that host logic: per-rank workloads are
disjoint and deterministic, and the max-over-ranks reduction is what every
rank sees.
"""
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
    import torch
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    insts = bench.make_instances(8, 2024 + 7919 * rank)
    sig = float(sum(d["beta"] for d in insts))
    t = torch.tensor([1.0 + rank, 10.0 - rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    sigs = [None] * world
    dist.all_gather_object(sigs, sig)
    q.put((rank, t.tolist(), sigs))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
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
    for rank, t, sigs in out:
        assert t == [2.0, 10.0]                 # max over ranks
        assert sigs[0] != sigs[1]                # disjoint per-rank batches
