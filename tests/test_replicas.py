"""Replica host logic with world_size 2 over gloo on CPU: each rank's seed, the
barrier, the max-over-ranks time and the whole-job throughput."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from filsim_b200.replicas import barrier, job_throughput, max_over_ranks, replica_seed


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        barrier(dist, cuda=False)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        m = max_over_ranks(ms, dist)
        out[rank] = (replica_seed(1002, rank), m, job_throughput(131072, 4, m, world))
        barrier(dist, cuda=False)
    finally:
        dist.destroy_process_group()


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0][0] == 1002 and out[1][0] == 1003
    assert out[0][1] == out[1][1] == 15.0
    assert abs(out[0][2] - 2 * 131072 * 4 / 0.015) < 1e-6 * out[0][2]


def test_single_process_defaults():
    assert max_over_ranks(3.5) == 3.5
    assert job_throughput(100, 2, 1000.0, 1) == 200.0
