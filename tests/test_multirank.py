"""Multi-rank logic of bench.py, run as world_size-2 gloo process groups on CPU:
ranks shard independent gate batches (different seeds), the timing is the
maximum over ranks and the whole-job rate counts every rank's batch."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 + 50.0 * rank           # rank 1 is the slow one
        mx = bench.max_over_ranks(torch, local_ms, "cpu")
        gates, *_ = bench.make_workload(np.random.default_rng(7 + rank), 64)
        out[rank] = (mx, bench.bootstraps(gates), int(gates.sum()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world,
                       start_method="spawn", join=True)
    assert out[0][0] == out[1][0] == 150.0
    # each rank drew its own shard of gates
    assert out[0][2] != out[1][2]
    rate = bench.whole_job_rate(1000, world, 10, 150.0)
    assert abs(rate - 1000 * 2 * 10 / 0.150) < 1e-6


def test_single_process_reduction_is_identity():
    assert bench.max_over_ranks(torch, 12.5, "cpu") == 12.5
    assert bench.bootstraps(np.array([0, 12, 12, 4])) == 6
