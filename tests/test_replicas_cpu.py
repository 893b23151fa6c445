"""The N-GPU bench path (replicas, no data-path collective) on CPU: two gloo
ranks time different amounts of work, the reported time is the maximum over
ranks, and each rank draws its own molecules."""

import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import bench
    from fml_b200 import synthetic
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        local_ms = 10.0 * (rank + 1)  # rank 1 is the slow replica
        out[rank] = bench.max_over_ranks(torch, dist, local_ms, torch.device("cpu"))
        b = synthetic.generate(8, nmax=12, seed=bench.replica_seed(7, rank))
        out[2 + rank] = float(np.sum(b.coords))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    world = 2
    out = mp.get_context("spawn").Array("d", 4)
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    assert out[0] == out[1] == 20.0
    assert out[2] != out[3]  # replicas hold different problems
