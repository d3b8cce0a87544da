"""CPU: the multi-GPU path is replicas only; its one collective reduces the
ranks' timings (slowest rank) and work (sum of edges).  Two gloo ranks on the
CPU run the same reduction bench.py runs over NCCL."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from dynamicgraphs_scc_b200.replicas import reduce_replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms, edges = reduce_replicas(10.0 * (rank + 1), 1000 * (rank + 1), dist, "cpu")
        out[rank] = (ms, edges)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_slowest_time_and_total_edges():
    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        got = dict(out)
    assert got == {0: (20.0, 3000), 1: (20.0, 3000)}


def test_single_process_keeps_local_values():
    assert reduce_replicas(12.5, 77) == (12.5, 77)
    assert reduce_replicas(12.5, 77, dist) == (12.5, 77)     # not initialised
