"""The multi-rank bookkeeping of bench.py on CPU (gloo, world size 2): every
rank takes the same collective (the max of the per-rank times), and the
job-wide throughput counts the units of all ranks over the slowest rank's
time.  The path has no data-path collective: ranks are replicas."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        ms = 2.0 + rank  # rank 1 is the slow one
        m = bench._max_over_ranks(ms, world, torch.device("cpu"))
        out[rank] = m
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this (threaded) process
    out = mgr.dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1] == 3.0
    # value = units of all ranks / slowest time (weak scaling)
    units = 11.5e9
    assert units * world / (out[0] * 1e-3) == pytest.approx(2 * 11.5e9 / 3e-3)
