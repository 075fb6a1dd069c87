"""Replicas-only multi-GPU path of bench.py, host logic on CPU with gloo (world size 2):
the timing reduction is the max over ranks and the reported value is the whole-job
(weak-scaling) throughput. No collective touches the data path."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, r, lr = bench.dist_env()
        assert (w, r, lr) == (world, rank, rank)
        ms = 10.0 + 5.0 * rank                   # rank 1 is the slow one
        ms_max = bench.max_over_ranks(ms, w)
        out[rank] = (ms_max, bench.weak_scaling_value(w, 100, 5e-4, ms_max))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_reduction():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this (threaded) test process
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1]
    ms_max, value = out[0]
    assert ms_max == 15.0
    assert value == pytest.approx(2 * 100 * 5e-4 / 0.015)


def test_single_rank_is_identity():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.weak_scaling_value(1, 10, 1e-3, 1000.0) == pytest.approx(0.01)
