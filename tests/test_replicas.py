"""Replica timing over ranks (the multi-GPU host logic of bench.py) with the
gloo backend on CPU, two processes on 127.0.0.1."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, values, out):
    import torch.distributed as dist
    from aerof_dev_b200.replicas import aggregate_rate, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = max_over_ranks(values[rank], "cpu")
        out[rank] = (ms, aggregate_rate(1000.0, world, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    values = [3.5, 7.25]
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, values, out), nprocs=world, join=True)
    for r in range(world):
        ms, rate = out[r]
        assert ms == 7.25
        assert rate == pytest.approx(1000.0 * 2 / 7.25e-3)


def test_single_process_is_identity():
    from aerof_dev_b200.replicas import aggregate_rate, max_over_ranks
    assert max_over_ranks(1.5) == 1.5
    assert aggregate_rate(10.0, 1, 2.0) == pytest.approx(5000.0)
