"""The N>1 replica path on CPU: two gloo ranks combine their timings as the benchmark does."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from amrclaw_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = replicas.assign(7, rank, world)
        ms, cells = replicas.combine(10.0 + 5.0 * rank, 1000.0 * (rank + 1), dist)
        out[rank] = (mine, ms, cells)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_max_time_and_sum_cells():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][0] == [0, 2, 4, 6] and res[1][0] == [1, 3, 5]
    for r in (0, 1):
        assert res[r][1] == 15.0
        assert res[r][2] == 3000.0


def test_single_process_is_identity_and_percentiles():
    assert replicas.combine(3.0, 5.0) == (3.0, 5.0)
    assert replicas.assign(3, 0, 1) == [0, 1, 2]
    with pytest.raises(ValueError):
        replicas.assign(3, 2, 2)
    p50, p99 = replicas.percentiles(list(range(1, 101)))
    assert (p50, p99) == (50, 99)
