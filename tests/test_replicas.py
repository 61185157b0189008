"""Multi-GPU runs of bench.py are independent replicas (no data-path
collective): the timed region ends with the maximum over ranks and the
reported value counts every rank's determinants over that time.  Checked
here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r pretends its timed region took 1 + r seconds and its e2e 5 - r
        got = bench.max_over_ranks(dist, [1.0 + rank, 5.0 - rank], "cpu")
        dist.barrier()
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    assert out[0] == out[1] == [2.0, 5.0]


def test_single_rank_and_rate():
    assert bench.max_over_ranks(None, [3.0, 4.0], "cpu") == [3.0, 4.0]
    # 2 replicas x 1e9 determinant-vectors in 2 s (slowest rank) = 1e9 per s
    assert bench.replica_rate(2, 1e9, 2.0) == pytest.approx(1e9)
