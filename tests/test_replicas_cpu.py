"""Multi-GPU use is independent replicas (one job per GPU, no data
exchange); the ranks share only timings.  Two gloo ranks on the CPU check
the max-over-ranks reduction and the whole-job rate that bench.py reports."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from mbirtorch_b200.replicas import max_over_ranks, replica_rate


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=__import__('datetime').timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank          # each replica's own step time
        slowest = max_over_ranks(ms)
        out[rank] = (slowest, replica_rate(4, slowest / 1e3, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time_and_rate():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True,
                           start_method='spawn')
        res = dict(out)
    assert res[0] == res[1]
    slowest, rate = res[0]
    assert slowest == 150.0
    assert rate == pytest.approx(2 * 4 / 0.150)


def test_single_process_is_its_own_maximum():
    assert max_over_ranks(12.5) == 12.5
    assert replica_rate(3, 1.5, 1) == pytest.approx(2.0)
    with pytest.raises(ValueError):
        replica_rate(3, 0.0, 2)
