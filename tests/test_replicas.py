"""Replica path of multi-GPU runs, exercised with two gloo ranks on the CPU: instance
sharding covers every instance exactly once, the job time is the max over ranks and the
whole-job rate counts every rank's work."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from laqphysics_b200.replicas import gather_to_root, max_over_ranks, shard, whole_job_rate


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = shard(list(range(13)), rank, world)
        slowest = max_over_ranks(10.0 + rank * 5.0, dist)
        gathered = gather_to_root(np.array(mine), dist)
        results[rank] = (mine, slowest, [list(g) for g in gathered])
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_with_gloo():
    world = 2
    manager = mp.get_context('spawn').Manager()
    results = manager.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world, start_method='spawn', join=True)
    mine0, slow0, gathered0 = results[0]
    mine1, slow1, _ = results[1]
    assert sorted(mine0 + mine1) == list(range(13)) and not set(mine0) & set(mine1)
    assert slow0 == slow1 == 15.0
    assert gathered0 == [mine0, mine1]


def test_single_process_fallbacks_and_rate():
    assert shard([1, 2, 3], 0, 1) == [1, 2, 3]
    assert max_over_ranks(3.5) == 3.5
    assert whole_job_rate(100., 2., 4) == 200.
    with pytest.raises(ValueError):
        shard([1], 2, 2)
