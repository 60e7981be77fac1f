"""Multi-GPU path on CPU: replicas over two gloo ranks.

bench.py --gpus N runs one independent simulation per rank (no collective
on the data path); the ranks meet in a barrier before the timed region and
take the maximum of their device times after it.  Here two processes on the
gloo backend run that logic with per-rank times standing in for device
times, and check the whole-job figure, the seeds of the replicas and the
rank -> GPU mapping.
"""
import os
import socket

import pytest
import torch.distributed as td
import torch.multiprocessing as mp

from rakali_b200 import replicas as rp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world,
                          timeout=datetime.timedelta(seconds=60))
    try:
        rp.barrier(td)
        ms = 10.0 + 3.0 * rank            # this rank's "device time"
        slowest = rp.max_over_ranks(ms, td, device="cpu")
        rp.barrier(td)
        cells, steps = 4096 * 4096, 500
        out[rank] = (slowest, rp.weak_value(world, cells, steps, slowest),
                     rp.replica_seed(7, rank))
    finally:
        td.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks_and_weak_value():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    slowest = 10.0 + 3.0 * (world - 1)
    for rank in range(world):
        assert res[rank][0] == slowest  # every rank reports the slowest rank's time
        assert res[rank][1] == pytest.approx(world * 4096 * 4096 * 500 / (slowest * 1e-3))
    assert {res[r][2] for r in range(world)} == {7, 8}  # independent replica workloads


def test_single_process_has_no_collective():
    assert rp.max_over_ranks(5.0, None) == 5.0
    rp.barrier(None)
    assert rp.weak_value(1, 100, 10, 1000.0) == 1000.0


def test_visible_gpu_index():
    assert rp.visible_gpu_index(1, {"CUDA_VISIBLE_DEVICES": "3,5"}) == 5
    assert rp.visible_gpu_index(0, {"CUDA_VISIBLE_DEVICES": "GPU-uuid"}) == 0
    assert rp.visible_gpu_index(2, {}) == 2
