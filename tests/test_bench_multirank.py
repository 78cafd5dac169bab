"""The N > 1 path of bench.py on CPU: two gloo ranks each time their own
replica; the whole-job figures take the slowest rank's time and every
rank's work (bench.replica_result), the only collective of the benchmark."""
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


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms = [100.0, 140.0][rank]            # rank 1 is the slow one
    pairs = [1_000_000.0, 1_200_000.0][rank]
    r = bench.replica_result(ms, pairs, steps=10, world=world, device="cpu")
    out[rank] = (r["ms"], r["pairs"], r["value"], r["steps_per_s"])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ms, pairs, value, sps = res[rank]
        assert ms == 140.0
        assert pairs == 2_200_000.0
        assert value == pytest.approx(2_200_000.0 / 0.14)
        assert sps == pytest.approx(10 / 0.14)


def test_single_rank_is_identity():
    import bench
    r = bench.replica_result(50.0, 1000.0, steps=5, world=1, device="cpu")
    assert r["ms"] == 50.0 and r["value"] == pytest.approx(1000.0 / 0.05)
