"""CPU, world_size 2 over gloo: the replica bookkeeping of bench.py --gpus N.

The path does not shard (one independent replica per GPU, no collective in
the step); the only cross-rank step is the timing: the job time is the
slowest rank's, and the rate counts every rank's atoms."""
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


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms_local = 10.0 * (rank + 1)  # rank 1 is the slow one
    ms_max, value = bench.whole_job_rate(ms_local, 1000, 50, dist, torch, device="cpu")
    q.put((rank, ms_max, value))
    dist.barrier()
    dist.destroy_process_group()


def test_whole_job_rate_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms_max, value in out:
        assert ms_max == pytest.approx(20.0)
        assert value == pytest.approx(2 * 1000 * 50 / 0.020)


def test_single_rank_rate():
    import bench
    ms, v = bench.whole_job_rate(4.0, 100, 10, None, torch)
    assert ms == 4.0 and v == pytest.approx(100 * 10 / 0.004)
