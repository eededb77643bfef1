"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1.

On N GPUs every rank steps its own replica (the path shards horizontally
with no exchange in this build), times its region with CUDA events, and
rank 0 reports the whole-job rate from the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms, rates = bench.job_rates([10.0 + rank, 20.0 - rank], 1000, 5, dist, device="cpu")
    out.put((rank, ms, rates))
    dist.barrier()
    dist.destroy_process_group()


def test_job_rates_take_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rates in res:
        assert ms == [11.0, 20.0]  # max over ranks of each region
        assert rates[0] == pytest.approx(world * 1000 * 5 / 11e-3)
        assert rates[1] == pytest.approx(world * 1000 * 5 / 20e-3)


def test_single_rank_without_process_group():
    import bench
    ms, rates = bench.job_rates([4.0], 10, 2, None, device="cpu")
    assert ms == [4.0] and rates == [pytest.approx(10 * 2 / 4e-3)]
