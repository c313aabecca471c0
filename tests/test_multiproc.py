"""Multi-process path of bench.py on CPU (gloo, world size 2): replicas only,
the slowest rank's time decides the whole-job rate."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["RANK"] = str(rank)
    os.environ["WORLD_SIZE"] = str(world)
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env()[:2] == (rank, world)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        slowest = bench.max_over_ranks(ms, world, "cpu")
        out[rank] = (slowest, bench.whole_job_rate(1e9, slowest, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        slowest, rate = out[r]
        assert slowest == pytest.approx(15.0)
        assert rate == pytest.approx(2 * 1e9 / 0.015 / 1e9)



def test_single_process_needs_no_collective():
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.whole_job_rate(2e9, 1000.0, 1) == pytest.approx(2.0)
