"""The multi-rank bench path on the CPU (gloo, two ranks): every rank builds
the same seeded request batch (replicas), and the reported rate is all
ranks' solves over the slowest rank's time."""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench

        reqs = bench.make_requests(6, 0)
        names = [p.name for p in reqs]
        # rank r solved 10 + r requests in (1 + r) seconds
        rate, ms = bench.aggregate_rate(10 + rank, 1000.0 * (1 + rank), world, device="cpu")
        out[rank] = (names, rate, ms)
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_and_replicas():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    names0, rate0, ms0 = out[0]
    names1, rate1, ms1 = out[1]
    assert names0 == names1  # the same request batch on every rank
    assert ms0 == ms1 == 2000.0  # the slowest rank's time
    assert rate0 == rate1 == pytest.approx((10 + 11) / 2.0)


def test_single_rank_needs_no_group():
    import bench

    rate, ms = bench.aggregate_rate(30, 1500.0, 1)
    assert ms == 1500.0 and rate == pytest.approx(20.0)
