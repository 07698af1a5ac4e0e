"""The multi-rank path of the benchmark on CPU: two `gloo` ranks.

The reconstruction does not shard, so N GPUs run N independent replicas.
The only exchange is the timing: each rank's device time is reduced to the
maximum over ranks, and the whole-job throughput is N x pixels / that time.
These tests run that reduction over a real process group of two ranks."""

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, times: list, out) -> None:
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    ws, r, local = bench.dist_env()
    assert (ws, r, local) == (world, rank, rank)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(times[rank], "cpu")
        # A second reduction at the same point on every rank (the e2e leg).
        t2 = bench.max_over_ranks(10.0 * times[rank], "cpu")
        out.put((rank, t, t2))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_max_over_two_gloo_ranks():
    times = [2.5, 4.0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.spawn(_rank, args=(2, _free_port(), times, q), nprocs=2, join=True)
    got = sorted(q.get(timeout=30) for _ in range(2))
    for rank, t, t2 in got:
        assert t == max(times) and t2 == 10.0 * max(times)
    # Whole-job throughput of the replicas: every rank reconstructs one
    # frame per step, and the job takes as long as its slowest rank.
    px = 3840 * 2160
    value = 2 * px / (max(times) * 1e-3) / 1e6
    assert abs(value - 2 * px / 4e-3 / 1e6) < 1e-9


def test_single_process_is_identity():
    assert bench.max_over_ranks(3.25, "cpu") == 3.25
