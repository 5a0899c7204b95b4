"""Multi-GPU plan is replicas only: bench.py --gpus N runs one process per
GPU, each solving its own replica, timed per rank and reduced with a
max-over-ranks.  The host side of that path runs here as world_size-2 gloo
ranks on the CPU (no GPU)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms_local = 100.0 + 37.5 * rank          # each rank's own device time
        ms = bench.max_over_ranks(ms_local, dist, device="cpu")
        value = bench.replica_throughput(1_000_000, world, 5, ms)
        dist.barrier()
        out.put((rank, ms, value, bench.replica_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = 100.0 + 37.5 * (world - 1)
    for rank, ms, value, seed in res:
        assert ms == slowest                                   # every rank sees the slowest time
        assert value == pytest.approx(world * 1_000_000 * 5 / (slowest / 1e3) / 1e6)
    assert len({seed for *_, seed in res}) == world            # distinct replicas


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.replica_throughput(150_000_000, 1, 5, 750.0) == pytest.approx(1000.0)
