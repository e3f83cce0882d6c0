"""bench.py's N > 1 path on CPU with two gloo ranks: every rank runs its own replica of the Gram step (no
data-path collective); the step time reported is the slowest rank's (one MAX all-reduce, taken by every rank
in the same order), and the reference arm runs on rank 0 only while the other ranks return at once."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import types

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = [bench.max_over_ranks(10.0 * (rank + 1) + k, world, "cpu") for k in range(3)]
        args = types.SimpleNamespace(steps=1, warmup=0)
        skipped = bench.run_reference(args, rank, world) is None if rank != 0 else True
        dist.barrier()
        out.put((rank, got, skipped))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_time_and_rank0_reference():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, got, skipped = out.get(timeout=120)
        res[r] = (got, skipped)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        got, skipped = res[r]
        assert got == [10.0 * world + k for k in range(3)]       # every rank sees the slowest rank's time
        assert skipped


def test_single_rank_time_is_its_own():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25
