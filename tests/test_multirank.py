"""Host logic of bench.py under torchrun, on CPU with the gloo backend and
two ranks (the same calls the NCCL run makes): the reported time is the
maximum over ranks, every rank has its own history seeds, and the reference
arm runs on rank 0 only (the other ranks exit 0 without work or output)."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from tests.conftest import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(REPO))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.reduce_max([1.0 + rank, 10.0 - rank, 0.5 * rank], dist, "cpu")
        seeds = [None] * world
        dist.all_gather_object(seeds, bench.rank_seed(rank))
        out = io.StringIO()
        if rank != 0:
            with redirect_stdout(out):
                rc = bench.run_reference_arm(type("A", (), {"gpus": world, "steps": 1, "warmup": 0,
                                                            "ref_sample": 1000})())
        else:
            rc = 0
        q.put((rank, got, seeds, rc, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, seeds, rc, out in res:
        assert got == [2.0, 10.0, 0.5]
        assert len(set(seeds)) == world
        assert rc == 0
        if rank != 0:
            assert out == ""


def test_reduce_max_without_process_group():
    sys.path.insert(0, str(REPO))
    import bench
    assert bench.reduce_max([3, 1.5], None, "cpu") == [3.0, 1.5]
