"""The multi-GPU bench path is independent replicas (one image per rank) timed as the max over
ranks; the reference arm runs on rank 0 only.  Exercised here with two gloo ranks on CPU."""

from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(1.5 + rank, world)
        # the reference arm: rank != 0 returns before any work or output
        printed = []

        class Args:
            size, prims, ref_step_s, steps, warmup, gpus = 64, 4, 0.05, 1, 0, world

        if rank != 0:
            bench.reference_arm(Args, world, rank, executor=None)
            printed.append("nothing")
        q.put((rank, slowest, printed))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_only_rank0_reports():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]
    assert out[1][2] == ["nothing"]
