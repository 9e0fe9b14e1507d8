"""Multi-process plumbing on CPU (gloo, world size 2): the partition of a
batch's instances over ranks is a disjoint cover, and the max / sum
reductions the benchmark uses agree on every rank."""
import os
import socket

import pytest

from hmat_lib_b200 import multi


def test_partition_is_a_disjoint_cover():
    for world in (1, 2, 3, 8):
        parts = [multi.partition(512, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(512))
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        multi.partition(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = multi.partition(512, rank, world)
        count = multi.sum_over_ranks(len(mine), dist)
        slowest = multi.max_over_ranks(1.5 + rank, dist)
        out.put((rank, count, slowest, mine[:3]))
    finally:
        dist.destroy_process_group()


def test_reductions_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [512.0, 512.0]
    assert [r[2] for r in res] == [2.5, 2.5]
    assert res[0][3] == [0, 2, 4] and res[1][3] == [1, 3, 5]
