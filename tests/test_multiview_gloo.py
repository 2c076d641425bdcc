"""View-parallel host logic on two CPU ranks (gloo): round-robin sharding
covers every view once, the bucketed gradient reduction equals the
single-process sum over all views, and step times reduce to the slowest
rank.  The per-view "gradient" is a seeded stand-in for a render (this
suite has no GPU); the path under test is the sharding and the exchange."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from powerfoam_b200.multiview import GradReducer, max_over_ranks, shard_views

SHAPES = [(1000, 3), (1000,), (1000, 3), (1000,), (1000, 8, 3), (1000, 8)]
N_VIEWS = 7


def view_grads(v):
    g = torch.Generator().manual_seed(1000 + v)
    return [torch.randn(s, generator=g, dtype=torch.float64) for s in SHAPES]


def reference_sum():
    total = [torch.zeros(s, dtype=torch.float64) for s in SHAPES]
    for v in range(N_VIEWS):
        for t, g in zip(total, view_grads(v)):
            t += g
    return total


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, bucket_bytes, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        grads = [torch.zeros(s, dtype=torch.float64) for s in SHAPES]
        mine = shard_views(N_VIEWS, rank, world)
        for v in mine:
            for t, g in zip(grads, view_grads(v)):
                t += g
        GradReducer(grads, bucket_bytes=bucket_bytes)()
        slow = max_over_ranks(10.0 + rank, torch.device("cpu"))
        torch.save(dict(grads=grads, views=mine, slow=slow), os.path.join(out_dir, f"rank{rank}.pt"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bucket_bytes", [1 << 30, 20000])
def test_view_parallel_gradient_sum_two_ranks(tmp_path, bucket_bytes):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), bucket_bytes, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    ref = reference_sum()
    seen = []
    for r in range(world):
        res = torch.load(tmp_path / f"rank{r}.pt")
        seen += res["views"]
        assert res["slow"] == 10.0 + world - 1
        for a, b in zip(res["grads"], ref):
            torch.testing.assert_close(a, b, rtol=1e-12, atol=1e-12)
    assert sorted(seen) == list(range(N_VIEWS))


def test_shard_views_and_reducer_arguments():
    assert shard_views(5, 1, 2) == [1, 3]
    assert shard_views(1, 1, 2) == []
    with pytest.raises(ValueError):
        shard_views(4, 2, 2)
    with pytest.raises(ValueError):
        GradReducer([])
    with pytest.raises(ValueError):
        GradReducer([torch.zeros(3), torch.zeros(3, dtype=torch.float64)])
