"""View-parallel host logic on two CPU ranks (gloo): round-robin sharding
covers every view once, the gradient exchange on the flat GradBuffer
(all-reduce, and reduce-scatter to primitive-range owners) equals the
single-process sum over all views, and step times reduce to the slowest
rank.  The per-view "gradients" are seeded stand-ins for renders with the
shapes of BatchStep's gradient buffer (this suite has no GPU); the path under
test is the sharding and the exchange."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from powerfoam_b200.multiview import GradBuffer, max_over_ranks, raster_fields, shard_views

N_PRIMS = 1001  # not a multiple of the world size: the owners' ranges are padded
FIELDS = {"points": (N_PRIMS, 3), "radii": (N_PRIMS,), "normals": (N_PRIMS, 3), "density": (N_PRIMS,),
          "texel_sites": (N_PRIMS, 8, 3), "texel_height": (N_PRIMS, 8), "sh": (N_PRIMS, 16, 3)}
N_VIEWS = 7


def view_grads(v):
    g = torch.Generator().manual_seed(1000 + v)
    return {k: torch.randn(s, generator=g, dtype=torch.float64) for k, s in FIELDS.items()}


def reference_sum():
    total = {k: torch.zeros(s, dtype=torch.float64) for k, s in FIELDS.items()}
    for v in range(N_VIEWS):
        for k, g in view_grads(v).items():
            total[k] += g
    return total


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, bucket_bytes, mode, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        gb = GradBuffer(FIELDS, torch.device("cpu"), dtype=torch.float64, world=world, bucket_bytes=bucket_bytes)
        views = gb.views()  # the kernels' outputs write these in place
        mine = shard_views(N_VIEWS, rank, world)
        for v in mine:
            for k, g in view_grads(v).items():
                views[k] += g
        flat_ptr = gb.flat.data_ptr()
        if mode == "allreduce":
            gb.allreduce()
            res = {k: gb.view(k).clone() for k in FIELDS}
        else:
            res = {k: t.clone() for k, t in gb.reduce_scatter(rank).items()}
        assert gb.flat.data_ptr() == flat_ptr  # summed in place
        slow = max_over_ranks(10.0 + rank, torch.device("cpu"))
        torch.save(dict(grads=res, views=mine, slow=slow, owned=gb.owned_range(rank),
                        bytes=(gb.bytes_per_rank("allreduce"), gb.bytes_per_rank("reduce_scatter"))),
                   os.path.join(out_dir, f"rank{rank}.pt"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode,bucket_bytes", [("allreduce", 1 << 30), ("allreduce", 20000),
                                               ("reduce_scatter", 1 << 30)])
def test_view_parallel_gradient_exchange_two_ranks(tmp_path, mode, bucket_bytes):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), bucket_bytes, mode, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    ref = reference_sum()
    seen, covered = [], []
    for r in range(world):
        res = torch.load(tmp_path / f"rank{r}.pt")
        seen += res["views"]
        assert res["slow"] == 10.0 + world - 1
        lo, hi = res["owned"]
        covered += list(range(lo, hi))
        ar, rs = res["bytes"]
        assert ar == 2 * rs  # a ring all-reduce moves twice what a reduce-scatter does
        for k in FIELDS:
            want = ref[k] if mode == "allreduce" else ref[k][lo:hi]
            torch.testing.assert_close(res["grads"][k], want, rtol=1e-12, atol=1e-12)
    assert sorted(seen) == list(range(N_VIEWS))
    if mode == "reduce_scatter":
        assert covered == list(range(N_PRIMS))  # the owners' ranges partition the primitives


def test_shard_views_and_buffer_arguments():
    assert shard_views(5, 1, 2) == [1, 3]
    assert shard_views(1, 1, 2) == []
    with pytest.raises(ValueError):
        shard_views(4, 2, 2)
    with pytest.raises(ValueError):
        GradBuffer({}, torch.device("cpu"))
    with pytest.raises(ValueError):
        GradBuffer({"a": (3,), "b": (4, 2)}, torch.device("cpu"))
    gb = GradBuffer(raster_fields(10, 8), torch.device("cpu"), world=4)
    assert gb.n == 10 and gb.n_pad == 12
    assert gb.flat.numel() == 12 * 64  # 64 gradient floats per (padded) primitive
    v = gb.view("texel_rgb")
    assert v.shape == (10, 8, 3) and v.data_ptr() != gb.view("texel_sites").data_ptr()
    assert [gb.owned_range(r) for r in range(4)] == [(0, 3), (3, 6), (6, 9), (9, 10)]
