"""View-parallel training across GPUs: one process per GPU, the scene
replicated, the views split round-robin over the ranks, the per-primitive
gradients summed across ranks.

No counterpart in the reference (it renders one view per call on one GPU).
The exchange is the only collective on the path: rendering a view needs no
data from other ranks, and the gradient of a sum of per-view losses is the sum
of the per-rank gradients.  With NCCL the sum runs over NVLink; the CPU tests
run the same code with gloo.

The gradients live in one persistent flat buffer (``GradBuffer``): the
adjoint kernels write straight into its views, and the collectives run on
slices of it, so nothing is packed or unpacked around the exchange.  Two
exchanges:

* ``allreduce()`` -- every rank ends with the full sum (data-parallel
  optimiser step on every rank).  A ring all-reduce moves 2 (W-1)/W of the
  buffer in and out of each rank: 2 (W-1)/W x 256 B per primitive for the
  rasterizer's 64 gradient floats.
* ``reduce_scatter()`` -- each rank ends with the sum over its own primitive
  range only (the owner steps its shard of the parameters, then an
  all-gather of the updated parameters replaces the all-reduce's second
  half): (W-1)/W x 256 B per primitive.

Every field's first dimension is the primitive index; fields are stored
one after another, each padded to a multiple of the world size in that
dimension so that every rank's range is a contiguous slice of every field.
"""

import math

import torch
import torch.distributed as dist

BUCKET_BYTES = 256 << 20


def shard_views(n_views, rank, world):
    """Indices of the views rank `rank` renders (round-robin, so uneven view
    sizes spread over the ranks)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return list(range(rank, n_views, world))


class GradBuffer:
    """Per-primitive gradient fields in one flat buffer.

    ``fields``: {name: shape} with a common first dimension N (the primitive
    count); ``view(name)`` is the (N, ...) view that kernels and autograd
    write; every rank must build the buffer with the same fields in the same
    order."""

    def __init__(self, fields, device, dtype=torch.float32, world=1, bucket_bytes=BUCKET_BYTES):
        fields = dict(fields)
        if not fields:
            raise ValueError("no gradient fields")
        ns = {shape[0] for shape in fields.values()}
        if len(ns) != 1:
            raise ValueError("every field's first dimension must be the primitive count")
        self.n = ns.pop()
        self.world = int(world)
        self.n_pad = math.ceil(self.n / self.world) * self.world
        self.bucket = max(1, bucket_bytes // torch.empty((), dtype=dtype).element_size())
        self.layout = {}  # name -> (offset, row elements, shape)
        off = 0
        for name, shape in fields.items():
            row = int(math.prod(shape[1:]))
            self.layout[name] = (off, row, tuple(shape))
            off += self.n_pad * row
        self.flat = torch.zeros(off, device=device, dtype=dtype)

    def view(self, name):
        """A fresh (N, ...) view of field `name`.  Fresh views matter for
        autograd: a gradient tensor that nothing else references becomes the
        parameter's .grad as it is (a referenced one would be copied), so
        .grad then aliases the buffer -- set .grad to None between steps (the
        optimisers' default zero_grad) so no step adds into it."""
        o, row, shape = self.layout[name]
        return self.flat[o:o + self.n * row].view(shape)

    def views(self):
        return {name: self.view(name) for name in self.layout}

    def zero_(self):
        self.flat.zero_()

    def _chunks(self):
        for o in range(0, self.flat.numel(), self.bucket):
            yield self.flat[o:o + self.bucket]

    def allreduce(self, group=None):
        """Sum the buffer across ranks in place, one all-reduce per bucket
        (contiguous slices of the buffer: no copies)."""
        for c in self._chunks():
            dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)

    def owned_range(self, rank):
        """Primitive rows [lo, hi) rank `rank` owns after reduce_scatter."""
        per = self.n_pad // self.world
        return rank * per, min((rank + 1) * per, self.n)

    def reduce_scatter(self, rank, group=None):
        """Sum every field across ranks, each rank receiving only its own
        primitive range; returns {name: (rows, ...) view} of this rank's
        summed rows, which overwrite the start of its own range in place."""
        per = self.n_pad // self.world
        out = {}
        for name, (o, row, shape) in self.layout.items():
            full = self.flat[o:o + self.n_pad * row]
            mine = self.flat[o + rank * per * row:o + (rank + 1) * per * row]
            if dist.get_backend(group) == dist.Backend.NCCL:
                # in place: NCCL reduce-scatters into recvbuff == sendbuff + rank * recvcount
                dist.reduce_scatter_tensor(mine, full, op=dist.ReduceOp.SUM, group=group)
            else:  # other backends get a separate output slice
                res = torch.empty_like(mine)
                dist.reduce_scatter_tensor(res, full, op=dist.ReduceOp.SUM, group=group)
                mine.copy_(res)
            lo, hi = self.owned_range(rank)
            out[name] = mine[:(hi - lo) * row].view((hi - lo,) + shape[1:])
        return out

    def bytes_per_rank(self, kind):
        """Bytes each rank sends (and receives) in one exchange with ring
        algorithms: all-reduce 2 (W-1)/W of the buffer, reduce-scatter
        (W-1)/W of it."""
        b = self.flat.numel() * self.flat.element_size()
        f = (self.world - 1) / self.world
        return int((2 * f if kind == "allreduce" else f) * b)


def raster_fields(n_prims, n_sites=8):
    """The rasterizer's (and tracer's) gradient fields, in the order of
    Rasterizer.forward's arguments."""
    n, S = int(n_prims), int(n_sites)
    return {"points": (n, 3), "radii": (n,), "density": (n,), "normals": (n, 3), "texel_sites": (n, S, 3),
            "texel_rgb": (n, S, 3), "texel_height": (n, S)}


def max_over_ranks(value, device, group=None):
    """The largest of every rank's `value` (a float): step times are reported
    as the slowest rank's."""
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
