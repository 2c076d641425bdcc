"""View-parallel training across GPUs: one process per GPU, the scene
replicated, the views split round-robin over the ranks, the per-primitive
gradients summed with one collective per bucket.

No counterpart in the reference (it renders one view per call on one GPU).
The exchange is the only collective on the path: rendering a view needs no
data from other ranks, and the gradient of a sum of per-view losses is the sum
of the per-rank gradients.  With NCCL the sum runs over NVLink; the CPU tests
run the same code with gloo.
"""

import torch
import torch.distributed as dist

BUCKET_BYTES = 256 << 20


def shard_views(n_views, rank, world):
    """Indices of the views rank `rank` renders (round-robin, so uneven view
    sizes spread over the ranks)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return list(range(rank, n_views, world))


class GradReducer:
    """Sums a fixed set of gradient tensors across ranks in place.  The
    tensors are copied into flat buckets of at most BUCKET_BYTES (allocated
    once), all-reduced, and copied back; every rank must pass tensors of the
    same shapes in the same order."""

    def __init__(self, tensors, group=None, bucket_bytes=BUCKET_BYTES):
        self.tensors = list(tensors)
        self.group = group
        if not self.tensors:
            raise ValueError("nothing to reduce")
        dev, dt = self.tensors[0].device, self.tensors[0].dtype
        if any(t.device != dev or t.dtype != dt or not t.is_contiguous() for t in self.tensors):
            raise ValueError("gradients must be contiguous and share one device and dtype")
        per = max(1, bucket_bytes // self.tensors[0].element_size())
        self.buckets = []  # (flat buffer, [(tensor, offset, numel) ...])
        cur, used = [], 0
        for t in self.tensors:
            if cur and used + t.numel() > per:
                self.buckets.append(self._make(cur, used, dev, dt))
                cur, used = [], 0
            cur.append((t, used, t.numel()))
            used += t.numel()
        self.buckets.append(self._make(cur, used, dev, dt))

    @staticmethod
    def _make(items, n, dev, dt):
        return torch.empty(n, device=dev, dtype=dt), items

    def __call__(self):
        for flat, items in self.buckets:
            for t, o, n in items:
                flat[o:o + n].copy_(t.reshape(-1))
            dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=self.group)
            for t, o, n in items:
                t.reshape(-1).copy_(flat[o:o + n])


def allreduce_(tensors, group=None):
    """Sum tensors that change from step to step (autograd's fresh .grad
    tensors) across ranks in place: one flat buffer, one all-reduce."""
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    o = 0
    for t in tensors:
        t.reshape(-1).copy_(flat[o:o + t.numel()])
        o += t.numel()


def max_over_ranks(value, device, group=None):
    """The largest of every rank's `value` (a float): step times are reported
    as the slowest rank's."""
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
