"""Geometry terms of the training loss, mirroring powerfoam/geometry.py.

* ``InterpenetrationFunction`` -- autograd function of the interpenetration
  penalty (geometry.py:88-189): per sphere, the sum over its adjacency list of
  (r_i + r_j - |c_i - c_j|)^2 for the overlapping entries.  Same arguments
  (points (N,3), radii (N), adjacency, adjacency_offsets) and the same
  returns as the reference: areas (N) forward; (grad_points, grad_radii,
  None, None) backward, the two gradients being views of one (N,4) array as
  there.  Runs pf_interpenetration / pf_interpenetration_backward.
* ``morton_sort`` -- geometry.py:50-85, see adjacency.py.
"""

import torch

from . import _lib
from .adjacency import morton_sort

__all__ = ["InterpenetrationFunction", "interpenetration", "morton_sort"]


def _index(t):
    return t.to(torch.int32).contiguous()


class InterpenetrationFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, radii, adjacency, adjacency_offsets):
        spheres = torch.cat([points, radii[:, None]], dim=-1).to(torch.float32).contiguous()
        adjacency = _index(adjacency)
        adjacency_offsets = _index(adjacency_offsets)
        n = spheres.shape[0]
        if adjacency_offsets.numel() != n + 1:
            raise ValueError("adjacency_offsets must hold N + 1 entries")
        areas = torch.empty(n, dtype=torch.float32, device=spheres.device)
        status = torch.zeros(1, dtype=torch.int32, device=spheres.device)
        _lib.call("pf_interpenetration", _lib.ptr(spheres), _lib.ptr(adjacency), _lib.ptr(adjacency_offsets), n,
                  adjacency.numel(), _lib.ptr(areas), _lib.ptr(status), _lib.stream_ptr())
        ctx.save_for_backward(spheres, adjacency, adjacency_offsets, status)
        return areas

    @staticmethod
    def backward(ctx, areas_grad_in):
        spheres, adjacency, adjacency_offsets, status = ctx.saved_tensors
        areas_grad_in = areas_grad_in.to(torch.float32).contiguous()
        n = spheres.shape[0]
        grad = torch.empty((n, 4), dtype=torch.float32, device=spheres.device)
        _lib.call("pf_interpenetration_backward", _lib.ptr(spheres), _lib.ptr(adjacency), _lib.ptr(adjacency_offsets),
                  n, adjacency.numel(), _lib.ptr(areas_grad_in), _lib.ptr(grad), _lib.ptr(status), _lib.stream_ptr())
        return grad[..., :3], grad[..., 3], None, None


def interpenetration(points, radii, adjacency, adjacency_offsets, validate=False):
    """areas (N) with autograd to points and radii (scene.py:476-482).  The
    kernels skip neighbour indices outside [0, N) (the reference reads out of
    bounds there); validate=True checks the structure on the host first."""
    if validate:
        check_adjacency(adjacency, adjacency_offsets, points.shape[0])
    return InterpenetrationFunction.apply(points, radii, adjacency, adjacency_offsets)


def check_adjacency(adjacency, adjacency_offsets, n):
    """Host-side validation of an adjacency structure (raises ValueError):
    N + 1 non-decreasing offsets from 0 to E, every index in [0, N)."""
    off = adjacency_offsets.to(torch.int64)
    if off.numel() != n + 1 or int(off[0]) != 0 or int(off[-1]) != adjacency.numel():
        raise ValueError("adjacency_offsets must run from 0 to len(adjacency) over N + 1 entries")
    if n > 0 and bool((off[1:] < off[:-1]).any()):
        raise ValueError("adjacency_offsets must be non-decreasing")
    if adjacency.numel() and (int(adjacency.min()) < 0 or int(adjacency.max()) >= n):
        raise ValueError("adjacency index out of range")
