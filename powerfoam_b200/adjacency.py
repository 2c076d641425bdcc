"""Neighbour structures consumed by the render kernels.

* ``power_adjacency_diff`` -- (E,4) float16 (c_j - c_i, pm_j - pm_i),
  benchmark.py:296-302, on the GPU.
* ``start_cell`` -- argmin_i |p_i - eye|^2 - r_i^2, benchmark.py:320-324, on
  the GPU.
* ``power_adjacency`` / ``PowerBuilder`` -- the weighted-Delaunay edges of
  build_power_adjacency (benchmark.py:25-83) on the GPU by clipping power
  cells (pf_power_adjacency).
"""

import torch

from . import _lib


def power_adjacency_diff(points, radii, adjacency, adjacency_offsets):
    points = points.float().contiguous()
    radii = radii.float().contiguous()
    adjacency = adjacency.to(torch.int32).contiguous()
    adjacency_offsets = adjacency_offsets.to(torch.int32).contiguous()
    out = torch.empty((adjacency.shape[0], 4), dtype=torch.float16, device=points.device)
    _lib.call("pf_adjacency_power_diff", _lib.ptr(points), _lib.ptr(radii), _lib.ptr(adjacency),
              _lib.ptr(adjacency_offsets), points.shape[0], _lib.ptr(out), _lib.stream_ptr())
    return out


def start_cell(points, radii, eye, as_tensor=False):
    points = points.float().contiguous()
    radii = radii.float().contiguous()
    ws = torch.empty(256, dtype=torch.uint8, device=points.device)
    out = torch.empty(1, dtype=torch.int32, device=points.device)
    e = (_lib.ctypes.c_float * 3)(*[float(v) for v in torch.as_tensor(eye).float().cpu().tolist()])
    _lib.call("pf_start_cell", _lib.ptr(points), _lib.ptr(radii), points.shape[0], e, _lib.ptr(ws), ws.numel(),
              _lib.ptr(out), _lib.stream_ptr())
    return out if as_tensor else int(out.item())


class CechBuilder:
    """GPU Čech adjacency (bvh.py:72-123 semantics) with a reusable workspace;
    lists ascending.  Like the reference's build_cech_complex (.item() at
    bvh.py:110), it reads the edge count once to size the output."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.ws = None
        self.capacity = 0

    def __call__(self, points, radii):
        points = points.float().contiguous()
        radii = radii.float().contiguous()
        n = points.shape[0]
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_cech_workspace_size", n, _lib.ctypes.byref(nbytes))
        if self.ws is None or self.ws.numel() < nbytes.value:
            self.ws = torch.empty(nbytes.value, dtype=torch.uint8, device=self.device)
        cap = max(self.capacity, 16 * n, 1 << 16)
        while True:
            adj = torch.empty(cap, dtype=torch.int32, device=self.device)
            off = torch.empty(n + 1, dtype=torch.int32, device=self.device)
            scalars = torch.zeros(2, dtype=torch.int64, device=self.device)
            status = scalars[1:].view(torch.int32)[:1]
            _lib.call("pf_cech_adjacency", _lib.ptr(points), _lib.ptr(radii), n, _lib.ptr(self.ws), self.ws.numel(),
                      cap, _lib.ptr(adj), _lib.ptr(off), _lib.ptr(scalars[:1]), _lib.ptr(status), _lib.stream_ptr())
            e = int(scalars[0].item())
            if e <= cap:
                break
            if e >= (1 << 31) - 1:
                raise _lib.PfError(_lib.PF_ERR_OVERFLOW, f"{e} adjacency entries exceed int32 offsets")
            cap = min(1 << (int(e * 1.25) - 1).bit_length(), (1 << 31) - 1)
        self.capacity = max(self.capacity, cap)
        return adj[:e], off


class PowerBuilder:
    """GPU power-diagram adjacency (pf_power_adjacency): the neighbour sets of
    build_power_adjacency (benchmark.py:25-83) without the host hull, lists
    ascending.  Like CechBuilder it reads the edge count once to size the
    output; a cell beyond the kernel's capacity raises PF_ERR_CELL."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.ws = None
        self.capacity = 0

    def __call__(self, points, radii, alpha_complex=False):
        points = points.float().contiguous()
        radii = radii.float().contiguous()
        n = points.shape[0]
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_power_workspace_size", n, _lib.ctypes.byref(nbytes))
        if self.ws is None or self.ws.numel() < nbytes.value:
            self.ws = torch.empty(nbytes.value, dtype=torch.uint8, device=self.device)
        cap = max(self.capacity, 20 * n, 1 << 16)
        while True:
            adj = torch.empty(cap, dtype=torch.int32, device=self.device)
            off = torch.empty(n + 1, dtype=torch.int32, device=self.device)
            scalars = torch.zeros(2, dtype=torch.int64, device=self.device)
            status = scalars[1:].view(torch.int32)[:1]
            _lib.call("pf_power_adjacency", _lib.ptr(points), _lib.ptr(radii), n, int(bool(alpha_complex)),
                      _lib.ptr(self.ws), self.ws.numel(), cap, _lib.ptr(adj), _lib.ptr(off), _lib.ptr(scalars[:1]),
                      _lib.ptr(status), _lib.stream_ptr())
            e, st = (int(v) for v in torch.stack([scalars[0], status[0].long()]).tolist())
            if st == _lib.PF_ERR_CELL:
                raise _lib.PfError(st, "a power cell exceeded the kernel's plane / neighbour capacity")
            if e <= cap:
                break
            if e >= (1 << 31) - 1:
                raise _lib.PfError(_lib.PF_ERR_OVERFLOW, f"{e} adjacency entries exceed int32 offsets")
            cap = min(1 << (int(e * 1.25) - 1).bit_length(), (1 << 31) - 1)
        self.capacity = max(self.capacity, cap)
        return adj[:e], off


def power_adjacency(points, radii, alpha_complex=False):
    """build_power_adjacency on the GPU (the same neighbour sets)."""
    return PowerBuilder(points.device)(points, radii, alpha_complex)


def cech_adjacency(points, radii):
    return CechBuilder(points.device)(points, radii)


def morton_sort(points):
    """Permutation (int32) ordering the points along the Morton curve
    (geometry.py:50-85)."""
    points = points.float().contiguous()
    n = points.shape[0]
    if n == 0:
        return torch.zeros(0, dtype=torch.int32, device=points.device)
    nbytes = _lib.ctypes.c_size_t(0)
    _lib.call("pf_morton_workspace_size", n, _lib.ctypes.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=points.device)
    perm = torch.empty(n, dtype=torch.int32, device=points.device)
    _lib.call("pf_morton_sort", _lib.ptr(points), n, _lib.ptr(ws), ws.numel(), _lib.ptr(perm), _lib.stream_ptr())
    return perm
