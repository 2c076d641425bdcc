"""Steiner points for reference-faithful tracing, mirroring benchmark.py:
``inverse_softplus`` (:86-91), ``get_steiner_points`` (:137-180) with the
nearest-neighbour query (scipy's cKDTree there) and the greedy
minimum-overlap selection (``_greedy_min_overlap_fps``, :93-134) on the GPU
(pf_steiner_knn, pf_steiner_select).  Random sampling, masks and
concatenation stay in torch, as in the reference; ``sampler`` and
``seed_index`` let a caller supply the random draws.
"""

import torch

from . import _lib


def inverse_softplus(x, beta=100, threshold=20):
    """benchmark.py:86-91."""
    mask = x * beta > threshold
    y = torch.empty_like(x)
    y[mask] = x[mask]
    y[~mask] = torch.log(torch.exp(beta * x[~mask]) - 1) / beta
    return y


def knn_min_radius(points, radii, samples, k=32, workspace=None):
    """For each sample, min over its k nearest centres of (dist - r) and the
    primitive attaining it (benchmark.py:157-160)."""
    points = points.float().contiguous()
    radii = radii.float().contiguous()
    samples = samples.float().contiguous()
    n = points.shape[0]
    if workspace is None:
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_locator_workspace_size", n, _lib.ctypes.byref(nbytes))
        workspace = torch.empty(nbytes.value, dtype=torch.uint8, device=points.device)
    _lib.call("pf_locator_build", _lib.ptr(points), _lib.ptr(radii), n, _lib.ptr(workspace), workspace.numel(),
              _lib.stream_ptr())
    m = samples.shape[0]
    rad = torch.empty(m, dtype=torch.float32, device=points.device)
    idx = torch.empty(m, dtype=torch.int32, device=points.device)
    status = torch.zeros(1, dtype=torch.int32, device=points.device)
    _lib.call("pf_steiner_knn", _lib.ptr(points), _lib.ptr(radii), n, _lib.ptr(workspace), _lib.ptr(samples), m, k,
              _lib.ptr(rad), _lib.ptr(idx), _lib.ptr(status), _lib.stream_ptr())
    if m and int(status.item()) != 0:
        raise _lib.PfError(int(status.item()), f"fewer than {k} primitives for the nearest-neighbour query")
    return rad, idx.long()


def greedy_min_overlap(sample_points, sample_radii, seed_index=None, threshold=0.1):
    """_greedy_min_overlap_fps (benchmark.py:93-134): bool mask of the
    selected samples; the first pick is `seed_index` (else drawn with
    torch.randint as the reference does)."""
    n = sample_points.shape[0]
    dev = sample_points.device
    selected = torch.zeros(n, dtype=torch.uint8, device=dev)
    if n == 0:
        return selected.bool()
    if seed_index is None:
        seed_index = int(torch.randint(0, n, (1,), device=dev).item())
    scratch = torch.empty(n, dtype=torch.float32, device=dev)
    _lib.call("pf_steiner_select", _lib.ptr(sample_points.float().contiguous()),
              _lib.ptr(sample_radii.float().contiguous()), n, int(seed_index), float(threshold), _lib.ptr(scratch),
              _lib.ptr(selected), None, _lib.stream_ptr())
    return selected.bool()


def get_steiner_points(points, radii, cameras=None, rounds=10, sampler=None, seed_index=None):
    """benchmark.py:137-180.  sampler(round, n) -> (n, 3) samples (default:
    mean + 0.5 std * randn, the reference's draw); seed_index(round, n) ->
    first selected sample (default: torch.randint).  Returns the Steiner
    centres and their radii in inverse-softplus form."""
    del cameras  # unused, as in the reference
    points_mean = points.mean(dim=0, keepdim=True)
    points_std = points.std(dim=0, keepdim=True)
    steiner_points = torch.empty(0, 3, device=points.device)
    steiner_radii = torch.empty(0, device=points.device)
    ws = None
    for r in range(rounds):
        all_points = torch.cat([points, steiner_points], dim=0).float().contiguous()
        all_radii = torch.cat([radii, steiner_radii], dim=0).float().contiguous()
        num = int(0.25 * points.shape[0])
        if sampler is None:
            sample_points = points_mean + 0.5 * points_std * torch.randn(num, 3, device=points.device)
        else:
            sample_points = sampler(r, num).to(points.device)
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_locator_workspace_size", all_points.shape[0], _lib.ctypes.byref(nbytes))
        if ws is None or ws.numel() < nbytes.value:
            ws = torch.empty(nbytes.value, dtype=torch.uint8, device=points.device)
        sample_radii, closest = knn_min_radius(all_points, all_radii, sample_points, 32, ws)
        ratio = sample_radii / all_radii[closest]
        mask = (ratio > 2.0) & (ratio < 6.0)
        sample_points = sample_points[mask]
        sample_radii = sample_radii[mask]
        seed = None if seed_index is None else seed_index(r, sample_points.shape[0])
        is_candidate = greedy_min_overlap(sample_points, sample_radii, seed, threshold=0.1)
        steiner_points = torch.cat([steiner_points, sample_points[is_candidate]], dim=0)
        steiner_radii = torch.cat([steiner_radii, 0.8 * sample_radii[is_candidate]], dim=0)
    steiner_points = steiner_points.to(points.dtype)
    steiner_radii = inverse_softplus(steiner_radii, beta=100).to(radii.dtype)
    return steiner_points, steiner_radii
