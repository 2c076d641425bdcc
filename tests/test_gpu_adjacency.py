"""GPU Čech adjacency, Morton order and power-diagram adjacency against host
restatements and the reference's own hull construction."""

import numpy as np
import pytest
import torch

from powerfoam_b200.adjacency import CechBuilder, morton_sort
from powerfoam_b200.synthetic import morton_order_cpu
from tests.helpers import cech_np, np_scene, to_t

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,n,rmax", [(0, 500, 0.15), (1, 3000, 0.06), (2, 4000, 0.02)])
def test_cech_matches_bruteforce(seed, n, rmax):
    sc = np_scene(seed, n, -1.0, 1.0, rmax / 10, rmax)
    adj, off = cech_np(sc["points"], sc["radii"])
    a, o = CechBuilder("cuda")(to_t(sc["points"]), to_t(sc["radii"]))
    assert np.array_equal(o.cpu().numpy(), off)
    assert np.array_equal(a.cpu().numpy(), adj)


def test_cech_capacity_growth():
    sc = np_scene(3, 2000, -0.5, 0.5, 0.05, 0.2)
    adj, off = cech_np(sc["points"], sc["radii"])
    b = CechBuilder("cuda")
    b.capacity = 8
    a, o = b(to_t(sc["points"]), to_t(sc["radii"]))
    assert np.array_equal(a.cpu().numpy(), adj)


@pytest.mark.parametrize("n", [1, 1000, 100000])
def test_morton_matches_host(n):
    pts = torch.rand(n, 3, generator=torch.Generator().manual_seed(n)) * 4 - 2
    pts[: n // 10] = pts[0]  # ties keep index order
    p = morton_sort(pts.cuda()).cpu().long()
    assert torch.equal(p, morton_order_cpu(pts))


# ---------------------------------------------------------------------------
# power-diagram adjacency: the GPU cell clipping against the reference's
# algorithm (lifted hull by Qhull, benchmark.py:25-83) run on the host


def _power_case(seed, n, mode):
    rng = np.random.default_rng(seed)
    if mode == "mix":
        means = rng.uniform(-1, 1, (8, 3))
        pts = (means[rng.integers(0, 8, n)] + 0.15 * rng.standard_normal((n, 3))).astype(np.float32)
        pts[: n // 10] = rng.uniform(-1, 1, (n // 10, 3))
        radii = np.exp(rng.uniform(np.log(0.002), np.log(0.02), n)).astype(np.float32)
    elif mode == "hidden":  # large radius spread: many empty power cells
        pts = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
        radii = np.exp(rng.uniform(np.log(0.01), np.log(0.3), n)).astype(np.float32)
    else:
        pts = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
        radii = np.exp(rng.uniform(np.log(0.01), np.log(0.05), n)).astype(np.float32)
    return pts, radii


@pytest.mark.parametrize("seed,n,mode,alpha", [(0, 300, "uniform", False), (1, 2000, "uniform", True),
                                               (2, 5000, "mix", False), (3, 20000, "mix", True),
                                               (4, 3000, "hidden", False), (5, 6, "uniform", False)])
def test_power_adjacency_matches_hull(seed, n, mode, alpha):
    from oracle.power_hull import build_power_adjacency
    from powerfoam_b200.adjacency import PowerBuilder

    pts, radii = _power_case(seed, n, mode)
    a_ref, o_ref = build_power_adjacency(torch.from_numpy(pts), torch.from_numpy(radii), alpha_complex=alpha)
    a, o = PowerBuilder("cuda")(to_t(pts), to_t(radii), alpha_complex=alpha)
    assert torch.equal(o.cpu(), o_ref.cpu().to(torch.int32))
    assert torch.equal(a.cpu(), a_ref.cpu().to(torch.int32))
    if mode == "hidden":
        assert int(((o[1:] - o[:-1]) == 0).sum()) > n // 4  # hidden sites have no edges


def test_power_adjacency_synthetic_scene_matches_hull():
    """A 200,000-primitive mixture scene of the benchmark recipe (clusters,
    uniform background, radii spread tenfold)."""
    from powerfoam_b200 import synthetic
    from oracle.power_hull import build_power_adjacency
    from powerfoam_b200.adjacency import power_adjacency

    n = 200000
    s = (1048576 / n) ** (1 / 3)
    sc = synthetic.make_scene(n, seed=1, mixture=32, sigma=0.15, r_range=(0.002 * s, 0.02 * s), device="cpu")
    a_ref, o_ref = build_power_adjacency(sc["points"], sc["radii"])
    a, o = power_adjacency(sc["points"].cuda(), sc["radii"].cuda())
    assert torch.equal(o.cpu(), o_ref.to(torch.int32)) and torch.equal(a.cpu(), a_ref.to(torch.int32))


def test_power_adjacency_single_site():
    from powerfoam_b200.adjacency import power_adjacency

    a, o = power_adjacency(torch.zeros(1, 3, device="cuda"), torch.ones(1, device="cuda"))
    assert a.numel() == 0 and o.cpu().tolist() == [0, 0]


def test_power_adjacency_golden_trace_scene(golden):
    """The neighbour sets the reference's own build_power_adjacency produced
    for the tracer golden case.  Its lists repeat an edge that two
    tetrahedra name in opposite orders (torch.unique over unordered pairs,
    benchmark.py:53-59) and follow argsort order; the form here is ascending
    without repeats, the same sets (a repeated face yields the same exit, so
    cell walks do not change)."""
    from powerfoam_b200.adjacency import power_adjacency

    g = golden("trace_small")
    a, o = power_adjacency(to_t(g["points"]), to_t(g["radii"]))
    a, o = a.cpu().numpy(), o.cpu().numpy()
    ga, go = g["adjacency"], g["adjacency_offsets"]
    assert go[-1] > o[-1]  # the reference's lists carry repeats
    for i in range(len(go) - 1):
        assert a[o[i]:o[i + 1]].tolist() == sorted(set(ga[go[i]:go[i + 1]].tolist()))


def test_power_adjacency_capacity_growth_and_reuse():
    from powerfoam_b200 import _lib
    from oracle.power_hull import build_power_adjacency
    from powerfoam_b200.adjacency import PowerBuilder

    pts, radii = _power_case(6, 1500, "uniform")
    a_ref, o_ref = build_power_adjacency(torch.from_numpy(pts), torch.from_numpy(radii))
    b = PowerBuilder("cuda")
    for _ in range(2):  # workspace reused
        a, o = b(to_t(pts), to_t(radii))
        assert torch.equal(a.cpu(), a_ref.to(torch.int32)) and torch.equal(o.cpu(), o_ref.to(torch.int32))
    # a capacity below the edge count: true count, zeroed offsets, overflow status
    n = pts.shape[0]
    nbytes = _lib.ctypes.c_size_t(0)
    _lib.call("pf_power_workspace_size", n, _lib.ctypes.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    adj = torch.empty(16, dtype=torch.int32, device="cuda")
    off = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    sc = torch.zeros(2, dtype=torch.int64, device="cuda")
    st = sc[1:].view(torch.int32)[:1]
    p, r = to_t(pts), to_t(radii)
    _lib.call("pf_power_adjacency", _lib.ptr(p), _lib.ptr(r), n, 0, _lib.ptr(ws), ws.numel(), 16, _lib.ptr(adj),
              _lib.ptr(off), _lib.ptr(sc[:1]), _lib.ptr(st), _lib.stream_ptr())
    assert int(sc[0]) == a_ref.numel() and int(st[0]) == _lib.PF_ERR_OVERFLOW and not off.any()
