"""GPU Čech adjacency and Morton order against host restatements."""

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
