"""Steiner points (benchmark.py:93-180) on the GPU: the nearest-neighbour
radius query against scipy's cKDTree (the reference's), and the whole
get_steiner_points against the golden run of the reference's own function
with the same random draws (tests/golden/steiner_small.npz)."""

import numpy as np
import pytest
import torch

from powerfoam_b200.steiner import get_steiner_points, greedy_min_overlap, knn_min_radius

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,n,m", [(0, 2000, 3000), (1, 50000, 20000)])
def test_knn_min_radius_matches_kdtree(seed, n, m):
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pts = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    pts[: n // 3] = (rng.standard_normal((n // 3, 3)) * 0.1).astype(np.float32)  # a dense cluster
    radii = np.exp(rng.uniform(np.log(0.005), np.log(0.05), n)).astype(np.float32)
    q = (rng.standard_normal((m, 3)) * 0.8).astype(np.float32)  # some queries outside the cloud's box
    d, idx = cKDTree(pts).query(q, k=32)
    v = d.astype(np.float32) - radii[idx]
    ref_r = v.min(1)
    ref_i = idx[np.arange(m), v.argmin(1)]
    r, i = knn_min_radius(torch.from_numpy(pts).cuda(), torch.from_numpy(radii).cuda(), torch.from_numpy(q).cuda())
    assert np.array_equal(r.cpu().numpy().view(np.uint32), ref_r.view(np.uint32))
    assert np.array_equal(i.cpu().numpy(), ref_i)


def test_greedy_selection_properties():
    rng = np.random.default_rng(4)
    p = torch.from_numpy(rng.uniform(-1, 1, (5000, 3)).astype(np.float32)).cuda()
    r = torch.from_numpy(rng.uniform(0.02, 0.08, 5000).astype(np.float32)).cuda()
    sel = greedy_min_overlap(p, r, seed_index=17, threshold=0.1)
    s = torch.nonzero(sel).squeeze(1)
    assert bool(sel[17]) and s.numel() > 50
    d = torch.cdist(p[s], p[s])
    sr = r[s][:, None] + r[s][None, :]
    ov = (sr - d) / sr
    ov.fill_diagonal_(-1)
    assert float(ov.max()) <= 0.1 + 1e-6  # no two selected overlap by more than the threshold
    # every unselected sample overlaps some selected one by more than the threshold
    rest = torch.nonzero(~sel).squeeze(1)
    d2 = torch.cdist(p[rest], p[s])
    sr2 = r[rest][:, None] + r[s][None, :]
    assert bool((((sr2 - d2) / sr2).max(1).values > 0.1 - 1e-6).all())


def test_get_steiner_points_matches_reference_run(golden):
    g = golden("steiner_small")
    pts = torch.from_numpy(g["points"]).cuda()
    radii = torch.from_numpy(g["radii"]).cuda()
    samples = torch.from_numpy(g["samples"])
    seeds = g["seeds"]
    sp, sr = get_steiner_points(pts, radii, None, sampler=lambda r, n: samples[r],
                                seed_index=lambda r, n: int(seeds[r]))
    assert sp.shape == g["steiner_points"].shape
    assert np.array_equal(sp.cpu().numpy(), g["steiner_points"])
    np.testing.assert_allclose(sr.cpu().numpy(), g["steiner_radii"], rtol=1e-6, atol=1e-7)
