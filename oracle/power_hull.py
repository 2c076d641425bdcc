"""The reference's power-diagram adjacency on the host (test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker of pf_power_adjacency and the CPU
baseline of bench.py's power-diagram workload; the product package never
imports it.  It restates build_power_adjacency (benchmark.py:25-83): lift the
points to (p, |p|^2 - r^2), take scipy's Qhull convex hull (the reference's
third-party algorithm; scipy==1.16.2 pinned at requirements.txt:3), keep the
facets whose normal points down in the lifted coordinate, and emit the
tetrahedra's edges.
"""

import numpy as np
import torch


def build_power_adjacency(points, radii, alpha_complex=False):
    """Weighted Delaunay adjacency (benchmark.py:25-83): lift (p, |p|^2 - r^2)
    to 4-D, keep the facets of the convex hull whose normal points down in the
    lifted coordinate, take the tetrahedra's edges; with ``alpha_complex`` keep
    only edges whose balls overlap.  Returns (adjacency int32 (E), offsets int32
    (N+1)) grouped by source vertex, neighbours ascending and without the
    repeats the reference's lists carry (it runs torch.unique over unordered
    pairs, so an edge two tetrahedra name in opposite orders appears twice)."""
    from scipy.spatial import ConvexHull

    p = points.detach().cpu().double()
    r = radii.detach().cpu().double()
    lifted = torch.cat([p, (p.norm(dim=-1) ** 2 - r**2)[:, None]], dim=-1).numpy()
    hull = ConvexHull(lifted)
    simp = hull.simplices[hull.equations[:, 3] < 0]
    pairs = np.concatenate([simp[:, [a, b]] for a, b in ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))], 0)
    pairs = np.unique(np.sort(pairs, axis=1), axis=0)
    if alpha_complex:
        d = np.linalg.norm(p.numpy()[pairs[:, 0]] - p.numpy()[pairs[:, 1]], axis=-1)
        pairs = pairs[d < (r.numpy()[pairs[:, 0]] + r.numpy()[pairs[:, 1]])]
    directed = np.concatenate([pairs, pairs[:, ::-1]], 0)
    order = np.lexsort((directed[:, 1], directed[:, 0]))
    directed = directed[order]
    n = points.shape[0]
    counts = np.bincount(directed[:, 0], minlength=n)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    dev = points.device
    return (torch.from_numpy(directed[:, 1].astype(np.int32)).to(dev), torch.from_numpy(offsets).to(dev))
