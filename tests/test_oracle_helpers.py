"""The oracle's helpers for the large-configuration parity tests, checked on
the CPU: the Čech restatement against brute force, the pixel-list walk
against the whole-frame walk, restricted tile lists and the float64
finite-difference routine against the float64 adjoint."""

import numpy as np
import pytest

from oracle import oracle as orc
from oracle.power_hull import build_power_adjacency
from tests.helpers import (FD_NAMES, PrimTiles, cech_np, fd_gradient, np_camera, np_scene, orc_cam, packed,
                           restrict_lists, tile_pixels)


@pytest.mark.parametrize("seed,n,rmax", [(0, 500, 0.15), (1, 3000, 0.06), (2, 4000, 0.02), (3, 1, 0.1)])
def test_cech_matches_bruteforce(seed, n, rmax):
    sc = np_scene(seed, n, -1.0, 1.0, rmax / 10, rmax)
    a, o = cech_np(sc["points"], sc["radii"])
    b, p = orc.cech_adjacency(sc["points"], sc["radii"])
    assert np.array_equal(o, p) and np.array_equal(a, b)


def test_trace_pixel_list_matches_whole_frame():
    import torch

    sc = np_scene(52, 300, -0.6, 0.6, 0.05, 0.15)
    cam = np_camera((0.3, 0.2, 2.2), (0, 0, 0), 24, 18, 55.0)
    adj, off = (t.numpy() for t in build_power_adjacency(torch.from_numpy(sc["points"]), torch.from_numpy(sc["radii"])))
    pm = orc.power_adjacency_diff(sc["points"], sc["radii"], adj, off)
    s = orc.start_cell(sc["points"], sc["radii"], cam["eye"])
    sph, nsig, _ = packed(sc)
    args = (orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj, off, pm)
    full = orc.trace_forward(*args, s, visit_cap=64)
    pix = np.array([0, 5, 17, 100, 431, 24 * 18 - 1], np.int64)
    sub = orc.trace_forward_pixels(*args, pix, s, visit_cap=64)
    assert sub["rc"] == 0
    assert np.array_equal(sub["visits"], full["visits"].reshape(-1, 64)[pix])
    assert np.array_equal(sub["visit_count"], full["visit_count"].reshape(-1)[pix])
    assert np.array_equal(sub["color"], full["color"].reshape(-1, 3)[pix])
    bad = orc.trace_forward_pixels(*args, np.array([24 * 18], np.int64), s)
    assert bad["rc"] == 3 and bad["status"][0] == 3  # ORC_ERR_ARGS for a pixel outside the image


def test_restricted_lists_and_fd_gradient():
    sc = np_scene(80, 400, -0.6, 0.6, 0.03, 0.12, height_scale=0.0, toward=(0.1, 0.2, 2.2))
    # one colour per primitive on all its sites, as the SH pre-step gives: the
    # reference's texture adjoint leaves out the soft-Voronoi weights'
    # dependence on the radius (texture.py:114-131 has no radius output), which
    # only matters when a primitive's sites differ
    sc["texel_rgb"] = np.repeat(sc["texel_rgb"][:, :1], sc["texel_rgb"].shape[1], axis=1).copy()
    cam = np_camera((0.1, 0.2, 2.2), (0, 0, 0), 40, 32, 55.0)
    adj, off = cech_np(sc["points"], sc["radii"])
    oc = orc_cam(cam)
    sph, nsig, rgbh = packed(sc)
    keys, prims, offs, _ = orc.bin(oc, sph, 8)
    T = offs.shape[0] - 1
    pt = PrimTiles(keys, prims, offs)
    # no change of any primitive's keys: the lists of the chosen tiles are the restricted ones
    tiles = np.array([0, 3, 7, T - 1])
    p = int(prims[offs[3]])
    a = pt.order[pt.first[p]:pt.first[p + 1]]
    ro, rp = restrict_lists(offs, prims, tiles)
    lo, lp = pt.lists_with(tiles, p, keys[a])
    assert np.array_equal(ro, lo) and np.array_equal(rp, lp)
    assert sorted(tile_pixels(T - 1, 32, 40, 8).tolist())[-1] == 32 * 40 - 1
    # central differences against the float64 adjoint of the whole frame
    target = np.random.default_rng(4).uniform(0, 1, (32, 40, 3)).astype(np.float32)
    o = orc.raster_forward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, off, None, offs, prims, prec="f64")
    g_c = (2 * (o["color"] - target)).astype(np.float32)
    z = np.zeros((32, 40), np.float32)
    g = orc.raster_backward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, off, None, offs, prims, o["early_stop"],
                            o["log_t"].astype(np.float32), g_c, z, z, np.zeros((32, 40, 3), np.float32),
                            np.zeros(400, np.float32), prec="f64")
    G = dict(points=g["spheres"][:, :3], radii=g["spheres"][:, 3], density=g["nsigmas"][:, 3],
             normals=g["nsigmas"][:, :3], texel_rgb=g["texel_rgb"])
    rng = np.random.default_rng(5)
    ok = 0
    for i in range(15):
        name = FD_NAMES[i % 5]
        nz = np.argwhere(np.abs(G[name]) > 1e-3 * np.abs(G[name]).max())
        idx = tuple(int(v) for v in nz[rng.integers(0, nz.shape[0])])
        fd, _ = fd_gradient(oc, 8, sc, adj, off, pt, target, name, idx)
        an = float(G[name][idx])
        ok += abs(fd - an) <= 2e-2 * abs(an) + 1e-4 * np.abs(G[name]).max()
    assert ok >= 13
