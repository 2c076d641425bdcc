"""Finite-difference checks of the adjoints on the float64 oracle.

The tracer adjoint has no counterpart in the reference; it is pinned here by
central differences of the float64 forward.  The rasterizer adjoint is the
reference's, including its known double routing of dL/dt_far when the
texture plane bounds the far end (rasterize.py:1428-1433 with :1466-1470), so
its check uses primitives whose normals face the camera (the plane then
bounds the near end) and exact texel heights of zero."""

import numpy as np
import pytest

from oracle import oracle as orc
from tests.helpers import cech_np, np_camera, np_scene, orc_cam, packed

F32 = np.float32


def _power_adj(sc):
    import torch

    from oracle.power_hull import build_power_adjacency

    a, o = build_power_adjacency(torch.from_numpy(sc["points"]), torch.from_numpy(sc["radii"]))
    return a.numpy(), o.numpy()


def _perturb(arr, idx, eps):
    a = arr.copy()
    x = float(a[idx])
    h = max(abs(x), 1e-2) * eps
    a[idx] = F32(x + h)
    hp = float(a[idx]) - x
    b = arr.copy()
    b[idx] = F32(x - h)
    hm = x - float(b[idx])
    return a, b, hp + hm


def test_tracer_adjoint_matches_central_differences():
    sc = np_scene(70, 160, -0.6, 0.6, 0.08, 0.2, height_scale=0.2)
    cam = np_camera((0.2, 0.25, 2.2), (0, 0, 0), 14, 12, 55.0)
    adj, off = _power_adj(sc)
    oc = orc_cam(cam)
    rng = np.random.default_rng(3)
    H, W = cam["height"], cam["width"]
    wC = rng.standard_normal((H, W, 3)).astype(F32)
    wL = rng.standard_normal((H, W)).astype(F32)
    wD = rng.standard_normal((H, W)).astype(F32)
    wN = rng.standard_normal((H, W, 3)).astype(F32)
    start = orc.start_cell(sc["points"], sc["radii"], cam["eye"])

    def run(s):
        # exact face encoding (adj_diff None): the float16 one is piecewise constant in the positions
        sph, nsig, _ = packed(s)
        pm = None
        f = orc.trace_forward(oc, sph, nsig, s["texel_sites"], s["texel_rgb"], s["texel_height"], adj, off, pm, start,
                              visit_cap=64, prec="f64")
        loss = float((f["color"] * wC).sum() + (f["log_t"] * wL).sum() + (f["depth"] * wD).sum()
                     + (f["normal"] * wN).sum())
        return f, loss, pm

    f0, _, pm0 = run(sc)
    sph, nsig, _ = packed(sc)
    g = orc.trace_backward(oc, sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj, off, pm0, f0,
                           wC, wL, wD, wN, start, prec="f64")
    grads = dict(points=g["spheres"][:, :3], radii=g["spheres"][:, 3], density=g["nsigmas"][:, 3],
                 normals=g["nsigmas"][:, :3], texel_sites=g["texel_sites"], texel_rgb=g["texel_rgb"],
                 texel_height=g["texel_height"])
    checked = 0
    for name in ["points", "radii", "density", "normals", "texel_sites", "texel_rgb", "texel_height"]:
        an_all = grads[name]
        cand = np.argwhere(np.abs(an_all) > 1e-3 * np.abs(an_all).max())
        rng.shuffle(cand)
        for idx in [tuple(c) for c in cand[:6]]:
            a, b, h = _perturb(sc[name], idx, 1e-4)
            fa, la, _ = run({**sc, name: a})
            fb, lb, _ = run({**sc, name: b})
            same_walk = (np.array_equal(fa["visits"], f0["visits"]) and np.array_equal(fb["visits"], f0["visits"])
                         and np.array_equal(fa["depth_seg"], f0["depth_seg"])
                         and np.array_equal(fb["depth_seg"], f0["depth_seg"]))
            if not same_walk:
                continue
            fd = (la - lb) / h
            an = float(an_all[idx])
            assert abs(fd - an) <= 2e-3 * abs(an) + 1e-6 * np.abs(an_all).max() + 1e-7, (name, idx, fd, an)
            checked += 1
    assert checked >= 20


def test_raster_adjoint_matches_central_differences_where_the_reference_is_exact():
    sc = np_scene(71, 150, -0.6, 0.6, 0.06, 0.2, height_scale=0.0, toward=(0.1, 0.2, 2.2))
    cam = np_camera((0.1, 0.2, 2.2), (0, 0, 0), 16, 16, 55.0)
    adj, off = cech_np(sc["points"], sc["radii"])
    oc = orc_cam(cam)
    rng = np.random.default_rng(5)
    wC = rng.standard_normal((16, 16, 3)).astype(F32)

    def run(s):
        sph, nsig, rgbh = packed(s)
        keys, prims, offs, _ = orc.bin(oc, sph, 8)
        ad = None  # exact neighbour spheres (the float16 encoding is piecewise constant)
        f = orc.raster_forward(oc, 8, sph, nsig, s["texel_sites"], rgbh, adj, off, ad, offs, prims, prec="f64")
        return f, float((f["color"] * wC).sum()), (keys, prims, offs, ad)

    f0, _, (keys, prims, offs, ad) = run(sc)
    sph, nsig, rgbh = packed(sc)
    z = np.zeros((16, 16), F32)
    g = orc.raster_backward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, off, ad, offs, prims, f0["early_stop"],
                            f0["log_t"], wC, z, z, np.zeros((16, 16, 3), F32), np.zeros(150, F32), prec="f64")
    grads = dict(points=g["spheres"][:, :3], density=g["nsigmas"][:, 3], texel_rgb=g["texel_rgb"])
    checked = 0
    for name, an_all in grads.items():
        cand = np.argwhere(np.abs(an_all) > 1e-2 * np.abs(an_all).max())
        rng.shuffle(cand)
        for idx in [tuple(c) for c in cand[:8]]:
            a, b, h = _perturb(sc[name], idx, 1e-4)
            fa, la, ka = run({**sc, name: a})
            fb, lb, kb = run({**sc, name: b})
            if not (np.array_equal(ka[0] >> 32, keys >> 32) and np.array_equal(kb[0] >> 32, keys >> 32)):
                continue
            fd = (la - lb) / h
            an = float(an_all[idx])
            assert abs(fd - an) <= 5e-3 * abs(an) + 1e-5 * np.abs(an_all).max() + 1e-7, (name, idx, fd, an)
            checked += 1
    assert checked >= 10
