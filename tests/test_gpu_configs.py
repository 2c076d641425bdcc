"""Parity at the measured configurations (the sizes bench.py times).

* 16,384 primitives, 256x256, 60 degrees, eye (0,0,3): the whole frame at
  tile widths 8 and 16 -- binning (tile keys, sort order, offsets) bit-exact,
  the nine forward outputs within 1e-5 (contrib / point_err normwise), every
  gradient within 1e-4 normwise, against the oracle.
* raster1m (1,048,576 primitives, 1920x1080): the Čech adjacency, the fp16
  neighbour records and the full binning bit-exact; forward + adjoint of 288
  seeded tiles (256 random, the 32 longest lists) through the C ABI against
  the oracle on the same restricted lists; 64 seeded gradient entries against
  central differences of the float64 oracle.
* trace1m (1,048,576 primitives, 1280x720): visited-cell sequences of 8,192
  seeded rays bit-exact, and the whole frame's adjoint against the oracle's.

Tolerances: integer/index outputs bit-exact; images max-abs 1e-5; gradients
normwise relative 1e-4 (max |g - g_ref| <= 1e-4 max |g_ref|).
Reference lines: rasterize.py:140-363 (binning), :892-1146 (forward),
:1150-1514 (backward); raytrace.py:115-241 (walk)."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from powerfoam_b200 import _lib, synthetic
from powerfoam_b200.rasterize import Rasterizer, TileBins
from powerfoam_b200.raytrace import RayTracer
from tests.helpers import (FD_NAMES, PrimTiles, assert_close_rel, assert_quantiles_close, fd_gradient, max_abs, packed,
                           restrict_lists, vary_sites)

pytestmark = pytest.mark.gpu


class Args:
    is_pinhole = True
    render_objective = "volume"
    num_texel_sites = 8


def _np(t):
    return t.detach().cpu().numpy()


def _ocam(cam):
    return orc.camera(_np(cam.eye), _np(cam.right), _np(cam.up), cam.width, cam.height)


def _scene_np(scene, rgb):
    sc = {k: _np(v) for k, v in scene.items() if k != "sh"}
    sc["texel_rgb"] = _np(rgb)
    return sc


# ---------------------------------------------------------------------------
# 16,384 primitives, 256 x 256


def _frame_parity(R, cam, sc, adj, adj_off, tw, seed, check_sites):
    """Forward (dq, ray_gt, point_err) and adjoint (random upstream gradients
    of every output) of the whole frame against the oracle."""
    H, W = cam.height, cam.width
    N = sc["points"].shape[0]
    oc = _ocam(cam)
    sph, nsig, rgbh = packed(sc)
    keys, prims, offs, _ = orc.bin(oc, sph, tw)
    rng = np.random.default_rng(seed)
    dq = np.sort(rng.uniform(0.05, 0.95, (H, W, 2)).astype(np.float32), axis=-1)[..., ::-1].copy()
    gt = rng.uniform(0, 1, (H, W, 3)).astype(np.float32)
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    t = {k: cu(sc[k]).requires_grad_(True) for k in ("points", "radii", "density", "normals", "texel_sites",
                                                     "texel_rgb", "texel_height")}
    R.collect_stats = True
    out = R.forward(cam, cu(dq), t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    t["texel_rgb"], t["texel_height"], adj, adj_off, cu(gt), True)
    color, opacity, nd, normal, qd, err, contrib, perr, vis = out
    a_np, o_np = _np(adj), _np(adj_off)
    ad = orc.prefetch_adjacency(sph, a_np, o_np)
    o = orc.raster_forward(oc, tw, sph, nsig, sc["texel_sites"], rgbh, a_np, o_np, ad, offs, prims, dq, gt, 1e-3,
                           True)
    assert np.array_equal(_np(R.last_stats["early_stop"]), o["early_stop"])
    for a, ref in [(color, o["color"]), (nd, o["normal_distance"]), (normal, o["normal"])]:
        assert max_abs(_np(a), ref) <= 1e-5
    assert_quantiles_close(_np(qd), o["quantile_depths"])
    assert max_abs(_np(opacity), 1 - np.exp(o["log_t"])) <= 1e-5
    assert_close_rel(_np(contrib), o["contrib"], 1e-5, "contrib")
    assert_close_rel(_np(perr), o["point_err"], 1e-5, "point_err")
    visible = np.zeros(N, bool)
    visible[prims] = True
    assert np.array_equal(_np(vis), visible)
    g_c = rng.standard_normal((H, W, 3)).astype(np.float32)
    g_o = rng.standard_normal((H, W)).astype(np.float32)
    g_n = rng.standard_normal((H, W, 3)).astype(np.float32)
    g_nd = rng.standard_normal((H, W)).astype(np.float32)
    g_q = rng.standard_normal((H, W, 2)).astype(np.float32)
    g_con = (rng.standard_normal(N) * 100).astype(np.float32)
    # pixels whose quantile decisions differ (see assert_quantiles_close) get no quantile gradient
    g_q[(np.abs(_np(qd) - o["quantile_depths"]) > 1e-5).any(-1)] = 0.0
    loss = ((color * cu(g_c)).sum() + (opacity * cu(g_o)).sum() + (normal * cu(g_n)).sum() + (nd * cu(g_nd)).sum()
            + (qd * cu(g_q)).sum() + (contrib * cu(g_con)).sum())
    loss.backward()
    g_logt = (-g_o * np.exp(o["log_t"])).astype(np.float32)
    gr = orc.raster_backward(oc, tw, sph, nsig, sc["texel_sites"], rgbh, a_np, o_np, ad, offs, prims,
                             o["early_stop"], o["log_t"], g_c, g_logt, g_nd, g_n, g_con, dq, g_q)
    assert_close_rel(_np(t["points"].grad), gr["spheres"][:, :3], 1e-4, "points")
    assert_close_rel(_np(t["radii"].grad), gr["spheres"][:, 3], 1e-4, "radii")
    assert_close_rel(_np(t["normals"].grad), gr["nsigmas"][:, :3], 1e-4, "normals")
    assert_close_rel(_np(t["density"].grad), gr["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(_np(t["texel_rgb"].grad), gr["texel_rgb"], 1e-4, "rgb")
    assert_close_rel(_np(t["texel_height"].grad), gr["texel_height"], 1e-4, "height")
    if check_sites:
        assert_close_rel(_np(t["texel_sites"].grad), gr["texel_sites"], 1e-4, "sites")
    return offs, prims


@pytest.mark.parametrize("tw", [8, 16])
def test_raster16k_whole_frame(tw):
    """The scene as generated (colours equal on a primitive's sites, heights
    zero), then the same primitives with per-site colours and heights, where
    the texel-site gradient is well conditioned (vary_sites)."""
    cfg = synthetic.CONFIGS["raster16k"]
    scene = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=0, r_range=cfg["r_range"])
    cam = synthetic.front_camera(cfg["width"], cfg["height"], cfg["vfov"])
    rgb = synthetic.texel_rgb(scene, cam)
    sc = _scene_np(scene, rgb)
    sh = _np(scene["sh"])
    assert max_abs(rgb.cpu(), orc.sh_texel_rgb(sc["points"], sh, _np(cam.eye))) <= 1e-6
    from powerfoam_b200.adjacency import cech_adjacency, power_adjacency_diff

    adj, adj_off = cech_adjacency(scene["points"], scene["radii"])
    a_ref, o_ref = orc.cech_adjacency(sc["points"], sc["radii"])
    assert np.array_equal(_np(adj_off), o_ref) and np.array_equal(_np(adj), a_ref)
    R = Rasterizer(Args(), "cuda", tile_width=tw)
    sph, nsig, rgbh = packed(sc)
    keys, prims, offs, _ = orc.bin(_ocam(cam), sph, tw)
    b = R.bin(cam, torch.from_numpy(sph).cuda(), return_keys=True)
    assert b.n_pairs == keys.shape[0] > 0
    assert np.array_equal(_np(b.sort_keys), keys)
    assert np.array_equal(_np(b.tile_prims), prims)
    assert np.array_equal(_np(b.tile_offsets), offs)
    _frame_parity(R, cam, sc, adj, adj_off, tw, 16 + tw, check_sites=False)
    _frame_parity(R, cam, vary_sites(sc, 3), adj, adj_off, tw, 17 + tw, check_sites=True)

    # the reference's timed path (benchmark_kernel) on the same frame
    pm = power_adjacency_diff(scene["points"], scene["radii"], adj, adj_off)
    assert np.array_equal(_np(pm).view(np.uint16), orc.power_adjacency_diff(sc["points"], sc["radii"], _np(adj),
                                                                            _np(adj_off)))
    c = R.benchmark(cam, scene["points"], scene["radii"], scene["density"], scene["normals"], scene["texel_sites"], rgb,
                    scene["texel_height"], adj, adj_off, pm, 1e-3)
    ref = orc.raster_benchmark(_ocam(cam), tw, sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"],
                               _np(adj_off), _np(pm).view(np.uint16), offs, prims, 1e-3)
    assert max_abs(_np(c), ref) <= 1e-5


# ---------------------------------------------------------------------------
# raster1m: 1,048,576 primitives, 1920 x 1080


@pytest.fixture(scope="module")
def raster1m():
    cfg, scene, cam, adj, adj_off, target = synthetic.raster_workload("raster1m", "cuda")
    rgb = synthetic.texel_rgb(scene, cam)
    torch.cuda.synchronize()
    return dict(cfg=cfg, scene=scene, cam=cam, adj=adj, adj_off=adj_off, target=target, rgb=rgb,
                sc=_scene_np(scene, rgb), sh=_np(scene["sh"]))


def test_raster1m_adjacency_and_binning_bit_exact(raster1m):
    d = raster1m
    sc, cam = d["sc"], d["cam"]
    a_ref, o_ref = orc.cech_adjacency(sc["points"], sc["radii"])
    assert np.array_equal(_np(d["adj_off"]), o_ref)
    assert np.array_equal(_np(d["adj"]), a_ref)
    assert max_abs(_np(d["rgb"]), orc.sh_texel_rgb(sc["points"], d["sh"], _np(cam.eye))) <= 1e-6
    sph, _, _ = packed(sc)
    R = Rasterizer(Args(), "cuda")
    sph_t, _ = R.pack(d["scene"]["points"], d["scene"]["radii"])
    assert np.array_equal(_np(sph_t), sph)
    ad = R.prefetch_adjacency(sph_t, d["adj"], d["adj_off"])
    assert np.array_equal(_np(ad).view(np.uint16), orc.prefetch_adjacency(sph, a_ref, o_ref))
    keys, prims, offs, _ = orc.bin(_ocam(cam), sph, 8)
    b = R.bin(cam, sph_t, return_keys=True)
    assert b.n_pairs == keys.shape[0] > 3_000_000
    assert np.array_equal(_np(b.tile_offsets), offs)
    assert np.array_equal(_np(b.sort_keys), keys)
    assert np.array_equal(_np(b.tile_prims), prims)
    visible = np.zeros(sph.shape[0], bool)
    visible[prims] = True
    assert np.array_equal(_np(b.prim_visible), visible)


def _restricted_gpu(R, d, sph_t, nsig_t, offs, prims, ad_t, g_c, rgb_t, height_t):
    """Forward + adjoint through the C ABI over the given (restricted) tile
    lists, tiles in index order; returns numpy outputs and gradients."""
    cam = d["cam"]
    H, W = cam.height, cam.width
    N = sph_t.shape[0]
    bins = TileBins(torch.from_numpy(offs).cuda(), torch.from_numpy(prims).cuda(), int(prims.shape[0]), None)
    inp = R._inputs(cam, sph_t, nsig_t, d["scene"]["texel_sites"], rgb_t, height_t, d["adj"], d["adj_off"], ad_t,
                    bins)
    T = offs.shape[0] - 1
    f = lambda *s: torch.empty(s, dtype=torch.float32, device="cuda")  # noqa: E731
    color, log_t, nd, normal, contrib = f(H, W, 3), f(H, W), f(H, W), f(H, W, 3), f(N)
    es = torch.empty(T, dtype=torch.int32, device="cuda")
    _lib.call("pf_raster_forward", ctypes.byref(inp), 0, _lib.ptr(color), _lib.ptr(log_t), _lib.ptr(nd),
              _lib.ptr(normal), None, None, _lib.ptr(contrib), None, _lib.ptr(es), None, _lib.stream_ptr())
    S = rgb_t.shape[1]
    g = dict(points=f(N, 3), radii=f(N), normals=f(N, 3), density=f(N), sites=f(N, S, 3), rgb=f(N, S, 3),
             height=f(N, S))
    gc = torch.from_numpy(g_c).cuda()
    go = torch.zeros((H, W), dtype=torch.float32, device="cuda")
    _lib.call("pf_raster_backward", ctypes.byref(inp), _lib.ptr(es), _lib.ptr(log_t), _lib.ptr(gc), _lib.ptr(go), None,
              None, None, None, *[_lib.ptr(g[k]) for k in ("points", "radii", "normals", "density", "sites", "rgb",
                                                           "height")], _lib.stream_ptr())
    torch.cuda.synchronize()
    out = dict(color=_np(color), log_t=_np(log_t), nd=_np(nd), normal=_np(normal), contrib=_np(contrib),
               early_stop=_np(es))
    return out, {k: _np(v) for k, v in g.items()}


@pytest.mark.parametrize("varied", [False, True])
def test_raster1m_sampled_tiles_forward_and_adjoint(raster1m, varied):
    """288 tiles (256 seeded, the 32 longest lists) of the 1080p frame; the
    scene as generated and with per-site colours and heights (vary_sites),
    where the texel-site gradient is compared too."""
    d = raster1m
    sc, cam = d["sc"], d["cam"]
    if varied:
        sc = vary_sites(sc, 11)
    H, W = cam.height, cam.width
    sph, nsig, rgbh = packed(sc)
    oc = _ocam(cam)
    keys, prims, offs, _ = orc.bin(oc, sph, 8)
    T = offs.shape[0] - 1
    lens = np.diff(offs)
    rng = np.random.default_rng(1080)
    tiles = np.unique(np.concatenate([rng.choice(T, 256, replace=False), np.argsort(-lens, kind="stable")[:32]]))
    assert tiles.shape[0] >= 280 and lens[tiles].max() > 500
    ro, rp = restrict_lists(offs, prims, tiles)
    adj, adj_off = _np(d["adj"]), _np(d["adj_off"])
    ad = orc.prefetch_adjacency(sph, adj, adj_off)
    R = Rasterizer(Args(), "cuda")
    sph_t, nsig_t = R.pack(d["scene"]["points"], d["scene"]["radii"], d["scene"]["normals"], d["scene"]["density"])
    ad_t = R.prefetch_adjacency(sph_t, d["adj"], d["adj_off"])
    target = d["target"].numpy()
    o = orc.raster_forward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, ro, rp)
    g_c = (2.0 * (o["color"] - target)).astype(np.float32)
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    out, g = _restricted_gpu(R, d, sph_t, nsig_t, ro, rp, ad_t, g_c, cu(sc["texel_rgb"]), cu(sc["texel_height"]))
    assert np.array_equal(out["early_stop"], o["early_stop"])
    assert max_abs(out["color"], o["color"]) <= 1e-5
    assert max_abs(out["log_t"], o["log_t"]) <= 1e-5 * max(1.0, float(np.abs(o["log_t"]).max()))
    assert max_abs(out["nd"], o["normal_distance"]) <= 1e-5
    assert max_abs(out["normal"], o["normal"]) <= 1e-5
    assert_close_rel(out["contrib"], o["contrib"], 1e-5, "contrib")
    z = np.zeros((H, W), np.float32)
    gr = orc.raster_backward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, ro, rp, o["early_stop"],
                             o["log_t"], g_c, z, z, np.zeros((H, W, 3), np.float32),
                             np.zeros(sph.shape[0], np.float32))
    assert np.abs(gr["texel_rgb"]).max() > 0
    assert_close_rel(g["points"], gr["spheres"][:, :3], 1e-4, "points")
    assert_close_rel(g["radii"], gr["spheres"][:, 3], 1e-4, "radii")
    assert_close_rel(g["normals"], gr["nsigmas"][:, :3], 1e-4, "normals")
    assert_close_rel(g["density"], gr["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(g["rgb"], gr["texel_rgb"], 1e-4, "rgb")
    assert_close_rel(g["height"], gr["texel_height"], 1e-4, "height")
    if varied:
        assert_close_rel(g["sites"], gr["texel_sites"], 1e-4, "sites")


def test_raster1m_gradients_match_central_differences(raster1m):
    """64 seeded entries of the gradients of L = sum (color - target)^2 (the
    bench loss) with respect to points, radii, density, normals and texel
    colours, drawn among the entries the GPU adjoint makes non-zero.

    Two checks, because the reference's float32 arithmetic is itself far
    from the exact derivative here: for spheres of radius 0.002-0.02 seen
    from about 3 units the ray/sphere discriminant qb^2 - 4qc cancels
    catastrophically, so float32 segment lengths (and their gradients) of
    the small primitives carry errors of 10-100 % -- in the reference and,
    bit for bit, here.  Hence
    (1) the float64 oracle adjoint (exact neighbour spheres) against central
        differences of the float64 oracle forward, step 1e-3 of the input's
        scale: within 2e-2 |g| + 1e-4 max |g| of the category for at least
        60 of the 64 entries (a few steps cross a discrete event: a tile
        entry, a face becoming the bounding one);
    (2) the GPU adjoint against the float32 oracle adjoint (the reference's
        arithmetic, fp16 neighbour records) on the same entries, 1e-4
        normwise per category.
    Normals are turned to face the camera (within 60 degrees of the direction
    to it, so the texture plane bounds the near end of every ray through the
    sphere): the reference's adjoint routes dL/dt_far to both the texture
    plane and the surface it replaced when the plane bounds the far end
    (rasterize.py:1428-1433, 1466-1470), which is not the derivative of its
    forward; with the plane at the near end it is."""
    d = raster1m
    cam = d["cam"]
    H, W = cam.height, cam.width
    sc = dict(d["sc"])
    eye = _np(cam.eye)
    v = sc["points"] - eye
    v /= np.linalg.norm(v, axis=-1, keepdims=True)
    nrm = -v + 0.5 * sc["normals"]  # within 60 degrees of the direction to the camera
    sc["normals"] = (nrm / np.linalg.norm(nrm, axis=-1, keepdims=True)).astype(np.float32)
    scene = dict(d["scene"])
    scene["normals"] = torch.from_numpy(sc["normals"]).cuda()
    target = d["target"].numpy()

    R = Rasterizer(Args(), "cuda")
    t = {k: scene[k].clone().requires_grad_(True) for k in ("points", "radii", "density", "normals", "texel_sites",
                                                           "texel_height")}
    t["texel_rgb"] = d["rgb"].clone().requires_grad_(True)
    out = R.forward(cam, None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"], t["texel_rgb"],
                    t["texel_height"], d["adj"], d["adj_off"], None, False)
    ((out[0] - d["target"].cuda()) ** 2).sum().backward()
    G = {k: _np(t[k].grad) for k in FD_NAMES}

    rng = np.random.default_rng(64)
    chosen = []
    for i in range(64):
        name = FD_NAMES[i % len(FD_NAMES)]
        nz = np.argwhere(G[name] != 0)
        chosen.append((name, tuple(int(v) for v in nz[rng.integers(0, nz.shape[0])])))

    oc = _ocam(cam)
    adj, adj_off = _np(d["adj"]), _np(d["adj_off"])
    sph, nsig, rgbh = packed(sc)
    keys, prims, offs, _ = orc.bin(oc, sph, 8)
    pt = PrimTiles(keys, prims, offs)
    fds, tiles = [], []
    for name, idx in chosen:
        fd, tl = fd_gradient(oc, 8, sc, adj, adj_off, pt, target, name, idx, eps=1e-3)
        fds.append(fd)
        tiles.append(tl)
    U = np.unique(np.concatenate(tiles))
    ro, rp = restrict_lists(offs, prims, U)
    z = np.zeros((H, W), np.float32)
    zn = np.zeros((H, W, 3), np.float32)
    zc = np.zeros(sph.shape[0], np.float32)

    def oracle_grads(prec, ad):
        o = orc.raster_forward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, ro, rp, prec=prec)
        g_c = (2.0 * (o["color"] - target)).astype(np.float32)
        g = orc.raster_backward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, ro, rp, o["early_stop"],
                                o["log_t"].astype(np.float32), g_c, z, z, zn, zc, prec=prec)
        return dict(points=g["spheres"][:, :3], radii=g["spheres"][:, 3], density=g["nsigmas"][:, 3],
                    normals=g["nsigmas"][:, :3], texel_rgb=g["texel_rgb"])

    g64 = oracle_grads("f64", None)
    g32 = oracle_grads("f32", orc.prefetch_adjacency(sph, adj, adj_off))
    ok = 0
    rows = []
    for (name, idx), fd in zip(chosen, fds):
        scale = max(abs(float(g64[name][i])) for (n2, i) in chosen if n2 == name)
        an = float(g64[name][idx])
        good = abs(fd - an) <= 2e-2 * abs(an) + 1e-4 * scale
        ok += good
        rows.append((name, idx, fd, an, float(g32[name][idx]), float(G[name][idx]), good))
    assert ok >= 60, "\n".join(str(r) for r in rows)
    for name in FD_NAMES:
        sel = [idx for (n2, idx) in chosen if n2 == name]
        a = np.array([G[name][i] for i in sel])
        b = np.array([g32[name][i] for i in sel])
        assert_close_rel(a, b, 1e-4, name)


# ---------------------------------------------------------------------------
# trace1m: 1,048,576 primitives, 1280 x 720


@pytest.fixture(scope="module")
def trace1m():
    cfg, sc, cam, adj, off, pm, st = synthetic.trace_workload("trace1m", "cuda")
    rgb = synthetic.texel_rgb(sc, cam)
    torch.cuda.synchronize()
    return dict(cfg=cfg, scene=sc, cam=cam, adj=adj, off=off, pm=pm, start=st, rgb=rgb, sc=_scene_np(sc, rgb))


class TArgs:
    num_texel_sites = 8


def test_trace1m_visited_cells_bit_exact(trace1m):
    d = trace1m
    sc, cam = d["sc"], d["cam"]
    assert d["start"] == orc.start_cell(sc["points"], sc["radii"], _np(cam.eye))
    adj, off = _np(d["adj"]), _np(d["off"])
    assert np.array_equal(_np(d["pm"]).view(np.uint16), orc.power_adjacency_diff(sc["points"], sc["radii"], adj, off))
    cap = 1024
    tr = RayTracer(TArgs(), "cuda")
    s = d["scene"]
    r = tr.trace(cam, d["start"], s["points"], s["radii"], s["density"], s["normals"], s["texel_sites"], d["rgb"],
                 s["texel_height"], d["adj"], d["off"], d["pm"], 1e-3, visit_cap=cap)
    HW = cam.height * cam.width
    rng = np.random.default_rng(720)
    pix = np.sort(rng.choice(HW, 8192, replace=False))
    sph, nsig, _ = packed(sc)
    o = orc.trace_forward_pixels(_ocam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj,
                                 off, _np(d["pm"]).view(np.uint16), pix, d["start"], thr=1e-3, visit_cap=cap)
    assert o["rc"] == 0
    vc = _np(r.visit_count).reshape(-1)[pix]
    assert np.array_equal(vc, o["visit_count"])
    assert vc.max() <= cap and vc.mean() > 16
    pix_t = torch.from_numpy(pix).cuda()
    assert np.array_equal(_np(r.visits.reshape(HW, cap)[pix_t]), o["visits"])
    assert max_abs(_np(r.color).reshape(-1, 3)[pix], o["color"]) <= 1e-5
    assert max_abs(_np(r.normal).reshape(-1, 3)[pix], o["normal"]) <= 1e-5
    assert np.array_equal(_np(r.depth_seg).reshape(-1)[pix], o["depth_seg"])
    lt = _np(r.log_t).reshape(-1)[pix]
    assert max_abs(lt, o["log_t"]) <= 1e-5 * max(1.0, float(np.abs(o["log_t"]).max()))


@pytest.mark.parametrize("varied", [False, True])
def test_trace1m_adjoint_whole_frame(trace1m, varied):
    """The whole 1280x720 frame's walk + adjoint of L = sum (color - target)^2
    against the oracle's; the scene as generated and with per-site colours and
    heights (vary_sites), where the texel-site gradient is compared too."""
    d = trace1m
    sc, cam, s = d["sc"], d["cam"], d["scene"]
    if varied:
        sc = vary_sites(sc, 12)
    H, W = cam.height, cam.width
    tr = RayTracer(TArgs(), "cuda")
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    t = {k: cu(sc[k]).requires_grad_(True) for k in ("points", "radii", "density", "normals", "texel_sites",
                                                     "texel_rgb", "texel_height")}
    color, log_t, depth, normal = tr.forward(cam, d["start"], t["points"], t["radii"], t["density"], t["normals"],
                                             t["texel_sites"], t["texel_rgb"], t["texel_height"], d["adj"], d["off"],
                                             d["pm"])
    target = torch.rand((H, W, 3), generator=torch.Generator().manual_seed(202))
    ((color - target.cuda()) ** 2).sum().backward()
    sph, nsig, _ = packed(sc)
    args = (_ocam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], _np(d["adj"]),
            _np(d["off"]), _np(d["pm"]).view(np.uint16))
    f = orc.trace_forward(*args, d["start"], thr=1e-3)
    assert max_abs(_np(color), f["color"]) <= 1e-5
    g_c = (2.0 * (f["color"] - target.numpy())).astype(np.float32)
    g = orc.trace_backward(*args, f, g_c, None, None, None, d["start"], thr=1e-3)
    assert_close_rel(_np(t["points"].grad), g["spheres"][:, :3], 1e-4, "points")
    assert_close_rel(_np(t["radii"].grad), g["spheres"][:, 3], 1e-4, "radii")
    assert_close_rel(_np(t["normals"].grad), g["nsigmas"][:, :3], 1e-4, "normals")
    assert_close_rel(_np(t["density"].grad), g["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(_np(t["texel_rgb"].grad), g["texel_rgb"], 1e-4, "rgb")
    assert_close_rel(_np(t["texel_height"].grad), g["texel_height"], 1e-4, "height")
    if varied:
        assert_close_rel(_np(t["texel_sites"].grad), g["texel_sites"], 1e-4, "sites")


# ---------------------------------------------------------------------------
# The cycle guard at scale: 1,048,576 primitives of opaque shells, 2048 x 1536


def test_shells1m_cycling_rays_bit_exact():
    """On the shells scene some rays come back to a cell they walked (float16
    faces of neighbouring cells that disagree); before the cycle guard they
    ran to the 65,536-step cap.  The 2,048 longest walks of the frame and
    2,048 random rays: visited cells bit-exact against the oracle, every walk
    ends without the step cap, and the sample holds walks that revisit a cell
    (the guard's subjects)."""
    from powerfoam_b200.adjacency import power_adjacency, power_adjacency_diff, start_cell

    cfg = dict(synthetic.CONFIGS["trace6m"])
    n = 1048576
    r_scale = (cfg["n"] / n) ** (1 / 3)
    sc_t = synthetic.make_scene(n, seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"],
                                r_range=tuple(r * r_scale for r in cfg["r_range"]), shells=(0.12, 0.02, 30.0))
    adj, off = power_adjacency(sc_t["points"], sc_t["radii"])
    pm = power_adjacency_diff(sc_t["points"], sc_t["radii"], adj, off)
    cam = synthetic.orbit_camera(4242, 2048, 1536, cfg["vfov"])
    rgb = synthetic.texel_rgb(sc_t, cam)
    st = start_cell(sc_t["points"], sc_t["radii"], cam.eye)
    cap = 256
    tr = RayTracer(TArgs(), "cuda")
    r = tr.trace(cam, st, sc_t["points"], sc_t["radii"], sc_t["density"], sc_t["normals"], sc_t["texel_sites"], rgb,
                 sc_t["texel_height"], adj, off, pm, 1e-3, visit_cap=cap)  # raises on the step cap
    vc_all = _np(r.visit_count).reshape(-1)
    assert vc_all.max() <= cap
    HW = cam.height * cam.width
    longest = np.argsort(vc_all, kind="stable")[-2048:]
    rng = np.random.default_rng(4242)
    pix = np.unique(np.concatenate([longest, rng.choice(HW, 2048, replace=False)]))
    sc = _scene_np(sc_t, rgb)
    sph, nsig, _ = packed(sc)
    o = orc.trace_forward_pixels(_ocam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"],
                                 _np(adj), _np(off), _np(pm).view(np.uint16), pix, st, thr=1e-3, visit_cap=cap)
    assert o["rc"] == 0 and (o["status"] == 0).all()
    assert np.array_equal(vc_all[pix], o["visit_count"])
    pix_t = torch.from_numpy(pix).cuda()
    visits = _np(r.visits.reshape(HW, cap)[pix_t])
    assert np.array_equal(visits, o["visits"])
    assert max_abs(_np(r.color).reshape(-1, 3)[pix], o["color"]) <= 1e-5
    revisit = sum(len(set(v[v >= 0].tolist())) < int((v >= 0).sum()) for v in visits)
    assert revisit > 0
