"""Generate golden vectors by executing the reference's own kernel source.

Imports powerfoam/rasterize.py, raytrace.py, geometry.py and color_fn.py (and
functions of benchmark.py) from the reference checkout named by
$PF_REFERENCE (required) with warp replaced by tests/golden/warp_shim.py, runs
the kernels on small seeded scenes, and writes tests/golden/*.npz.  Run from
the repository root:

    PF_REFERENCE=<path of the powerfoam checkout> python tests/golden/make_golden.py

The fixtures are committed; tests read only the .npz files.
"""

import ast
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("PF_REFERENCE")
if not REF or not os.path.isdir(os.path.join(REF, "powerfoam")):
    sys.exit("set PF_REFERENCE to the reference checkout (the directory holding powerfoam/ and benchmark.py)")
sys.path.insert(0, HERE)
import warp_shim  # noqa: E402

wp = warp_shim.install()
sys.path.insert(0, REF)
import torch  # noqa: E402

import powerfoam.camera as rcam  # noqa: E402
import powerfoam.geometry as rgeo  # noqa: E402
import powerfoam.rasterize as rras  # noqa: E402
import powerfoam.raytrace as rtrace  # noqa: E402
import powerfoam.rendering_math as rmath  # noqa: E402
import powerfoam.texture as rtex  # noqa: E402

for m in (rcam, rgeo, rras, rtrace, rmath, rtex):
    warp_shim.patch_module_builtins(m)
warp_shim.patch_camera_module(rcam, wp)

F32 = np.float32
TILE_WIDTH = rras.TILE_WIDTH


def load_power_adjacency_fn():
    """Extract build_power_adjacency from benchmark.py (its module imports
    training-only dependencies) and compile it on its own."""
    src = open(os.path.join(REF, "benchmark.py")).read()
    tree = ast.parse(src)
    fn = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "build_power_adjacency"][0]
    mod = ast.Module(body=[fn], type_ignores=[])
    from scipy.spatial import ConvexHull

    ns = {"torch": torch, "ConvexHull": ConvexHull}
    exec(compile(mod, "benchmark.py", "exec"), ns)
    return ns["build_power_adjacency"]


# ----------------------------------------------------------------------------
# scene construction (seeded; float32 throughout)
def quat_frames(q):
    """Normals/tangents/bitangents from unit quaternions (scene.py:242-285)."""
    q = q / np.linalg.norm(q, axis=-1, keepdims=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    n = np.stack([1 - 2 * (y**2 + z**2), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1)
    t = np.stack([2 * (x * y + z * w), 1 - 2 * (x**2 + z**2), 2 * (y * z - x * w)], -1)
    b = np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x**2 + y**2)], -1)
    f = lambda v: (v / np.linalg.norm(v, axis=-1, keepdims=True)).astype(F32)
    return f(n), f(t), f(b)


def make_scene(seed, N, lo, hi, rmin, rmax, S=8, height_scale=0.1, toward=None):
    rng = np.random.default_rng(seed)
    pts = rng.uniform(lo, hi, size=(N, 3)).astype(F32)
    radii = np.exp(rng.uniform(np.log(rmin), np.log(rmax), N)).astype(F32)
    dens = (np.log1p(np.exp(rng.standard_normal(N))) * 10).astype(F32)
    q = rng.standard_normal((N, 4))
    n, t, b = quat_frames(q)
    if toward is not None:
        # orient normals against the view direction (used by FD cases)
        v = pts - np.asarray(toward, F32)
        s = np.sign(np.sum(n * v, -1, keepdims=True))
        n = (-n * s).astype(F32)
    s2 = (rng.standard_normal((N, S, 2)) * 0.1).astype(F32)
    off = s2 * radii[:, None, None]
    off = off[..., 0:1] * t[:, None, :] + off[..., 1:2] * b[:, None, :]
    sites = (pts[:, None, :] + off).astype(F32)
    rgb = rng.uniform(0.0, 1.0, size=(N, S, 3)).astype(F32)
    height = (rng.standard_normal((N, S)) * height_scale * radii[:, None]).astype(F32)
    return dict(points=pts, radii=radii, density=dens, normals=n, texel_sites=sites, texel_rgb=rgb,
                texel_height=height)


def cech_adjacency(points, radii):
    """bvh.py:7-69 semantics (overlapping balls, centre and radius recovered
    from the AABB as the kernels do), lists in ascending neighbour order."""
    lo = (points - radii[:, None]).astype(F32)
    hi = (points + radii[:, None]).astype(F32)
    c = (F32(0.5) * (lo + hi)).astype(F32)
    r = (F32(0.5) * (hi[:, 0] - lo[:, 0])).astype(F32)
    N = points.shape[0]
    adj, off = [], [0]
    for i in range(N):
        d = c[i][None, :] - c
        dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(F32)
        ov = np.all(lo[i] <= hi, axis=1) & np.all(hi[i] >= lo, axis=1)
        m = ov & (dist < (r[i] + r)) & (np.arange(N) != i)
        js = np.nonzero(m)[0]
        adj.extend(js.tolist())
        off.append(len(adj))
    return np.array(adj, dtype=np.int32), np.array(off, dtype=np.int32)


def look_at_camera(eye, target, W, H, vfov_deg, up_w=(0.0, 1.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, up_w)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    th = np.tan(np.radians(vfov_deg) / 2)
    return dict(eye=eye.astype(F32), right=(r * th * W / H).astype(F32), up=(u * th).astype(F32),
                width=W, height=H)


def warp_camera(cam):
    c = rcam.WarpCamera()
    c.eye = cam["eye"].copy()
    c.right = cam["right"].copy()
    c.up = cam["up"].copy()
    c.width = warp_shim.CInt(cam["width"])
    c.height = warp_shim.CInt(cam["height"])
    c.ray_maps = None
    c.fov_cos_cutoff = F32(0.0)
    return c


class Args:
    is_pinhole = True
    render_objective = "volume"
    num_texel_sites = 8
    disable_coop_prim_load = False
    disable_coop_adj_load = False


# ----------------------------------------------------------------------------
def run_binning(R, wcam, spheres):
    """rasterize.py:1671-1768 with the reference's kernels; the stable argsort
    gives equal keys in emission order, which is primitive order here."""
    N = spheres.shape[0]
    H, W = int(wcam.height), int(wcam.width)
    tiles_h = 1 + (H - 1) // TILE_WIDTH
    tiles_w = 1 + (W - 1) // TILE_WIDTH
    T = tiles_h * tiles_w
    counts = np.zeros(T + 1, np.int32)
    wp.launch(R.count_visible_kernel, dim=N, inputs=[wcam, spheres, counts])
    offsets = np.cumsum(counts.astype(np.int64))
    n = int(offsets[-1])
    prims = np.zeros(n, np.int32)
    keys = np.zeros(n, np.int64)
    wc = np.zeros(T, np.int32)
    wp.launch(R.write_visible_kernel, dim=N, inputs=[wcam, spheres, offsets, prims, keys, wc])
    perm = np.argsort(keys, kind="stable")
    return keys[perm], prims[perm], offsets, T


def raster_case(name, scene, cam, seed, Q=3, thr=1e-3, bench_thr=1e-2):
    t0 = time.time()
    R = rras.Rasterizer(Args(), "cpu", "float")
    wcam = warp_camera(cam)
    N = scene["points"].shape[0]
    H, W = cam["height"], cam["width"]
    spheres = np.concatenate([scene["points"], scene["radii"][:, None]], -1).astype(F32)
    nsig = np.concatenate([scene["normals"], scene["density"][:, None]], -1).astype(F32)
    rgbh = np.concatenate([scene["texel_rgb"], scene["texel_height"][..., None]], -1).astype(F32)
    adj, adj_off = cech_adjacency(scene["points"], scene["radii"])
    keys, prims, offsets, T = run_binning(R, wcam, spheres)

    adj_diff = np.zeros((adj.shape[0], 4), np.float16)
    wp.launch(R.prefetch_adjacency_kernel, dim=N, inputs=[spheres, adj, adj_off, adj_diff, N])

    rng = np.random.default_rng(seed + 1000)
    dq = np.sort(rng.uniform(0.05, 0.95, (H, W, Q)).astype(F32), axis=-1)[..., ::-1].copy()
    gt = rng.uniform(0, 1, (H, W, 3)).astype(F32)
    color = np.zeros((H, W, 3), F32)
    log_t = np.zeros((H, W), F32)
    nd = np.zeros((H, W), F32)
    normal = np.zeros((H, W, 3), F32)
    qd = -np.ones((H, W, Q), F32)
    contrib = np.zeros(N, F32)
    perr = np.zeros(N, F32)
    es = np.zeros(T, np.int32)
    TS = TILE_WIDTH * TILE_WIDTH
    wp.launch(R.forward_kernel, dim=T * TS, block_dim=TS, cooperative=True, inputs=[
        wcam, dq, True, spheres, nsig, scene["texel_sites"], rgbh, adj, adj_off, adj_diff, prims,
        offsets, es, gt, F32(thr), True, color, log_t, nd, normal, qd, None, contrib, perr])
    t1 = time.time()

    g_color = rng.standard_normal((H, W, 3)).astype(F32)
    g_opac = rng.standard_normal((H, W)).astype(F32)
    g_nd = rng.standard_normal((H, W)).astype(F32)
    g_normal = rng.standard_normal((H, W, 3)).astype(F32)
    g_qd = rng.standard_normal((H, W, Q)).astype(F32)
    g_contrib = (rng.standard_normal(N) * 100).astype(F32)
    g_logt = (-g_opac * np.exp(log_t)).astype(F32)  # rasterize.py:1905
    sg = np.zeros((N, 4), F32)
    ng = np.zeros((N, 4), F32)
    tsg = np.zeros((N, 8, 3), F32)
    trg = np.zeros((N, 8, 3), F32)
    thg = np.zeros((N, 8), F32)
    wp.launch(R.backward_kernel, dim=T * TS, block_dim=TS, cooperative=True, inputs=[
        wcam, dq, True, spheres, nsig, scene["texel_sites"], rgbh, adj, adj_off, adj_diff, prims,
        offsets, es, gt, color, log_t, g_color, g_logt, g_nd, g_normal, g_qd, None, g_contrib,
        sg, ng, tsg, trg, thg])
    for a in (sg, ng, tsg, trg, thg):
        a[~np.isfinite(a)] = 0
    t2 = time.time()

    # benchmark path: (dc, dpm) encoded neighbours, rasterize.py:614-734
    pm = F32(0.5) * (np.sqrt((scene["points"] ** 2).sum(-1)).astype(F32) ** 2 - scene["radii"] ** 2)
    pm = pm.astype(F32)
    cnt = np.diff(adj_off)
    self_pts = np.repeat(scene["points"], cnt, axis=0)
    adj_diff_pm = np.concatenate([scene["points"][adj] - self_pts,
                                  (pm[adj] - np.repeat(pm, cnt))[:, None]], -1).astype(np.float16)
    bcolor = np.zeros((H, W, 3), F32)
    wp.launch(R.benchmark_kernel, dim=T * TS, inputs=[
        wcam, spheres, nsig, scene["texel_sites"], scene["texel_rgb"], scene["texel_height"], adj, adj_off,
        adj_diff_pm, prims, offsets, F32(bench_thr), bcolor])

    # viewer path, rasterize.py:738-888 with the default VisOptions of :2145-2149
    # plus depth_quantile 0.5
    opt = rras.VisOptions()
    opt.transmittance_threshold = F32(1e-3)
    opt.max_intersections = warp_shim.CInt(1024)
    opt.depth_quantile = F32(0.5)
    opt.bkgd_color = np.zeros(3, F32)
    vc, vd, vn, va = (np.zeros((H, W, 3), F32), np.zeros((H, W), F32), np.zeros((H, W, 3), F32),
                      np.zeros((H, W), F32))
    vi = np.zeros((H, W), np.int32)
    wp.launch(R.visualization_kernel, dim=T * TS, inputs=[
        wcam, spheres, nsig, scene["texel_sites"], rgbh, scene["texel_rgb"], scene["texel_height"], adj,
        adj_off, adj_diff, prims, offsets, opt, vc, vd, vn, va, vi])
    t3 = time.time()

    out = dict(cam_eye=cam["eye"], cam_right=cam["right"], cam_up=cam["up"], width=W, height=H,
               tile_width=TILE_WIDTH, thr=F32(thr), bench_thr=F32(bench_thr), **scene,
               adjacency=adj, adjacency_offsets=adj_off, sort_keys=keys, tile_prims=prims,
               tile_offsets=offsets, adjacency_diff=adj_diff.view(np.uint16),
               adjacency_diff_pm=adj_diff_pm.view(np.uint16), depth_quantiles=dq, ray_gt=gt,
               color=color, log_t=log_t, normal_distance=nd, normal=normal, quantile_depths=qd,
               contrib=contrib, point_err=perr, early_stop=es, grad_color=g_color,
               grad_opacity=g_opac, grad_normal_distance=g_nd, grad_normal=g_normal,
               grad_quantile_depths=g_qd, grad_contrib=g_contrib, grad_log_t=g_logt,
               spheres_grad=sg, nsigmas_grad=ng, texel_sites_grad=tsg, texel_rgb_grad=trg,
               texel_height_grad=thg, bench_color=bcolor, vis_color=vc, vis_depth=vd, vis_normal=vn,
               vis_alpha=va, vis_intersections=vi)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: N={N} {W}x{H} pairs={keys.shape[0]} E={adj.shape[0]} "
          f"fwd {t1 - t0:.1f}s bwd {t2 - t1:.1f}s bench+vis {t3 - t2:.1f}s")


class ArgsGeneric(Args):
    is_pinhole = False


def run_cones(R, wcam, H, W):
    """Rasterizer._precompute_cones (rasterize.py:1518-1585) with the
    reference's cone kernels."""
    leaf = rras.LEAF_SIZE
    dh, dw = (H + leaf - 1) // leaf, (W + leaf - 1) // leaf
    offs, dhs, dws, total = [], [], [], 0
    while True:
        offs.append(total)
        dhs.append(dh)
        dws.append(dw)
        total += dh * dw
        if dh == 1 and dw == 1:
            break
        dh, dw = (dh + 1) // 2, (dw + 1) // 2
    tile_level, sz = 0, leaf
    while sz < TILE_WIDTH:
        tile_level += 1
        sz *= 2
    cones = np.zeros((total, 4), F32)
    wp.launch(R.compute_leaf_cones_kernel, dim=dhs[0] * dws[0], inputs=[wcam, cones, dws[0]])
    for l in range(1, len(offs)):
        wp.launch(R.merge_cones_kernel, dim=dhs[l] * dws[l],
                  inputs=[cones, offs[l], offs[l - 1], dws[l], dhs[l - 1], dws[l - 1]])
    return (cones, np.array(offs, np.int32), np.array(dhs, np.int32), np.array(dws, np.int32), len(offs),
            tile_level)


def run_binning_generic(R, wcam, spheres, cone_args):
    """The generic-camera branch of rasterize.py:1681-1768."""
    N = spheres.shape[0]
    H, W = int(wcam.height), int(wcam.width)
    T = (1 + (H - 1) // TILE_WIDTH) * (1 + (W - 1) // TILE_WIDTH)
    counts = np.zeros(T + 1, np.int32)
    wp.launch(R.count_visible_kernel, dim=N, inputs=[wcam, spheres, *cone_args, counts])
    offsets = np.cumsum(counts.astype(np.int64))
    n = int(offsets[-1])
    prims = np.zeros(n, np.int32)
    keys = np.zeros(n, np.int64)
    wc = np.zeros(T, np.int32)
    wp.launch(R.write_visible_kernel, dim=N, inputs=[wcam, spheres, *cone_args, offsets, prims, keys, wc])
    perm = np.argsort(keys, kind="stable")
    return keys[perm], prims[perm], offsets, T


def fisheye_ray_maps(cam, fov_deg, scale=1.7, shift=0.02):
    """A generic camera: equidistant fisheye directions (length `scale`, so the
    kernels' normalisation is exercised) from per-pixel origins spread along
    the image axes by up to `shift`."""
    H, W = cam["height"], cam["width"]
    r_hat = cam["right"] / np.linalg.norm(cam["right"])
    u_hat = cam["up"] / np.linalg.norm(cam["up"])
    f = np.cross(cam["up"], cam["right"])
    f = f / np.linalg.norm(f)
    jj, ii = np.meshgrid(np.arange(W), np.arange(H))
    x = 2.0 * jj / (W - 1) - 1.0
    y = 1.0 - 2.0 * ii / (H - 1)
    rad = np.sqrt(x * x + y * y)
    th = rad * np.deg2rad(fov_deg) / 2.0
    s = np.where(rad > 0, np.sin(th) / np.maximum(rad, 1e-12), 0.0)
    d = (np.cos(th)[..., None] * f + (s * x)[..., None] * r_hat + (s * y)[..., None] * u_hat) * scale
    o = cam["eye"] + shift * (x[..., None] * r_hat + y[..., None] * u_hat)
    return np.concatenate([o, d], -1).astype(F32)


def generic_case(name, scene, cam, ray_maps, seed, Q=3, thr=1e-3):
    """Binning through the cone hierarchy and the forward / adjoint with
    per-pixel rays (is_pinhole=False)."""
    t0 = time.time()
    R = rras.Rasterizer(ArgsGeneric(), "cpu", "float")
    wcam = warp_camera(cam)
    wcam.ray_maps = ray_maps
    N = scene["points"].shape[0]
    H, W = cam["height"], cam["width"]
    spheres = np.concatenate([scene["points"], scene["radii"][:, None]], -1).astype(F32)
    nsig = np.concatenate([scene["normals"], scene["density"][:, None]], -1).astype(F32)
    rgbh = np.concatenate([scene["texel_rgb"], scene["texel_height"][..., None]], -1).astype(F32)
    adj, adj_off = cech_adjacency(scene["points"], scene["radii"])
    cone_args = run_cones(R, wcam, H, W)
    keys, prims, offsets, T = run_binning_generic(R, wcam, spheres, cone_args)
    adj_diff = np.zeros((adj.shape[0], 4), np.float16)
    wp.launch(R.prefetch_adjacency_kernel, dim=N, inputs=[spheres, adj, adj_off, adj_diff, N])
    rng = np.random.default_rng(seed + 1000)
    dq = np.sort(rng.uniform(0.05, 0.95, (H, W, Q)).astype(F32), axis=-1)[..., ::-1].copy()
    gt = rng.uniform(0, 1, (H, W, 3)).astype(F32)
    color = np.zeros((H, W, 3), F32)
    log_t = np.zeros((H, W), F32)
    nd = np.zeros((H, W), F32)
    normal = np.zeros((H, W, 3), F32)
    qd = -np.ones((H, W, Q), F32)
    contrib = np.zeros(N, F32)
    perr = np.zeros(N, F32)
    es = np.zeros(T, np.int32)
    TS = TILE_WIDTH * TILE_WIDTH
    wp.launch(R.forward_kernel, dim=T * TS, block_dim=TS, cooperative=True, inputs=[
        wcam, dq, True, spheres, nsig, scene["texel_sites"], rgbh, adj, adj_off, adj_diff, prims,
        offsets, es, gt, F32(thr), True, color, log_t, nd, normal, qd, None, contrib, perr])
    t1 = time.time()
    g_color = rng.standard_normal((H, W, 3)).astype(F32)
    g_opac = rng.standard_normal((H, W)).astype(F32)
    g_nd = rng.standard_normal((H, W)).astype(F32)
    g_normal = rng.standard_normal((H, W, 3)).astype(F32)
    g_qd = rng.standard_normal((H, W, Q)).astype(F32)
    g_contrib = (rng.standard_normal(N) * 100).astype(F32)
    g_logt = (-g_opac * np.exp(log_t)).astype(F32)
    sg = np.zeros((N, 4), F32)
    ng = np.zeros((N, 4), F32)
    tsg = np.zeros((N, 8, 3), F32)
    trg = np.zeros((N, 8, 3), F32)
    thg = np.zeros((N, 8), F32)
    wp.launch(R.backward_kernel, dim=T * TS, block_dim=TS, cooperative=True, inputs=[
        wcam, dq, True, spheres, nsig, scene["texel_sites"], rgbh, adj, adj_off, adj_diff, prims,
        offsets, es, gt, color, log_t, g_color, g_logt, g_nd, g_normal, g_qd, None, g_contrib,
        sg, ng, tsg, trg, thg])
    for a in (sg, ng, tsg, trg, thg):
        a[~np.isfinite(a)] = 0
    t2 = time.time()
    cones, lo, ldh, ldw, nl, tl = cone_args
    out = dict(cam_eye=cam["eye"], cam_right=cam["right"], cam_up=cam["up"], width=W, height=H,
               tile_width=TILE_WIDTH, thr=F32(thr), ray_maps=ray_maps, cones=cones, level_offsets=lo,
               level_dims_h=ldh, level_dims_w=ldw, num_levels=nl, tile_level=tl, **scene,
               adjacency=adj, adjacency_offsets=adj_off, sort_keys=keys, tile_prims=prims,
               tile_offsets=offsets, adjacency_diff=adj_diff.view(np.uint16), depth_quantiles=dq, ray_gt=gt,
               color=color, log_t=log_t, normal_distance=nd, normal=normal, quantile_depths=qd,
               contrib=contrib, point_err=perr, early_stop=es, grad_color=g_color,
               grad_opacity=g_opac, grad_normal_distance=g_nd, grad_normal=g_normal,
               grad_quantile_depths=g_qd, grad_contrib=g_contrib, grad_log_t=g_logt,
               spheres_grad=sg, nsigmas_grad=ng, texel_sites_grad=tsg, texel_rgb_grad=trg,
               texel_height_grad=thg)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: N={N} {W}x{H} pairs={keys.shape[0]} levels={nl} fwd {t1 - t0:.1f}s bwd {t2 - t1:.1f}s")


def binning_case(name, scene, cam):
    R = rras.Rasterizer(Args(), "cpu", "float")
    wcam = warp_camera(cam)
    spheres = np.concatenate([scene["points"], scene["radii"][:, None]], -1).astype(F32)
    keys, prims, offsets, T = run_binning(R, wcam, spheres)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), cam_eye=cam["eye"], cam_right=cam["right"],
                        cam_up=cam["up"], width=cam["width"], height=cam["height"], tile_width=TILE_WIDTH,
                        spheres=spheres, sort_keys=keys, tile_prims=prims, tile_offsets=offsets)
    print(f"{name}: N={spheres.shape[0]} pairs={keys.shape[0]}")


class VisitLog:
    """Wraps all_spheres; records which cells each ray's walk reads."""

    def __init__(self, a):
        self.a = a
        self.shape = a.shape
        self.log = {}

    def __getitem__(self, i):
        self.log.setdefault(warp_shim._tls.tid, []).append(int(i))
        return self.a[i]


def trace_case(name, scene, cam, thr=1e-2):
    build_power_adjacency = load_power_adjacency_fn()
    pts = torch.from_numpy(scene["points"])
    radii = torch.from_numpy(scene["radii"])
    with torch.no_grad():
        adjacency, adjacency_offsets = build_power_adjacency(pts, radii, alpha_complex=False)
        num_adjs = adjacency_offsets.diff()
        # benchmark.py:297-302
        pm = 0.5 * (pts.norm(dim=-1) ** 2 - radii**2)
        self_points = pts.repeat_interleave(num_adjs, dim=0)
        adjacency_diff = pts[adjacency] - self_points
        pm_diff = pm[adjacency] - pm.repeat_interleave(num_adjs, dim=0)
        adjacency_diff = torch.cat([adjacency_diff, pm_diff[:, None]], dim=-1).to(torch.float16)
        # benchmark.py:320-324
        eye = torch.from_numpy(cam["eye"])
        dists = torch.linalg.norm(pts - eye[None, :], dim=-1)
        start = int(torch.argmin(dists**2 - radii**2))
    adj = adjacency.numpy().astype(np.int32)
    adj_off = adjacency_offsets.numpy().astype(np.int32)
    adiff = adjacency_diff.numpy()
    T = rtrace.RayTracer(Args(), "cpu", "float")
    wcam = warp_camera(cam)
    H, W = cam["height"], cam["width"]
    tiles_h = 1 + (H - 1) // 8
    tiles_w = 1 + (W - 1) // 8
    spheres = np.concatenate([scene["points"], scene["radii"][:, None]], -1).astype(F32)
    nsig = np.concatenate([scene["normals"], scene["density"][:, None]], -1).astype(F32)
    log = VisitLog(spheres)
    color = np.zeros((H, W, 3), F32)
    t0 = time.time()
    wp.launch(T.benchmark_kernel, dim=tiles_h * tiles_w * 64, inputs=[
        wcam, start, log, nsig, scene["texel_sites"], scene["texel_rgb"], scene["texel_height"], adj,
        adj_off, adiff, F32(thr), color])
    # visited cells per pixel (tile-major thread order -> pixel)
    maxlen = max(len(v) for v in log.log.values())
    visits = -np.ones((H, W, maxlen), np.int32)
    counts = np.zeros((H, W), np.int32)
    for t, cells in log.log.items():
        tile, l = t // 64, t % 64
        ti, tj = tile % tiles_h, tile // tiles_h
        pi, pj = ti * 8 + l % 8, tj * 8 + l // 8
        if pi >= H or pj >= W:
            continue
        visits[pi, pj, : len(cells)] = cells
        counts[pi, pj] = len(cells)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), cam_eye=cam["eye"], cam_right=cam["right"],
                        cam_up=cam["up"], width=W, height=H, thr=F32(thr), **scene, adjacency=adj,
                        adjacency_offsets=adj_off, adjacency_diff_pm=adiff.view(np.uint16),
                        start_idx=start, color=color, visits=visits, visit_count=counts)
    print(f"{name}: N={spheres.shape[0]} E={adj.shape[0]} start={start} maxlen={maxlen} {time.time() - t0:.1f}s")


def interpen_case(name, seed):
    """interpenetration_kernel (geometry.py:88-117) on overlapping spheres.
    The lists are the Čech lists (the reference's caller, scene.py:476-482)
    plus, on every fifth sphere, two far spheres that do not overlap (the
    d >= r_i + r_j branch), a self entry (d = 0), a pair of spheres with one
    centre (d = 0 between two spheres) and a sphere with an empty list."""
    sc = make_scene(seed, 200, -0.5, 0.5, 0.04, 0.16)
    pts, radii = sc["points"], sc["radii"]
    pts[1] = pts[0]
    pts[199] = np.array([3.0, 3.0, 3.0], F32)
    adj, off = cech_adjacency(pts, radii)
    rng = np.random.default_rng(seed + 1)
    lists = [adj[off[i]:off[i + 1]].tolist() for i in range(pts.shape[0])]
    for i in range(0, 195, 5):
        far = np.argsort(np.linalg.norm(pts[:195] - pts[i], axis=1))[-2:]
        lists[i] += far.tolist()
    lists[7].append(7)
    assert 1 in lists[0] and not lists[199]
    adj = np.array([j for l in lists for j in l], np.int32)
    off = np.concatenate([[0], np.cumsum([len(l) for l in lists])]).astype(np.int32)
    spheres = np.concatenate([pts, radii[:, None]], -1).astype(F32)
    areas = np.zeros(pts.shape[0], F32)
    wp.launch(rgeo.interpenetration_kernel, dim=pts.shape[0], inputs=[spheres, adj, off, areas])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), spheres=spheres, adjacency=adj, adjacency_offsets=off,
                        areas=areas)
    print(name, "pairs", adj.shape[0], "overlapping", int((areas > 0).sum()))


def steiner_case(name, seed, n=4000):
    """get_steiner_points (benchmark.py:137-180) with its helpers, executed
    from benchmark.py's own source on a small seeded scene (cKDTree on the
    host).  The random draws are recorded: per round the samples
    (points_mean + 0.5 * points_std * randn, evaluated as the function does)
    and the greedy selection's first pick."""
    from scipy.spatial import cKDTree

    src = open(os.path.join(REF, "benchmark.py")).read()
    tree = ast.parse(src)
    keep = {"inverse_softplus", "_greedy_min_overlap_fps", "get_steiner_points"}
    fns = [nd for nd in tree.body if isinstance(nd, ast.FunctionDef) and nd.name in keep]
    rec = dict(randn=[], randint=[])

    class TorchRec(types.ModuleType):
        def __getattr__(self, k):
            return getattr(torch, k)

    trec = TorchRec("torch_rec")

    def randn(*a, **k):
        v = torch.randn(*a, **k)
        rec["randn"].append(v.clone())
        return v

    def randint(*a, **k):
        v = torch.randint(*a, **k)
        rec["randint"].append(int(v.item()))
        return v

    trec.randn = randn
    trec.randint = randint
    ns = {"torch": trec, "cKDTree": cKDTree}
    exec(compile(ast.Module(body=fns, type_ignores=[]), "benchmark.py", "exec"), ns)
    sc = make_scene(seed, n, -1.0, 1.0, 0.01, 0.05)
    pts = torch.from_numpy(sc["points"])
    radii = torch.from_numpy(sc["radii"])
    torch.manual_seed(seed)
    sp, sr = ns["get_steiner_points"](pts, radii, None)
    mean = pts.mean(dim=0, keepdim=True)
    std = pts.std(dim=0, keepdim=True)
    samples = [(mean + 0.5 * std * r).numpy() for r in rec["randn"]]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), points=sc["points"], radii=sc["radii"],
                        samples=np.stack(samples), seeds=np.array(rec["randint"], np.int64),
                        steiner_points=sp.numpy(), steiner_radii=sr.numpy())
    print(name, "steiner points", sp.shape[0], "rounds", len(samples))


def sv_case(name, seed, n=3000, dof=6):
    """spherical_voronoi_fwd_kernel / _bwd_kernel (color_fn.py:54-184) from
    the reference's own source, float32 attributes; a camera whose cone
    leaves some points out."""
    import powerfoam.color_fn as rcol

    warp_shim.patch_module_builtins(rcol)

    class SvArgs:
        sv_dof = dof

    sv = rcol.SphericalVoronoi(SvArgs(), "cpu", "float")
    rng = np.random.default_rng(seed)
    pts = rng.uniform(-1, 1, (n, 3)).astype(F32)
    cam = look_at_camera((0.2, 0.1, 0.3), (0, 0, -1.0), 64, 48, 70.0)  # inside the cloud
    origin = cam["eye"].astype(F32)
    fwd = np.cross(cam["up"], cam["right"]).astype(F32)
    fwd = (fwd / np.linalg.norm(fwd)).astype(F32)
    cutoff = F32(np.cos(np.arctan(np.hypot(np.linalg.norm(cam["right"]), np.linalg.norm(cam["up"])))
                        + np.radians(10.0)))
    ax = rng.standard_normal((dof, n, 3))
    sites = (ax / np.linalg.norm(ax, axis=-1, keepdims=True)).astype(F32)
    values = (rng.standard_normal((dof, n, 3)) * 0.4).astype(F32)
    temps = rng.uniform(1.0, 12.0, (dof, n)).astype(F32)
    vout = np.zeros((n, 3), F32)
    wout = np.zeros(n, F32)
    wp.launch(sv.spherical_voronoi_fwd_kernel, dim=n,
              inputs=[pts, origin, fwd, cutoff, sites, values, temps, n, vout, wout])
    g = rng.standard_normal((n, 3)).astype(F32)
    gp = np.zeros((n, 3), F32)
    gs = np.zeros((dof, n, 3), F32)
    gv = np.zeros((dof, n, 3), F32)
    gt = np.zeros((dof, n), F32)
    wp.launch(sv.spherical_voronoi_bwd_kernel, dim=n,
              inputs=[pts, origin, fwd, cutoff, sites, values, temps, wout, vout, g, n, gp, gs, gv, gt])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), points=pts, origin=origin, forward=fwd,
                        cutoff=np.float32(cutoff), sites=sites, values=values, temps=temps, value=vout, wsum=wout,
                        grad_value=g, grad_sites=gs, grad_values=gv, grad_temps=gt, cam_eye=cam["eye"],
                        cam_right=cam["right"], cam_up=cam["up"], width=cam["width"], height=cam["height"])
    print(name, "outside the cone", int((wout == 0).sum()), "of", n)


def edge_scene(seed):
    """Primitives that exercise culling and the tile-range arithmetic: behind
    the camera, closer than 4r, straddling the image border, one covering many
    tiles, one with no neighbours."""
    base = make_scene(seed, 90, -0.7, 0.7, 0.05, 0.25)
    extra_pts = np.array([
        [0.0, 0.0, 4.0],      # behind the eye (eye at z=2.5 looking at -z)
        [0.0, 0.0, 2.3],      # closer than 4r
        [1.6, 0.2, 0.0],      # right of the image
        [-1.5, 1.1, 0.2],     # left/top outside
        [0.1, 1.2, -0.3],     # above the image
        [0.0, 0.0, 1.2],      # large, near
        [0.9, -0.9, 0.6],     # isolated corner
    ], F32)
    extra_r = np.array([0.2, 0.1, 0.3, 0.4, 0.35, 0.3, 0.02], F32)
    ex = make_scene(seed + 7, extra_pts.shape[0], -1, 1, 0.05, 0.1)
    ex["points"] = extra_pts
    ex["radii"] = extra_r
    ex["texel_sites"] = (extra_pts[:, None, :] + (ex["texel_sites"] - ex["texel_sites"].mean(1, keepdims=True))
                         ).astype(F32)
    return {k: np.concatenate([base[k], ex[k]], 0).astype(base[k].dtype) for k in base}


def main():
    which = sys.argv[1:] or ["raster_small", "raster_edge", "raster_dense", "bin_large", "interpen_small", "raster_generic", "steiner_small",
                           "sv_small", "trace_small"]
    if "raster_small" in which:
        sc = make_scene(1, 120, -0.6, 0.6, 0.05, 0.2)
        raster_case("raster_small", sc, look_at_camera((0.3, 0.4, 2.0), (0, 0, 0), 36, 28, 60.0), 1)
    if "raster_edge" in which:
        sc = edge_scene(2)
        raster_case("raster_edge", sc, look_at_camera((0.0, 0.0, 2.5), (0, 0, 0), 40, 24, 55.0), 2)
    if "raster_dense" in which:
        # opaque enough that whole tiles fall below the transmittance threshold
        # (early termination); 24x24 so no tile is ragged
        sc = make_scene(5, 700, -1.0, 1.0, 0.12, 0.3)
        sc["density"] = (sc["density"] * 300.0).astype(F32)
        raster_case("raster_dense", sc, look_at_camera((0.2, 0.3, 2.2), (0, 0, 0), 24, 24, 40.0), 5)
    if "bin_large" in which:
        sc = make_scene(3, 3000, -1.0, 1.0, 0.01, 0.08)
        binning_case("bin_large", sc, look_at_camera((1.0, 0.5, 2.6), (0, 0, 0), 96, 64, 50.0))
    if "interpen_small" in which:
        interpen_case("interpen_small", 6)
    if "raster_generic" in which:
        # per-pixel rays of a wide fisheye; 40x28 so the last tiles are ragged
        sc = make_scene(8, 220, -0.9, 0.9, 0.06, 0.22)
        cam = look_at_camera((0.3, -0.2, 2.1), (0, 0, 0), 40, 28, 60.0)
        generic_case("raster_generic", sc, cam, fisheye_ray_maps(cam, 80.0), 8)
    if "steiner_small" in which:
        steiner_case("steiner_small", 9)
    if "sv_small" in which:
        sv_case("sv_small", 10)
    if "trace_small" in which:
        sc = make_scene(4, 150, -0.6, 0.6, 0.08, 0.2)
        trace_case("trace_small", sc, look_at_camera((0.2, 0.3, 2.2), (0, 0, 0), 24, 20, 60.0))


if __name__ == "__main__":
    main()
