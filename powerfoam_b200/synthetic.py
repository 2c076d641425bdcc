"""Seeded synthetic scenes and cameras for the rendering path.

The reference's benchmarks run on Mip-NeRF 360 / DL3DV captures; here seeded
synthetic scenes with the stated primitive counts, position distributions and
radius ranges stand in for them.  Attributes follow the reference's
initialiser (powerfoam/scene.py:124-179, 242-337):

* centres: uniform in [-1,1]^3, or a mixture -- K means uniform in [-1,1]^3,
  isotropic sigma, 90 % of the points from a uniformly chosen component,
  10 % uniform in [-1,1]^3;
* radius r log-uniform in [r_min, r_max] (power weight w = r^2);
* density softplus(N(0,1)) * 10;
* normals / tangents / bitangents from a random unit quaternion;
* texel sites c + r (s0 t + s1 b), s ~ 0.1 N(0,1); texel height 0;
* colour: degree-3 real SH, 16 x 3 coefficients ~ N(0, 0.2^2), evaluated per
  view at normalize(c - eye) + 0.5, clamped at 0 (pf_sh_texel_rgb).

Everything is drawn on the CPU from torch.Generator(seed) and then moved, so a
scene is identical on every machine.  Primitives are Morton-ordered as the
reference does before rendering (scene.py:197-233).
"""

import math

import numpy as np
import torch

from . import _lib
from .camera import TorchCamera, look_at


def quat_frames(q):
    """Normals, tangents, bitangents of unit quaternions (scene.py:242-285)."""
    q = q / q.norm(dim=-1, keepdim=True)
    w, x, y, z = q.unbind(-1)
    n = torch.stack([1 - 2 * (y**2 + z**2), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1)
    t = torch.stack([2 * (x * y + z * w), 1 - 2 * (x**2 + z**2), 2 * (y * z - x * w)], -1)
    b = torch.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x**2 + y**2)], -1)
    f = lambda v: v / v.norm(dim=-1, keepdim=True)
    return f(n), f(t), f(b)


def morton_order_cpu(points):
    """geometry.py:7-85 on the host (numpy), stable on equal codes."""
    p = points.numpy().astype(np.float32)
    lo = p.min(0)
    dims = np.maximum(p.max(0) - lo, np.float32(1e-6)).astype(np.float32)
    res = np.float32(2097152.0)
    q = np.clip(((p - lo) / dims).astype(np.float32) * res, 0, res - 1).astype(np.uint64)

    def expand(v):
        v = v & np.uint64(0x1FFFFF)
        for s, m in ((32, 0x001F00000000FFFF), (16, 0x001F0000FF0000FF), (8, 0x100F00F00F00F00F),
                     (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249)):
            v = (v | (v << np.uint64(s))) & np.uint64(m)
        return v

    code = expand(q[:, 0]) * np.uint64(4) + expand(q[:, 1]) * np.uint64(2) + expand(q[:, 2])
    return torch.from_numpy(np.argsort(code, kind="stable").astype(np.int64))


def make_scene(n, seed=0, mixture=0, sigma=0.15, r_range=(0.01, 0.05), n_sites=8, sh_std=0.2, device="cuda",
               morton=True, shells=None):
    """``shells`` = (radius, thickness, density scale): the mixture's
    components are spherical shells of that radius and thickness around the
    means instead of Gaussians, their density scaled, and the 10 % background
    points get density 0 (opaque shells in empty space)."""
    g = torch.Generator().manual_seed(seed)
    background = torch.zeros(n, dtype=torch.bool)
    if mixture:
        means = torch.rand(mixture, 3, generator=g) * 2 - 1
        n_uni = n // 10
        comp = torch.randint(0, mixture, (n - n_uni,), generator=g)
        if shells is None:
            pts_m = means[comp] + torch.randn(n - n_uni, 3, generator=g) * sigma
        else:
            u = torch.randn(n - n_uni, 3, generator=g)
            u = u / u.norm(dim=-1, keepdim=True)
            rad = shells[0] + shells[1] * (torch.rand(n - n_uni, 1, generator=g) - 0.5)
            pts_m = means[comp] + u * rad
        pts_u = torch.rand(n_uni, 3, generator=g) * 2 - 1
        points = torch.cat([pts_m, pts_u], 0)
        background[n - n_uni:] = True
        perm0 = torch.randperm(n, generator=g)
        points, background = points[perm0], background[perm0]
    else:
        points = torch.rand(n, 3, generator=g) * 2 - 1
    lr = torch.rand(n, generator=g) * (math.log(r_range[1]) - math.log(r_range[0])) + math.log(r_range[0])
    radii = torch.exp(lr)
    density = torch.nn.functional.softplus(torch.randn(n, generator=g)) * 10
    if shells is not None:
        density = torch.where(background, torch.zeros_like(density), density * shells[2])
    q = torch.randn(n, 4, generator=g)
    normals, tangents, bitangents = quat_frames(q)
    s2 = torch.randn(n, n_sites, 2, generator=g) * 0.1
    sh = torch.randn(n, 16, 3, generator=g) * sh_std
    if morton:
        perm = morton_order_cpu(points)
        points, radii, density, normals, tangents, bitangents, s2, sh = (
            t[perm] for t in (points, radii, density, normals, tangents, bitangents, s2, sh))
    off = s2 * radii[:, None, None]
    off = off[..., 0:1] * tangents[:, None, :] + off[..., 1:2] * bitangents[:, None, :]
    texel_sites = points[:, None, :] + off
    texel_height = torch.zeros(n, n_sites)
    out = dict(points=points, radii=radii, density=density, normals=normals, texel_sites=texel_sites,
               texel_height=texel_height, sh=sh)
    return {k: v.float().contiguous().to(device) for k, v in out.items()}


def orbit_camera(seed, width, height, vfov_deg, distance=3.0, device="cuda", azimuth=None, elevation=None):
    """Camera on a sphere of radius ``distance`` looking at the origin; angles
    seeded unless given (degrees)."""
    g = torch.Generator().manual_seed(seed)
    az = float(torch.rand(1, generator=g)) * 360.0 if azimuth is None else azimuth
    el = (float(torch.rand(1, generator=g)) * 120.0 - 60.0) if elevation is None else elevation
    a, e = math.radians(az), math.radians(el)
    eye = (distance * math.cos(e) * math.sin(a), distance * math.sin(e), distance * math.cos(e) * math.cos(a))
    return look_at(eye, (0.0, 0.0, 0.0), width, height, vfov_deg, device=device)


def fisheye_ray_maps(cam, fov_deg):
    """(H, W, 6) ray maps of an equidistant fisheye with the camera's eye,
    axes and image size: a generic camera (per-pixel rays) for the
    is_pinhole=False path.  The diagonal field of view is fov_deg."""
    H, W = cam.height, cam.width
    dev = cam.eye.device
    r_hat = cam.right / torch.linalg.norm(cam.right)
    u_hat = cam.up / torch.linalg.norm(cam.up)
    f = torch.cross(cam.up, cam.right, dim=-1)
    f = f / torch.linalg.norm(f)
    i = torch.arange(H, dtype=torch.float32, device=dev)
    j = torch.arange(W, dtype=torch.float32, device=dev)
    ii, jj = torch.meshgrid(i, j, indexing="ij")
    x = (2.0 * jj / (W - 1) - 1.0) * (W / math.hypot(W, H))
    y = (1.0 - 2.0 * ii / (H - 1)) * (H / math.hypot(W, H))
    rad = torch.sqrt(x * x + y * y)
    th = rad * math.radians(fov_deg) / 2.0
    s = torch.where(rad > 0, torch.sin(th) / rad.clamp_min(1e-12), torch.zeros_like(rad))
    d = torch.cos(th)[..., None] * f + (s * x)[..., None] * r_hat + (s * y)[..., None] * u_hat
    o = cam.eye.expand(H, W, 3)
    return torch.cat([o, d], dim=-1).float().contiguous()


BATCH_RESOLUTIONS = ((320, 240), (640, 480), (1280, 720), (1920, 1080))


def batch_cameras(n_views, seed, vfov_deg=50.0, distance=3.0, device="cuda", resolutions=BATCH_RESOLUTIONS):
    """n_views orbit cameras, each resolution drawn uniformly from
    `resolutions` (seeded)."""
    g = torch.Generator().manual_seed(seed)
    idx = torch.randint(0, len(resolutions), (n_views,), generator=g).tolist()
    return [orbit_camera(seed * 1000 + v, *resolutions[i], vfov_deg, distance, device=device)
            for v, i in enumerate(idx)]


def front_camera(width, height, vfov_deg, distance=3.0, device="cuda"):
    return look_at((0.0, 0.0, distance), (0.0, 0.0, 0.0), width, height, vfov_deg, device=device)


def texel_rgb(scene, camera, n_sites=8):
    """Per-view texel colours from the SH coefficients (GPU)."""
    pts = scene["points"]
    n = pts.shape[0]
    out = torch.empty((n, n_sites, 3), dtype=torch.float32, device=pts.device)
    e = camera.to_pf().eye  # the camera's cached C struct: no device read per call
    _lib.call("pf_sh_texel_rgb", _lib.ptr(pts), _lib.ptr(scene["sh"]), n, n_sites, e, _lib.ptr(out),
              _lib.stream_ptr())
    return out


# Configurations of the measured workloads (sizes as stated; data synthetic).
CONFIGS = {
    "raster16k": dict(n=16384, seed=0, mixture=0, r_range=(0.01, 0.05), width=256, height=256, vfov=60.0),
    "raster1m": dict(n=1048576, seed=1, mixture=32, sigma=0.15, r_range=(0.002, 0.02), width=1920, height=1080,
                     vfov=50.0),
    "raster256k": dict(n=262144, seed=1, mixture=32, sigma=0.15, r_range=(0.004, 0.04), width=960, height=540,
                       vfov=50.0),
    "trace1m": dict(n=1048576, seed=1, mixture=32, sigma=0.15, r_range=(0.002, 0.02), width=1280, height=720,
                    vfov=50.0),
    "batch3m": dict(n=3145728, seed=3, mixture=64, sigma=0.15, r_range=(0.002, 0.02), vfov=50.0, views=32),
    "batch256k": dict(n=262144, seed=3, mixture=64, sigma=0.15, r_range=(0.004, 0.04), vfov=50.0, views=8),
    "trace6m": dict(n=6291456, seed=4, mixture=64, sigma=0.1, r_range=(0.001, 0.01), width=2048, height=1536,
                    vfov=50.0),
}


def raster_workload(name="raster1m", device="cuda", view=0):
    """The rasterizer workload ``name`` of CONFIGS: scene, the orbit camera
    of view ``view`` (seed 100 + view), its Čech adjacency (built on the
    device) and the seeded uniform target image (host, seed 200 + view).
    Returns (cfg, scene, camera, adjacency, adjacency_offsets, target)."""
    from .adjacency import CechBuilder

    cfg = CONFIGS[name]
    scene = make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg.get("sigma", 0.15),
                       r_range=cfg["r_range"], device=device)
    cam = orbit_camera(100 + view, cfg["width"], cfg["height"], cfg["vfov"], device=device)
    adj, adj_off = CechBuilder(device)(scene["points"], scene["radii"])
    g = torch.Generator().manual_seed(200 + view)
    target = torch.rand((cfg["height"], cfg["width"], 3), generator=g)
    return cfg, scene, cam, adj, adj_off, target


def trace_workload(name="trace1m", device="cuda"):
    """The tracer workload: scene, its power-diagram adjacency (built on the
    device), the (c_j - c_i, pm_j - pm_i) neighbour encoding, the orbit
    camera (seed 2) and the camera's start cell (benchmark.py:320-324).
    Returns (cfg, scene, camera, adjacency, adjacency_offsets, adj_diff_pm,
    start)."""
    from .adjacency import power_adjacency, power_adjacency_diff, start_cell

    cfg = CONFIGS[name]
    sc = make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"], r_range=cfg["r_range"],
                    device=device)
    adj, off = power_adjacency(sc["points"], sc["radii"])
    pm = power_adjacency_diff(sc["points"], sc["radii"], adj, off)
    cam = orbit_camera(2, cfg["width"], cfg["height"], cfg["vfov"], device=device)
    st = start_cell(sc["points"], sc["radii"], cam.eye)
    return cfg, sc, cam, adj, off, pm, st
