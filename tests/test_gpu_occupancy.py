"""Occupancy seeding (pf_occupancy_build / pf_occupancy_entry), the
conservative proposal: the voxel bits against the same float32 arithmetic on
the host (bit-exact), the entry distance never past the first sphere of
significant density a ray meets (brute force over every primitive), and the
seeded walk against the plain walk."""

import math

import numpy as np
import pytest
import torch

from oracle.power_hull import build_power_adjacency
from powerfoam_b200.adjacency import power_adjacency_diff, start_cell
from powerfoam_b200.proposal import OccupancySeeder, VoxelLocator
from powerfoam_b200.raytrace import RayTracer
from tests.helpers import np_camera, np_scene, to_t, torch_cam

pytestmark = pytest.mark.gpu

F32 = np.float32


class TArgs:
    num_texel_sites = 8


def _scene(seed=70, n=1500):
    sc = np_scene(seed, n, -0.6, 0.6, 0.02, 0.08)
    rng = np.random.default_rng(seed + 1)
    sc["density"][rng.uniform(size=n) < 0.5] = 0.0  # half the primitives composite nothing
    return sc


def _host_bits(sc, lo, hi, res, sigma_min):
    """pf_occupancy_build's rule in float32 on the host."""
    lo = np.asarray(lo, F32)
    hi = np.asarray(hi, F32)
    ext = F32(max(float(np.max(hi - lo)), 1e-6))
    h = F32(ext / F32(res))
    inv_h = F32(F32(1.0) / h)
    bits = np.zeros(res ** 3, bool)
    for c, r, s in zip(sc["points"], sc["radii"], sc["density"]):
        if s < F32(sigma_min):
            continue
        a = np.floor(((c - r).astype(F32) - lo).astype(F32) * inv_h).astype(F32) - F32(1)
        b = np.floor(((c + r).astype(F32) - lo).astype(F32) * inv_h).astype(F32) + F32(1)
        a = np.clip(a, 0, res - 1).astype(int)
        b = np.clip(b, 0, res - 1).astype(int)
        z, y, x = np.meshgrid(np.arange(a[2], b[2] + 1), np.arange(a[1], b[1] + 1), np.arange(a[0], b[0] + 1),
                              indexing="ij")
        bits[((z * res + y) * res + x).ravel()] = True
    return bits


def _seeder(sc, res):
    t = {k: to_t(v) for k, v in sc.items()}
    adj, off = build_power_adjacency(t["points"], t["radii"])
    loc = VoxelLocator(t["points"], t["radii"], adj, off, res=64)
    return t, adj, off, loc, OccupancySeeder(t["points"], t["radii"], t["density"], loc, res=res)


@pytest.mark.parametrize("res", [32, 100])
def test_occupancy_bits_match_host(res):
    sc = _scene()
    _, _, _, _, occ = _seeder(sc, res)
    torch.cuda.synchronize()
    occ.check()
    words = occ.bits.cpu().numpy().view(np.uint32)
    got = ((words[:, None] >> np.arange(32, dtype=np.uint32)) & 1).astype(bool).ravel()[:res ** 3]
    want = _host_bits(sc, list(occ.box[0]), list(occ.box[1]), res, 1e-3)
    assert np.array_equal(got, want)
    assert 0 < got.sum() < res ** 3


def _first_hits(sc, cam, sigma_min=1e-3):
    """Per pixel ray: the smallest t >= 0 inside a sphere of density >=
    sigma_min (brute force, float64), inf where the ray meets none."""
    H, W = cam["height"], cam["width"]
    eye = cam["eye"].astype(np.float64)
    right, up = cam["right"].astype(np.float64), cam["up"].astype(np.float64)
    fwd = np.cross(up, right)
    fwd /= np.linalg.norm(fwd)
    j, i = np.meshgrid(np.arange(W), np.arange(H))
    x = 2.0 * j / (W - 1) - 1.0
    y = 1.0 - 2.0 * i / (H - 1)
    d = x[..., None] * right + y[..., None] * up + fwd
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    d = d.reshape(-1, 3)
    keep = sc["density"] >= sigma_min
    c, r = sc["points"][keep].astype(np.float64), sc["radii"][keep].astype(np.float64)
    oc = eye[None, :] - c
    b = d @ oc.T
    disc = b * b - (np.sum(oc * oc, -1) - r * r)[None, :]
    s = np.sqrt(np.maximum(disc, 0.0))
    t_in, t_out = -b - s, -b + s
    hit = (disc >= 0) & (t_out >= 0)
    t = np.where(hit, np.maximum(t_in, 0.0), np.inf)
    return t.min(-1).reshape(H, W)


def test_occupancy_entry_never_passes_a_significant_sphere():
    sc = _scene(71, 1200)
    _, _, _, _, occ = _seeder(sc, 64)
    cam = np_camera((0.5, 0.8, 2.3), (0, 0, 0), 48, 40, 55.0)
    t, c = occ.entry(torch_cam(cam))
    torch.cuda.synchronize()
    t, c = t.cpu().numpy().astype(np.float64), c.cpu().numpy()
    first = _first_hits(sc, cam)
    seeded = c > 0.5
    assert seeded.any() and (~seeded).any()
    assert np.all(t[seeded] <= first[seeded] * (1 + 1e-6))
    # and it skips most of the way there (a ray also crosses the marked box corners of spheres it
    # misses, so the entry can come well before the first sphere it hits)
    near = seeded & np.isfinite(first)
    assert near.sum() > 100 and np.median(t[near] / first[near]) >= 0.8


def test_occupancy_seeded_walk_matches_plain():
    """Opaque shells in empty space: the walk seeded at the occupancy entry
    visits fewer cells and gives the plain walk's image (>= 80 dB: the seeded
    walk starts in the exactly located cell, the plain walk crosses the
    float16 faces)."""
    from powerfoam_b200 import synthetic

    n = 60000
    scale = (6291456 / n) ** (1 / 3)
    sc = synthetic.make_scene(n, seed=4, mixture=16, sigma=0.1, r_range=(0.001 * scale, 0.01 * scale),
                              shells=(0.12, 0.02, 30.0))
    rgb = synthetic.texel_rgb(sc, synthetic.front_camera(64, 64, 50.0))
    adj, off = build_power_adjacency(sc["points"], sc["radii"])
    pm = power_adjacency_diff(sc["points"], sc["radii"], adj, off)
    args = (sc["points"], sc["radii"], sc["density"], sc["normals"], sc["texel_sites"], rgb, sc["texel_height"], adj,
            off, pm)
    loc = VoxelLocator(sc["points"], sc["radii"], adj, off, res=128)
    occ = OccupancySeeder(sc["points"], sc["radii"], sc["density"], loc, res=128)
    tr = RayTracer(TArgs(), "cuda")
    for k in range(2):
        ev = synthetic.orbit_camera(900 + k, 256, 192, 50.0)
        st = start_cell(sc["points"], sc["radii"], ev.eye)
        plain = tr.trace(ev, st, *args)
        n_seeded = torch.zeros(1, dtype=torch.int32, device="cuda")
        seeded = tr.trace(ev, occ.start_cells(ev, st, n_seeded), *args)
        torch.cuda.synchronize()
        occ.check()
        mse = float(((seeded.color.double() - plain.color.double()) ** 2).mean())
        psnr = 10 * math.log10(1.0 / max(mse, 1e-20))
        v_plain, v_seed = int(plain.visit_count.sum()), int(seeded.visit_count.sum())
        print(f"occupancy seeding: {int(n_seeded.item())}/{256 * 192} rays seeded, {psnr:.1f} dB, "
              f"cells {v_seed}/{v_plain}")
        assert int(n_seeded.item()) >= 0.3 * 256 * 192
        assert psnr >= 80.0 and v_seed < 0.8 * v_plain
