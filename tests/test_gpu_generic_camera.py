"""Generic cameras (is_pinhole=False): binning through the ray-cone hierarchy
and per-pixel rays in the forward and adjoint, on the GPU against the golden
case from the reference's own generic kernels and against the oracle.

Tolerances as for the pinhole path: sort keys, tile lists and early-stop
indices bit-exact; images max-abs 1e-5; gradients normwise relative 1e-4."""

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from powerfoam_b200.rasterize import Rasterizer
from tests.helpers import assert_close_rel, cech_np, max_abs, np_camera, np_scene, orc_cam, packed, to_t, torch_cam

pytestmark = pytest.mark.gpu

F32 = np.float32
NAMES = ["points", "radii", "density", "normals", "texel_sites", "texel_rgb", "texel_height"]


class Args:
    is_pinhole = False
    render_objective = "volume"
    num_texel_sites = 8
    disable_coop_prim_load = False
    disable_coop_adj_load = False


def fisheye(cam, fov_deg, scale=1.7, shift=0.02):
    """Equidistant fisheye directions of length `scale` from per-pixel
    origins spread along the image axes by up to `shift`."""
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


def run(sc, cam, ray_maps, adj, adj_off, dq, gt, tw=8):
    R = Rasterizer(Args(), "cuda", "float", tile_width=tw)
    tc = torch_cam(cam)
    if ray_maps is not None:
        tc.ray_maps = to_t(ray_maps)
    t = {k: to_t(sc[k]).requires_grad_(True) for k in NAMES}
    out = R.forward(tc, to_t(dq), t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    t["texel_rgb"], t["texel_height"], to_t(adj), to_t(adj_off), to_t(gt), True)
    return R, tc, t, out


def backprop(out, gc, go, gnd, gn, gq, gcon):
    color, opacity, nd, normal, qd, err, contrib, perr, vis = out
    loss = ((color * to_t(gc)).sum() + (opacity * to_t(go)).sum() + (nd * to_t(gnd)).sum()
            + (normal * to_t(gn)).sum() + (qd * to_t(gq)).sum() + (contrib * to_t(gcon)).sum())
    loss.backward()


def check_grads(t, sg, ng, tsg, trg, thg):
    assert_close_rel(t["points"].grad.cpu().numpy(), sg[:, :3], 1e-4, "points")
    assert_close_rel(t["radii"].grad.cpu().numpy(), sg[:, 3], 1e-4, "radii")
    assert_close_rel(t["normals"].grad.cpu().numpy(), ng[:, :3], 1e-4, "normals")
    assert_close_rel(t["density"].grad.cpu().numpy(), ng[:, 3], 1e-4, "density")
    assert_close_rel(t["texel_sites"].grad.cpu().numpy(), tsg, 1e-4, "sites")
    assert_close_rel(t["texel_rgb"].grad.cpu().numpy(), trg, 1e-4, "rgb")
    assert_close_rel(t["texel_height"].grad.cpu().numpy(), thg, 1e-4, "height")


def test_generic_golden_binning_forward_backward(golden):
    g = golden("raster_generic")
    sc = {k: g[k] for k in NAMES}
    cam = dict(eye=g["cam_eye"], right=g["cam_right"], up=g["cam_up"], width=int(g["width"]),
               height=int(g["height"]))
    R, tc, t, out = run(sc, cam, g["ray_maps"], g["adjacency"], g["adjacency_offsets"], g["depth_quantiles"],
                        g["ray_gt"])
    sph, _ = R.pack(to_t(sc["points"]), to_t(sc["radii"]))
    b = R.bin(tc, sph, return_keys=True)
    assert np.array_equal(b.sort_keys.cpu().numpy(), g["sort_keys"])
    assert np.array_equal(b.tile_prims.cpu().numpy(), g["tile_prims"])
    assert np.array_equal(b.tile_offsets.cpu().numpy(), g["tile_offsets"])
    color, opacity, nd, normal, qd, err, contrib, perr, vis = out
    assert max_abs(color.detach().cpu(), g["color"]) <= 1e-5
    assert max_abs(opacity.detach().cpu(), 1 - np.exp(g["log_t"])) <= 1e-5
    assert max_abs(nd.detach().cpu(), g["normal_distance"]) <= 1e-5
    assert max_abs(normal.detach().cpu(), g["normal"]) <= 1e-5
    assert max_abs(qd.detach().cpu(), g["quantile_depths"]) <= 1e-5
    assert_close_rel(contrib.detach().cpu().numpy(), g["contrib"], 1e-5, "contrib")
    assert_close_rel(perr.detach().cpu().numpy(), g["point_err"], 1e-5, "point_err")
    backprop(out, g["grad_color"], g["grad_opacity"], g["grad_normal_distance"], g["grad_normal"],
             g["grad_quantile_depths"], g["grad_contrib"])
    check_grads(t, g["spheres_grad"], g["nsigmas_grad"], g["texel_sites_grad"], g["texel_rgb_grad"],
                g["texel_height_grad"])


@pytest.mark.parametrize("tw", [8, 16, 32])
@pytest.mark.parametrize("seed", [0, 1])
def test_generic_matches_oracle(seed, tw):
    """Wide fisheye with per-pixel origins, ragged image, every tile width."""
    sc = np_scene(40 + seed, 900, -0.7, 0.7, 0.03, 0.15)
    cam = np_camera((0.3 * seed - 0.2, 0.4, 2.0), (0, 0, 0), 90, 61, 55.0)
    rm = fisheye(cam, 110.0 + 20 * seed)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    H, W = cam["height"], cam["width"]
    rng = np.random.default_rng(seed)
    dq = np.sort(rng.uniform(0.05, 0.95, (H, W, 2)).astype(F32), axis=-1)[..., ::-1].copy()
    gt = rng.uniform(0, 1, (H, W, 3)).astype(F32)
    R, tc, t, out = run(sc, cam, rm, adj, adj_off, dq, gt, tw)
    sph, nsig, rgbh = packed(sc)
    oc = orc_cam(cam)
    keys, prims, offs, _, _ = orc.bin_generic(oc, rm, sph, tw)
    sph_t, _ = R.pack(to_t(sc["points"]), to_t(sc["radii"]))
    b = R.bin(tc, sph_t, return_keys=True)
    assert np.array_equal(b.sort_keys.cpu().numpy(), keys)
    assert np.array_equal(b.tile_prims.cpu().numpy(), prims)
    assert np.array_equal(b.tile_offsets.cpu().numpy(), offs)
    ad = orc.prefetch_adjacency(sph, adj, adj_off)
    o = orc.raster_forward(oc, tw, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims, dq, gt, 1e-3,
                           True, ray_maps=rm)
    color, opacity, nd, normal, qd, err, contrib, perr, vis = out
    assert (o["color"].sum(-1) > 0).mean() > 0.1  # the fisheye sees the cloud
    for a, r in [(color, o["color"]), (nd, o["normal_distance"]), (normal, o["normal"]), (qd, o["quantile_depths"])]:
        assert max_abs(a.detach().cpu(), r) <= 1e-5
    assert max_abs(opacity.detach().cpu(), 1 - np.exp(o["log_t"])) <= 1e-5
    assert_close_rel(contrib.detach().cpu().numpy(), o["contrib"], 1e-5, "contrib")
    gc = rng.standard_normal((H, W, 3)).astype(F32)
    go = rng.standard_normal((H, W)).astype(F32)
    gn = rng.standard_normal((H, W, 3)).astype(F32)
    gnd = rng.standard_normal((H, W)).astype(F32)
    gq = rng.standard_normal((H, W, 2)).astype(F32)
    gcon = (rng.standard_normal(sc["points"].shape[0]) * 100).astype(F32)
    backprop(out, gc, go, gnd, gn, gq, gcon)
    g_logt = (-go * np.exp(o["log_t"])).astype(F32)
    gr = orc.raster_backward(oc, tw, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims,
                             o["early_stop"], o["log_t"], gc, g_logt, gnd, gn, gcon, dq, gq, ray_maps=rm)
    check_grads(t, gr["spheres"], gr["nsigmas"], gr["texel_sites"], gr["texel_rgb"], gr["texel_height"])


def test_generic_without_ray_maps_uses_pinhole_maps():
    """A generic rasterizer given a camera without ray maps builds the
    pinhole ones (TorchCamera.to_warp, camera.py:198-215) and bins them
    through the cones."""
    sc = np_scene(7, 500, -0.6, 0.6, 0.03, 0.15)
    cam = np_camera((0.2, 0.3, 2.1), (0, 0, 0), 64, 48, 55.0)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    H, W = cam["height"], cam["width"]
    rng = np.random.default_rng(3)
    dq = np.sort(rng.uniform(0.05, 0.95, (H, W, 1)).astype(F32), axis=-1)
    gt = rng.uniform(0, 1, (H, W, 3)).astype(F32)
    R, tc, t, out = run(sc, cam, None, adj, adj_off, dq, gt)
    rm = tc.build_pinhole_ray_maps().cpu().numpy()
    sph, nsig, rgbh = packed(sc)
    oc = orc_cam(cam)
    keys, prims, offs, _, _ = orc.bin_generic(oc, rm, sph, 8)
    o = orc.raster_forward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off,
                           orc.prefetch_adjacency(sph, adj, adj_off), offs, prims, dq, gt, 1e-3, True, ray_maps=rm)
    assert max_abs(out[0].detach().cpu(), o["color"]) <= 1e-5
    assert max_abs(out[1].detach().cpu(), 1 - np.exp(o["log_t"])) <= 1e-5


def test_generic_bin_arguments():
    from powerfoam_b200 import _lib

    cam = _lib.make_camera(torch.zeros(3), torch.tensor([1.0, 0, 0]), torch.tensor([0, 1.0, 0]), 32, 32)
    nbytes = _lib.ctypes.c_size_t(0)
    for tw in (3, 12, 0):
        with pytest.raises(_lib.PfError):
            _lib.call("pf_bin_generic_workspace_size", 10, 100, 32, 32, tw, _lib.ctypes.byref(nbytes))
    with pytest.raises(_lib.PfError):  # no ray maps
        _lib.call("pf_bin_generic", _lib.ctypes.byref(cam), None, 8, None, 0, None, 0, 0, None, None, None, None,
                  None, None, None, None)
