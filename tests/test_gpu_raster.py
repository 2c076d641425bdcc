"""Rasterizer parity: libpfoam (GPU, through the C ABI via the Python layer)
against the CPU oracle and the reference-source golden vectors.

Tolerances: tile keys, sort order, per-tile offsets, early-stop indices and
fp16 encodings bit-exact; images max-abs 1e-5; gradients normwise relative
1e-4 (max |g - g_ref| <= 1e-4 * max |g_ref|)."""

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from powerfoam_b200 import _lib
from powerfoam_b200.rasterize import Rasterizer, VisOptions
from tests.helpers import (assert_close_rel, cech_np, max_abs, np_camera, np_scene, orc_cam, packed, to_t,
                           torch_cam)

pytestmark = pytest.mark.gpu


class Args:
    is_pinhole = True
    render_objective = "volume"
    num_texel_sites = 8
    disable_coop_prim_load = False
    disable_coop_adj_load = False


def golden_inputs(g):
    sc = {k: g[k] for k in ["points", "radii", "density", "normals", "texel_sites", "texel_rgb", "texel_height"]}
    cam = dict(eye=g["cam_eye"], right=g["cam_right"], up=g["cam_up"], width=int(g["width"]), height=int(g["height"]))
    return sc, cam, g["adjacency"], g["adjacency_offsets"]


def run_forward(sc, cam, adj, adj_off, dq=None, gt=None, rpe=False, tw=8, thr=1e-3):
    R = Rasterizer(Args(), "cuda", "float", tile_width=tw)
    t = {k: to_t(v).requires_grad_(True) for k, v in sc.items()}
    out = R.forward(torch_cam(cam), None if dq is None else to_t(dq), t["points"], t["radii"], t["density"],
                    t["normals"], t["texel_sites"], t["texel_rgb"], t["texel_height"], to_t(adj), to_t(adj_off),
                    None if gt is None else to_t(gt), rpe)
    return R, t, out


def oracle_forward(sc, cam, adj, adj_off, dq=None, gt=None, rpe=False, tw=8, thr=1e-3):
    sph, nsig, rgbh = packed(sc)
    oc = orc_cam(cam)
    keys, prims, offs, _ = orc.bin(oc, sph, tw)
    ad = orc.prefetch_adjacency(sph, adj, adj_off)
    o = orc.raster_forward(oc, tw, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims, dq, gt, thr,
                           rpe)
    return o, (keys, prims, offs, ad)


@pytest.mark.parametrize("case", ["raster_small", "raster_edge", "raster_dense"])
def test_binning_matches_golden(golden, case):
    g = golden(case)
    sc, cam, adj, adj_off = golden_inputs(g)
    R = Rasterizer(Args(), "cuda")
    sph, _ = R.pack(to_t(sc["points"]), to_t(sc["radii"]))
    b = R.bin(torch_cam(cam), sph, return_keys=True)
    assert np.array_equal(b.sort_keys.cpu().numpy(), g["sort_keys"])
    assert np.array_equal(b.tile_prims.cpu().numpy(), g["tile_prims"])
    assert np.array_equal(b.tile_offsets.cpu().numpy(), g["tile_offsets"])
    vis = np.zeros(sc["points"].shape[0], bool)
    vis[g["tile_prims"]] = True
    assert np.array_equal(b.prim_visible.cpu().numpy(), vis)
    ad = R.prefetch_adjacency(sph, to_t(adj), to_t(adj_off))
    assert np.array_equal(ad.cpu().numpy().view(np.uint16), g["adjacency_diff"])


@pytest.mark.parametrize("tw", [8, 16, 32])
@pytest.mark.parametrize("seed", [0, 1])
def test_binning_matches_oracle(seed, tw):
    sc = np_scene(seed, 3000, -1.0, 1.0, 0.005, 0.08)
    cam = np_camera((0.7 * (seed + 1), 0.4, 2.4), (0, 0, 0), 150, 97, 55.0)
    sph, _, _ = packed(sc)
    keys, prims, offs, _ = orc.bin(orc_cam(cam), sph, tw)
    R = Rasterizer(Args(), "cuda", tile_width=tw)
    b = R.bin(torch_cam(cam), to_t(sph), return_keys=True)
    assert b.n_pairs == keys.shape[0]
    assert np.array_equal(b.sort_keys.cpu().numpy(), keys)
    assert np.array_equal(b.tile_prims.cpu().numpy(), prims)
    assert np.array_equal(b.tile_offsets.cpu().numpy(), offs)


def test_binning_overflow_retry_and_status():
    sc = np_scene(5, 2000, -1.0, 1.0, 0.02, 0.1)
    cam = np_camera((0.0, 0.3, 2.5), (0, 0, 0), 128, 96, 60.0)
    sph, _, _ = packed(sc)
    keys, prims, offs, _ = orc.bin(orc_cam(cam), sph, 8)
    R = Rasterizer(Args(), "cuda")
    c = torch_cam(cam)
    # too small a capacity: the C call flags PF_ERR_OVERFLOW and empties the lists
    import ctypes
    sp = to_t(sph)
    T = R.num_tiles(c)
    ws_n = ctypes.c_size_t(0)
    _lib.call("pf_bin_workspace_size", sph.shape[0], 16, T, ctypes.byref(ws_n))
    ws = torch.empty(ws_n.value, dtype=torch.uint8, device="cuda")
    offs_t = torch.full((T + 1,), 7, dtype=torch.int64, device="cuda")
    prims_t = torch.empty(16, dtype=torch.int32, device="cuda")
    npairs = torch.zeros(1, dtype=torch.int64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("pf_bin", ctypes.byref(c.to_pf()), 8, _lib.ptr(sp), sph.shape[0], _lib.ptr(ws), ws.numel(), 16,
              _lib.ptr(offs_t), _lib.ptr(prims_t), None, None, None, _lib.ptr(npairs), _lib.ptr(status),
              _lib.stream_ptr())
    assert int(status.item()) == _lib.PF_ERR_OVERFLOW
    assert int(npairs.item()) == keys.shape[0]
    assert int(offs_t.abs().sum().item()) == 0
    # the Python layer grows the capacity and re-bins
    b = R.binner(c.to_pf(), 8, sp, sph.shape[0], T, return_keys=True, capacity=16)
    assert np.array_equal(b.sort_keys.cpu().numpy(), keys)


def test_binning_empty_and_all_culled():
    R = Rasterizer(Args(), "cuda")
    cam = np_camera((0.0, 0.0, 3.0), (0, 0, 0), 40, 30, 60.0)
    c = torch_cam(cam)
    # every primitive behind the camera
    pts = np.array([[0, 0, 5.0], [0.1, 0, 4.0]], np.float32)
    sph = np.concatenate([pts, np.full((2, 1), 0.1, np.float32)], -1)
    b = R.bin(c, to_t(sph))
    assert b.n_pairs == 0
    assert int(b.tile_offsets.abs().sum().item()) == 0


@pytest.mark.parametrize("case", ["raster_small", "raster_edge", "raster_dense"])
def test_forward_backward_match_golden(golden, case):
    g = golden(case)
    sc, cam, adj, adj_off = golden_inputs(g)
    R, t, out = run_forward(sc, cam, adj, adj_off, g["depth_quantiles"], g["ray_gt"], True)
    color, opacity, nd, normal, qd, err, contrib, perr, vis = out
    assert max_abs(color.detach().cpu(), g["color"]) <= 1e-5
    assert max_abs(opacity.detach().cpu(), 1 - np.exp(g["log_t"])) <= 1e-5
    assert max_abs(nd.detach().cpu(), g["normal_distance"]) <= 1e-5
    assert max_abs(normal.detach().cpu(), g["normal"]) <= 1e-5
    assert max_abs(qd.detach().cpu(), g["quantile_depths"]) <= 1e-5
    assert_close_rel(contrib.detach().cpu().numpy(), g["contrib"], 1e-5, "contrib")
    assert_close_rel(perr.detach().cpu().numpy(), g["point_err"], 1e-5, "point_err")
    # adjoint through autograd with the golden upstream gradients
    loss = ((color * to_t(g["grad_color"])).sum() + (opacity * to_t(g["grad_opacity"])).sum()
            + (nd * to_t(g["grad_normal_distance"])).sum() + (normal * to_t(g["grad_normal"])).sum()
            + (qd * to_t(g["grad_quantile_depths"])).sum() + (contrib * to_t(g["grad_contrib"])).sum())
    loss.backward()
    sg, ng = g["spheres_grad"], g["nsigmas_grad"]
    assert_close_rel(t["points"].grad.cpu().numpy(), sg[:, :3], 1e-4, "points")
    assert_close_rel(t["radii"].grad.cpu().numpy(), sg[:, 3], 1e-4, "radii")
    assert_close_rel(t["normals"].grad.cpu().numpy(), ng[:, :3], 1e-4, "normals")
    assert_close_rel(t["density"].grad.cpu().numpy(), ng[:, 3], 1e-4, "density")
    assert_close_rel(t["texel_sites"].grad.cpu().numpy(), g["texel_sites_grad"], 1e-4, "sites")
    assert_close_rel(t["texel_rgb"].grad.cpu().numpy(), g["texel_rgb_grad"], 1e-4, "rgb")
    assert_close_rel(t["texel_height"].grad.cpu().numpy(), g["texel_height_grad"], 1e-4, "height")


@pytest.mark.parametrize("tw", [8, 16, 32])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_forward_backward_match_oracle(seed, tw):
    sc = np_scene(10 + seed, 600, -0.6, 0.6, 0.03, 0.15)
    cam = np_camera((0.3 * seed, 0.4, 2.2), (0, 0, 0), 70, 45, 55.0)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    H, W = cam["height"], cam["width"]
    rng = np.random.default_rng(seed)
    dq = np.sort(rng.uniform(0.05, 0.95, (H, W, 2)).astype(np.float32), axis=-1)[..., ::-1].copy()
    gt = rng.uniform(0, 1, (H, W, 3)).astype(np.float32)
    R, t, out = run_forward(sc, cam, adj, adj_off, dq, gt, True, tw=tw)
    o, (keys, prims, offs, ad) = oracle_forward(sc, cam, adj, adj_off, dq, gt, True, tw=tw)
    color, opacity, nd, normal, qd, err, contrib, perr, vis = out
    for a, b in [(color, o["color"]), (nd, o["normal_distance"]), (normal, o["normal"]), (qd, o["quantile_depths"])]:
        assert max_abs(a.detach().cpu(), b) <= 1e-5
    assert max_abs(opacity.detach().cpu(), 1 - np.exp(o["log_t"])) <= 1e-5
    assert_close_rel(contrib.detach().cpu().numpy(), o["contrib"], 1e-5, "contrib")
    g_c = rng.standard_normal((H, W, 3)).astype(np.float32)
    g_o = rng.standard_normal((H, W)).astype(np.float32)
    g_n = rng.standard_normal((H, W, 3)).astype(np.float32)
    g_nd = rng.standard_normal((H, W)).astype(np.float32)
    g_q = rng.standard_normal((H, W, 2)).astype(np.float32)
    g_con = (rng.standard_normal(sc["points"].shape[0]) * 100).astype(np.float32)
    loss = ((color * to_t(g_c)).sum() + (opacity * to_t(g_o)).sum() + (normal * to_t(g_n)).sum()
            + (nd * to_t(g_nd)).sum() + (qd * to_t(g_q)).sum() + (contrib * to_t(g_con)).sum())
    loss.backward()
    sph, nsig, rgbh = packed(sc)
    g_logt = (-g_o * np.exp(o["log_t"])).astype(np.float32)
    gr = orc.raster_backward(orc_cam(cam), tw, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims,
                             o["early_stop"], o["log_t"], g_c, g_logt, g_nd, g_n, g_con, dq, g_q)
    assert_close_rel(t["points"].grad.cpu().numpy(), gr["spheres"][:, :3], 1e-4, "points")
    assert_close_rel(t["radii"].grad.cpu().numpy(), gr["spheres"][:, 3], 1e-4, "radii")
    assert_close_rel(t["normals"].grad.cpu().numpy(), gr["nsigmas"][:, :3], 1e-4, "normals")
    assert_close_rel(t["density"].grad.cpu().numpy(), gr["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(t["texel_sites"].grad.cpu().numpy(), gr["texel_sites"], 1e-4, "sites")
    assert_close_rel(t["texel_rgb"].grad.cpu().numpy(), gr["texel_rgb"], 1e-4, "rgb")
    assert_close_rel(t["texel_height"].grad.cpu().numpy(), gr["texel_height"], 1e-4, "height")


@pytest.mark.parametrize("tw", [8, 16, 32])
def test_dense_early_termination_matches_oracle(tw):
    """Opaque scene: whole tiles fall below the transmittance threshold, so
    the barrier-free stop vote decides where every tile ends; early-stop
    indices must equal the oracle's (48x40 leaves ragged tiles at 16 and 32,
    which never stop)."""
    sc = np_scene(77, 700, -1.0, 1.0, 0.12, 0.3)
    sc["density"] = (sc["density"] * 300.0).astype(np.float32)
    cam = np_camera((0.2, 0.3, 2.2), (0, 0, 0), 48, 40, 40.0)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    R = Rasterizer(Args(), "cuda", "float", tile_width=tw)
    R.collect_stats = True
    t = {k: to_t(v).requires_grad_(True) for k, v in sc.items()}
    out = R.forward(torch_cam(cam), None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    t["texel_rgb"], t["texel_height"], to_t(adj), to_t(adj_off), None, False)
    o, (keys, prims, offs, ad) = oracle_forward(sc, cam, adj, adj_off, tw=tw)
    es = R.last_stats["early_stop"].cpu().numpy()
    assert np.array_equal(es, o["early_stop"])
    assert (o["early_stop"] < np.diff(offs)).sum() >= (2 if tw < 32 else 1)
    assert max_abs(out[0].detach().cpu(), o["color"]) <= 1e-5
    assert max_abs(out[1].detach().cpu(), 1 - np.exp(o["log_t"])) <= 1e-5
    loss = (out[0] * to_t(np.random.default_rng(3).standard_normal(o["color"].shape).astype(np.float32))).sum()
    loss.backward()
    sph, nsig, rgbh = packed(sc)
    H, W = cam["height"], cam["width"]
    g_c = np.random.default_rng(3).standard_normal(o["color"].shape).astype(np.float32)
    z = np.zeros((H, W), np.float32)
    gr = orc.raster_backward(orc_cam(cam), tw, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims,
                             o["early_stop"], o["log_t"], g_c, z, z, np.zeros((H, W, 3), np.float32),
                             np.zeros(sc["points"].shape[0], np.float32))
    assert_close_rel(t["points"].grad.cpu().numpy(), gr["spheres"][:, :3], 1e-4, "points")
    assert_close_rel(t["density"].grad.cpu().numpy(), gr["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(t["texel_rgb"].grad.cpu().numpy(), gr["texel_rgb"], 1e-4, "rgb")


def test_surface_objective_forward_and_errors():
    sc = np_scene(21, 300, -0.6, 0.6, 0.03, 0.15)
    cam = np_camera((0.0, 0.2, 2.2), (0, 0, 0), 48, 40, 55.0)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    gt = np.random.default_rng(1).uniform(0, 1, (40, 48, 3)).astype(np.float32)

    class A(Args):
        render_objective = "surface"

    R = Rasterizer(A(), "cuda")
    t = {k: to_t(v) for k, v in sc.items()}
    args = (torch_cam(cam), None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
            t["texel_rgb"], t["texel_height"], to_t(adj), to_t(adj_off))
    with pytest.raises(ValueError):
        R.forward(*args, None, False)
    out = R.forward(*args, to_t(gt), False)
    sph, nsig, rgbh = packed(sc)
    oc = orc_cam(cam)
    keys, prims, offs, _ = orc.bin(oc, sph, 8)
    ad = orc.prefetch_adjacency(sph, adj, adj_off)
    o = orc.raster_forward(oc, 8, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims, None, gt, 1e-3,
                           False, surface=True)
    assert max_abs(out[5].cpu(), o["err"]) <= 1e-5
    R2 = Rasterizer(Args(), "cuda")
    with pytest.raises(ValueError):
        R2.forward(*args, None, True)
    with pytest.raises(ValueError):
        Rasterizer(Args(), "cuda", attr_dtype="half").forward(*args, None, False)


@pytest.mark.parametrize("case", ["raster_small", "raster_edge", "raster_dense"])
def test_benchmark_and_visualize_match_golden(golden, case):
    g = golden(case)
    sc, cam, adj, adj_off = golden_inputs(g)
    R = Rasterizer(Args(), "cuda")
    t = {k: to_t(v) for k, v in sc.items()}
    c = R.benchmark(torch_cam(cam), t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    t["texel_rgb"], t["texel_height"], to_t(adj), to_t(adj_off),
                    to_t(g["adjacency_diff_pm"].view(np.float16)), float(g["bench_thr"]))
    assert max_abs(c.cpu(), g["bench_color"]) <= 1e-5
    v = R.visualize(torch_cam(cam), t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    t["texel_rgb"], t["texel_height"], to_t(adj), to_t(adj_off), VisOptions())
    for a, k in zip(v[:4], ["color", "depth", "normal", "alpha"]):
        assert max_abs(a.cpu(), g["vis_" + k]) <= 1e-5, k
    assert np.array_equal(v[4].cpu().numpy(), g["vis_intersections"])


def test_benchmark_half_attributes_match_oracle():
    sc = np_scene(31, 500, -0.6, 0.6, 0.03, 0.15)
    cam = np_camera((0.2, 0.1, 2.3), (0, 0, 0), 64, 48, 55.0)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    pm = orc.power_adjacency_diff(sc["points"], sc["radii"], adj, adj_off)
    R = Rasterizer(Args(), "cuda", attr_dtype="half")
    t = {k: to_t(v) for k, v in sc.items()}
    c = R.benchmark(torch_cam(cam), t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    t["texel_rgb"], t["texel_height"], to_t(adj), to_t(adj_off), to_t(pm.view(np.float16)), 1e-2)
    h = lambda a: a.astype(np.float16).astype(np.float32)
    sph, nsig, _ = packed(sc)
    oc = orc_cam(cam)
    keys, prims, offs, _ = orc.bin(oc, sph, 8)
    ref = orc.raster_benchmark(oc, 8, sph, h(nsig), h(sc["texel_sites"]), h(sc["texel_rgb"]), h(sc["texel_height"]),
                               adj_off, pm, offs, prims, 1e-2)
    assert max_abs(c.cpu(), ref) <= 1e-5


def test_nonfinite_gradients_are_zeroed():
    # a primitive whose texel sites sit exactly at its centre with zero radius
    # spread produces inf/nan terms; the reference zeroes them (rasterize.py:1954-1958)
    sc = np_scene(41, 200, -0.5, 0.5, 0.05, 0.2)
    cam = np_camera((0.0, 0.0, 2.2), (0, 0, 0), 32, 32, 55.0)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    R, t, out = run_forward(sc, cam, adj, adj_off)
    (out[0].sum() * 1e38 * 1e38).backward()
    for k in ["points", "radii", "density", "normals", "texel_sites", "texel_rgb", "texel_height"]:
        assert torch.isfinite(t[k].grad).all(), k


def _params(sc):
    return {k: to_t(v).requires_grad_(True) for k, v in sc.items()}


def _render_grads(R, cam, t, adj, adj_off, w):
    out = R.forward(cam, None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"], t["texel_rgb"],
                    t["texel_height"], adj, adj_off, None, False)
    loss = (out[0] * w[0]).sum() + (out[1] * w[1]).sum() + (out[3] * w[2]).sum()
    names = ["points", "radii", "density", "normals", "texel_sites", "texel_rgb", "texel_height"]
    grads = torch.autograd.grad(loss, [t[k] for k in names])
    return (out[0], out[1], out[2], out[3]), dict(zip(names, grads))


def test_sync_free_forward_backward_graph_replay():
    """host_sync=False: after the sizing call nothing is read back, so the
    whole forward + adjoint is captured in one CUDA graph; replays (also
    after the inputs are updated in place) give the eager images bit for bit
    and the eager gradients up to the order of float atomics."""
    sc = np_scene(61, 900, -0.6, 0.6, 0.03, 0.15)
    cam = torch_cam(np_camera((0.2, 0.3, 2.2), (0, 0, 0), 96, 72, 55.0))
    adj, adj_off = (to_t(a) for a in cech_np(sc["points"], sc["radii"]))
    rng = np.random.default_rng(9)
    w = [to_t(rng.standard_normal(s).astype(np.float32)) for s in ((72, 96, 3), (72, 96), (72, 96, 3))]
    R = Rasterizer(Args(), "cuda", host_sync=False)
    t = _params(sc)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(3):
            _render_grads(R, cam, t, adj, adj_off, w)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        imgs, grads = _render_grads(R, cam, t, adj, adj_off, w)
    for step in range(2):
        if step == 1:
            with torch.no_grad():
                t["points"].add_(to_t(rng.normal(0, 2e-3, sc["points"].shape).astype(np.float32)))
                t["density"].mul_(1.1)
        g.replay()
        torch.cuda.synchronize()
        ref_imgs, ref_grads = _render_grads(Rasterizer(Args(), "cuda"), cam, t, adj, adj_off, w)
        for a, b in zip(imgs, ref_imgs):
            assert torch.equal(a, b)
        for k in ref_grads:
            assert_close_rel(grads[k].cpu().numpy(), ref_grads[k].cpu().numpy(), 1e-5, k)
    assert R.check()


def test_sync_free_overflow_is_reported_by_check():
    sc = np_scene(62, 800, -0.8, 0.8, 0.05, 0.2)
    cam = torch_cam(np_camera((0.0, 0.2, 2.4), (0, 0, 0), 64, 48, 55.0))
    adj, adj_off = (to_t(a) for a in cech_np(sc["points"], sc["radii"]))
    R = Rasterizer(Args(), "cuda", host_sync=False)
    t = {k: to_t(v) for k, v in sc.items()}
    args = (cam, None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"], t["texel_rgb"],
            t["texel_height"], adj, adj_off, None, False)
    ref = R.forward(*args)[0]
    assert R.check()
    R.binner.capacity = 64  # far too small: the lists are emptied and the status word raised
    out = R.forward(*args)[0]
    assert float(out.abs().max()) == 0.0
    with pytest.raises(_lib.PfError) as e:
        R.check()
    assert e.value.code == _lib.PF_ERR_OVERFLOW
    R.binner.capacity = 0  # re-size on the next call
    assert torch.equal(R.forward(*args)[0], ref)
    assert R.check()


@pytest.mark.parametrize("field", ["radii", "points", "density", "normals"])
def test_nonfinite_attribute_raises(field):
    """A NaN / infinite primitive attribute is reported as PF_ERR_NONFINITE:
    at once with the default host read, by check() in the sync-free mode.
    Every loop of the kernels is bounded by integer list lengths, so the
    non-finite primitive only makes its own pixels non-finite."""
    sc = np_scene(63, 300, -0.6, 0.6, 0.03, 0.15)
    bad = {k: v.copy() for k, v in sc.items()}
    bad[field].reshape(bad[field].shape[0], -1)[17, 0] = np.nan if field != "density" else np.inf
    cam = torch_cam(np_camera((0.0, 0.2, 2.2), (0, 0, 0), 40, 30, 55.0))
    adj, adj_off = (to_t(a) for a in cech_np(sc["points"], sc["radii"]))

    def args(s):
        t = {k: to_t(v) for k, v in s.items()}
        return (cam, None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"], t["texel_rgb"],
                t["texel_height"], adj, adj_off, None, False)

    with pytest.raises(_lib.PfError) as e:
        Rasterizer(Args(), "cuda").forward(*args(bad))
    assert e.value.code == _lib.PF_ERR_NONFINITE
    R = Rasterizer(Args(), "cuda", host_sync=False)
    R.forward(*args(sc))  # the sizing call
    assert R.check()
    R.forward(*args(bad))
    with pytest.raises(_lib.PfError) as e:
        R.check()
    assert e.value.code == _lib.PF_ERR_NONFINITE
    R.forward(*args(sc))
    assert R.check()


def test_gradients_into_a_flat_buffer():
    """With Rasterizer.grad_buffer the adjoint writes every gradient into one
    flat buffer (the multi-GPU exchange sums it in place): autograd's .grad
    tensors are views of it and equal the gradients of the default path."""
    from powerfoam_b200.multiview import GradBuffer, raster_fields

    sc = np_scene(64, 500, -0.6, 0.6, 0.03, 0.15)
    cam = torch_cam(np_camera((0.1, 0.3, 2.2), (0, 0, 0), 56, 40, 55.0))
    adj, adj_off = (to_t(a) for a in cech_np(sc["points"], sc["radii"]))
    w = to_t(np.random.default_rng(2).standard_normal((40, 56, 3)).astype(np.float32))
    grads = []
    for use_buffer in (False, True):
        R = Rasterizer(Args(), "cuda")
        if use_buffer:
            R.grad_buffer = GradBuffer(raster_fields(500, 8), "cuda", world=3)
        t = _params(sc)
        out = R.forward(cam, None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                        t["texel_rgb"], t["texel_height"], adj, adj_off, None, False)
        (out[0] * w).sum().backward()
        grads.append({k: v.grad for k, v in t.items()})
        if use_buffer:
            lo = R.grad_buffer.flat.data_ptr()
            hi = lo + R.grad_buffer.flat.numel() * 4
            for k, g in grads[-1].items():
                assert lo <= g.data_ptr() < hi, k
    for k in grads[0]:
        assert_close_rel(grads[1][k].cpu().numpy(), grads[0][k].cpu().numpy(), 1e-5, k)


@pytest.mark.parametrize("tw", [8, 16])
def test_segment_records_give_the_clipping_adjoint(tw):
    """The adjoint that reads the forward's segment records (sphere interval
    after the power faces, bounding ids, texture-plane results) against the
    one that clips and evaluates the plane again: the same images, and
    gradients equal up to the order of the float atomics; so do budgets that
    hold the intervals only or nothing, and a record buffer too small for
    most primitives (those are clipped again in the adjoint)."""
    import powerfoam_b200.rasterize as rz

    sc = np_scene(63, 900, -0.6, 0.6, 0.03, 0.15)
    cam = torch_cam(np_camera((0.25, 0.2, 2.2), (0, 0, 0), 83, 61, 55.0))  # ragged tiles
    adj, adj_off = (to_t(a) for a in cech_np(sc["points"], sc["radii"]))
    rng = np.random.default_rng(10)
    w = [to_t(rng.standard_normal(s).astype(np.float32)) for s in ((61, 83, 3), (61, 83), (61, 83, 3))]
    probe = Rasterizer(Args(), "cuda", tile_width=tw)
    probe.collect_stats = True
    _render_grads(probe, cam, _params(sc), adj, adj_off, w)
    cap = probe.rec_capacity
    n_rec = int(probe.rec_count.item())
    assert 0 < n_rec <= cap
    res = []
    for rec, budget, capacity in ((True, rz.SEGMENT_BYTES, 0), (False, rz.SEGMENT_BYTES, 0), (True, 32 * cap, 0),
                                  (True, 8 * cap, 0), (True, rz.SEGMENT_BYTES, n_rec // 8)):
        R = Rasterizer(Args(), "cuda", tile_width=tw)
        R.record_segments = rec
        R.rec_capacity = capacity
        old, rz.SEGMENT_BYTES = rz.SEGMENT_BYTES, budget
        try:
            res.append(_render_grads(R, cam, _params(sc), adj, adj_off, w))
        finally:
            rz.SEGMENT_BYTES = old
    (imgs, grads) = res[0]
    for other_imgs, other_grads in res[1:]:
        for a, b in zip(imgs, other_imgs):
            assert torch.equal(a, b)
        for k in grads:
            d = (grads[k] - other_grads[k]).norm() / grads[k].norm().clamp_min(1e-30)
            assert d.item() <= 1e-5, k
