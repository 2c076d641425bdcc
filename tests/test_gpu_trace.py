"""Cell-walk tracer parity: visited-cell sequences bit-exact against the
reference-source golden vectors and the oracle; colour max-abs 1e-5; step cap
reported as a status, never a hang."""

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from powerfoam_b200 import _lib
from oracle.power_hull import build_power_adjacency
from powerfoam_b200.adjacency import power_adjacency_diff, start_cell
from powerfoam_b200.raytrace import RayTracer
from tests.helpers import max_abs, np_camera, np_scene, orc_cam, packed, to_t, torch_cam

pytestmark = pytest.mark.gpu


class Args:
    num_texel_sites = 8


def test_trace_matches_golden(golden):
    g = golden("trace_small")
    cam = dict(eye=g["cam_eye"], right=g["cam_right"], up=g["cam_up"], width=int(g["width"]), height=int(g["height"]))
    t = {k: to_t(g[k]) for k in ["points", "radii", "density", "normals", "texel_sites", "texel_rgb", "texel_height"]}
    s = start_cell(t["points"], t["radii"], torch.from_numpy(g["cam_eye"]))
    assert s == int(g["start_idx"])
    pm = power_adjacency_diff(t["points"], t["radii"], to_t(g["adjacency"]), to_t(g["adjacency_offsets"]))
    assert np.array_equal(pm.cpu().numpy().view(np.uint16), g["adjacency_diff_pm"])
    R = RayTracer(Args(), "cuda")
    r = R.trace(torch_cam(cam), s, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                t["texel_rgb"], t["texel_height"], to_t(g["adjacency"]), to_t(g["adjacency_offsets"]), pm,
                float(g["thr"]), visit_cap=g["visits"].shape[-1])
    assert np.array_equal(r.visit_count.cpu().numpy(), g["visit_count"])
    assert np.array_equal(r.visits.cpu().numpy(), g["visits"])
    assert max_abs(r.color.cpu(), g["color"]) <= 1e-5
    c = R.benchmark(torch_cam(cam), s, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    t["texel_rgb"], t["texel_height"], to_t(g["adjacency"]), to_t(g["adjacency_offsets"]), pm,
                    float(g["thr"]))
    assert max_abs(c.cpu(), g["color"]) <= 1e-5


@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("seed", [0, 1])
def test_trace_matches_oracle(seed, half):
    sc = np_scene(50 + seed, 400, -0.6, 0.6, 0.05, 0.15)
    cam = np_camera((0.3, 0.2 * seed, 2.2), (0, 0, 0), 40, 30, 55.0)
    tp = {k: to_t(v) for k, v in sc.items()}
    adj, off = build_power_adjacency(tp["points"], tp["radii"])
    adj_np, off_np = adj.cpu().numpy(), off.cpu().numpy()
    pm = power_adjacency_diff(tp["points"], tp["radii"], adj, off)
    s = start_cell(tp["points"], tp["radii"], torch.from_numpy(cam["eye"]))
    assert s == orc.start_cell(sc["points"], sc["radii"], cam["eye"])
    R = RayTracer(Args(), "cuda", "half" if half else "float")
    r = R.trace(torch_cam(cam), s, tp["points"], tp["radii"], tp["density"], tp["normals"], tp["texel_sites"],
                tp["texel_rgb"], tp["texel_height"], adj, off, pm, 1e-3, visit_cap=96)
    sph, nsig, _ = packed(sc)
    h = (lambda a: a.astype(np.float16).astype(np.float32)) if half else (lambda a: a)
    o = orc.trace_forward(orc_cam(cam), sph, h(nsig), h(sc["texel_sites"]), h(sc["texel_rgb"]), h(sc["texel_height"]),
                          adj_np, off_np, pm.cpu().numpy().view(np.uint16), s, thr=1e-3, visit_cap=96)
    assert np.array_equal(r.visit_count.cpu().numpy(), o["visit_count"])
    assert np.array_equal(r.visits.cpu().numpy(), o["visits"])
    for k in ["color", "log_t", "depth", "normal"]:
        assert max_abs(getattr(r, k).cpu(), o[k]) <= 1e-5, k
    assert np.array_equal(r.depth_seg.cpu().numpy(), o["depth_seg"])


def test_trace_step_cap_is_reported():
    sc = np_scene(60, 300, -0.6, 0.6, 0.05, 0.15)
    cam = np_camera((0.0, 0.0, 2.2), (0, 0, 0), 24, 16, 55.0)
    tp = {k: to_t(v) for k, v in sc.items()}
    adj, off = build_power_adjacency(tp["points"], tp["radii"])
    pm = power_adjacency_diff(tp["points"], tp["radii"], adj, off)
    s = start_cell(tp["points"], tp["radii"], torch.from_numpy(cam["eye"]))
    R = RayTracer(Args(), "cuda")
    args = (torch_cam(cam), s, tp["points"], tp["radii"], tp["density"], tp["normals"], tp["texel_sites"],
            tp["texel_rgb"], tp["texel_height"], adj, off, pm, 1e-3)
    with pytest.raises(_lib.PfError) as e:
        R.trace(*args, max_steps=2)
    assert e.value.code == _lib.PF_ERR_STEP_CAP
    r = R.trace(*args, max_steps=2, check_status=False)
    assert int(r.visit_count.max().item()) <= 2


def test_per_ray_start_cells():
    sc = np_scene(61, 300, -0.6, 0.6, 0.05, 0.15)
    cam = np_camera((0.1, 0.0, 2.2), (0, 0, 0), 24, 20, 55.0)
    tp = {k: to_t(v) for k, v in sc.items()}
    adj, off = build_power_adjacency(tp["points"], tp["radii"])
    pm = power_adjacency_diff(tp["points"], tp["radii"], adj, off)
    s = start_cell(tp["points"], tp["radii"], torch.from_numpy(cam["eye"]))
    R = RayTracer(Args(), "cuda")
    base = (tp["points"], tp["radii"], tp["density"], tp["normals"], tp["texel_sites"], tp["texel_rgb"],
            tp["texel_height"], adj, off, pm, 1e-3)
    a = R.trace(torch_cam(cam), s, *base)
    cells = torch.full((20, 24), s, dtype=torch.int32, device="cuda")
    b = R.trace(torch_cam(cam), cells, *base)
    assert torch.equal(a.color, b.color)


@pytest.mark.parametrize("seed,thr,W,H", [(0, 1e-3, 32, 24), (1, 1e-3, 32, 24), (2, 0.3, 29, 21), (3, 0.6, 37, 19)])
def test_trace_adjoint_matches_oracle(seed, thr, W, H):
    """Ragged images (lanes without a pixel in the adjoint's warps) and high
    transmittance thresholds (rays ending between queued hits)."""
    _adjoint_case(seed, thr, W, H, 32)


@pytest.mark.parametrize("kb", [0, 1, 3])
@pytest.mark.parametrize("seed,thr", [(0, 1e-3), (2, 0.3)])
@pytest.mark.parametrize("rec", [True, False])
def test_trace_adjoint_overflow(seed, thr, kb, rec):
    """Few recorded segments per ray: most rays overflow and are finished by
    the resume launch from their saved walk state (kb = 0: all of them);
    records from the forward or from the adjoint's own walk."""
    _adjoint_case(seed, thr, 29, 21, kb, record=rec)


@pytest.mark.parametrize("S", [4, 6])
def test_trace_adjoint_texel_counts(S):
    """Texel counts with (4) and without (6) the float4 gradient atomics."""
    _adjoint_case(5, 1e-3, 29, 21, None, S)



@pytest.mark.parametrize("kb", [None, 2])
def test_trace_adjoint_per_ray_start_cells(kb):
    """Per-ray start cells (the seeded tracer's input): half the rays start in
    the camera's cell, the others in seeded cells anywhere in the scene."""
    _adjoint_case(6, 1e-3, 29, 21, kb, per_ray_start=True)


def _adjoint_case(seed, thr, W, H, kb, S=8, per_ray_start=False, record=True):
    sc = np_scene(80 + seed, 300, -0.6, 0.6, 0.05, 0.15, S=S, height_scale=0.2)
    cam = np_camera((0.3, 0.2 * seed, 2.2), (0, 0, 0), W, H, 55.0)
    tp = {k: to_t(v).requires_grad_(True) for k, v in sc.items()}
    adj, off = build_power_adjacency(tp["points"].detach(), tp["radii"].detach())
    pm = power_adjacency_diff(tp["points"].detach(), tp["radii"].detach(), adj, off)
    s = start_cell(tp["points"].detach(), tp["radii"].detach(), torch.from_numpy(cam["eye"]))
    cells = None
    if per_ray_start:
        cells = np.random.default_rng(100 + seed).integers(0, 300, (H, W)).astype(np.int32)
        cells[: H // 2] = int(s)
    R = RayTracer(Args(), "cuda")
    R.segments_per_ray = kb
    R.record_segments = record
    start = s if cells is None else to_t(cells)
    color, log_t, depth, normal = R.forward(torch_cam(cam), start, tp["points"], tp["radii"], tp["density"],
                                            tp["normals"], tp["texel_sites"], tp["texel_rgb"], tp["texel_height"],
                                            adj, off, pm, thr)
    rng = np.random.default_rng(seed)
    wC = rng.standard_normal((H, W, 3)).astype(np.float32)
    wL = rng.standard_normal((H, W)).astype(np.float32)
    wD = rng.standard_normal((H, W)).astype(np.float32)
    wN = rng.standard_normal((H, W, 3)).astype(np.float32)
    loss = ((color * to_t(wC)).sum() + (log_t * to_t(wL)).sum() + (depth * to_t(wD)).sum()
            + (normal * to_t(wN)).sum())
    loss.backward()
    sph, nsig, _ = packed(sc)
    adj_np, off_np, pm_np = adj.cpu().numpy(), off.cpu().numpy(), pm.cpu().numpy().view(np.uint16)
    f = orc.trace_forward(orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj_np,
                          off_np, pm_np, s if cells is None else 0, start_cells=cells, thr=thr)
    for k, v in [("color", color), ("log_t", log_t), ("depth", depth), ("normal", normal)]:
        assert max_abs(v.detach().cpu(), f[k]) <= 1e-5, k
    g = orc.trace_backward(orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj_np,
                           off_np, pm_np, f, wC, wL, wD, wN, s if cells is None else 0, start_cells=cells,
                           thr=thr)
    from tests.helpers import assert_close_rel
    assert_close_rel(tp["points"].grad.cpu().numpy(), g["spheres"][:, :3], 1e-4, "points")
    assert_close_rel(tp["radii"].grad.cpu().numpy(), g["spheres"][:, 3], 1e-4, "radii")
    assert_close_rel(tp["normals"].grad.cpu().numpy(), g["nsigmas"][:, :3], 1e-4, "normals")
    assert_close_rel(tp["density"].grad.cpu().numpy(), g["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(tp["texel_sites"].grad.cpu().numpy(), g["texel_sites"], 1e-4, "sites")
    assert_close_rel(tp["texel_rgb"].grad.cpu().numpy(), g["texel_rgb"], 1e-4, "rgb")
    assert_close_rel(tp["texel_height"].grad.cpu().numpy(), g["texel_height"], 1e-4, "height")


def test_trace_adjoint_paths_agree_at_scale():
    """131,072 primitives, 320x240: the gradient launch over recorded
    segments (96 per ray), records of one segment (nearly every ray resumed)
    and none (every ray walked by the resume launch), with the records
    written by the forward or by the adjoint's own walk, give the same
    gradients (the atomics sum in different orders: 1e-5 normwise)."""
    from powerfoam_b200 import synthetic
    from powerfoam_b200.adjacency import power_adjacency

    sc = synthetic.make_scene(131072, seed=5, mixture=16, sigma=0.15, r_range=(0.004, 0.04))
    adj, off = power_adjacency(sc["points"], sc["radii"])
    pm = power_adjacency_diff(sc["points"], sc["radii"], adj, off)
    cam = synthetic.orbit_camera(3, 320, 240, 50.0)
    rgb = synthetic.texel_rgb(sc, cam)
    s = start_cell(sc["points"], sc["radii"], cam.eye)
    tw = torch.rand((240, 320, 3), generator=torch.Generator().manual_seed(9)).cuda()
    grads = []
    for kb, rec in ((96, True), (96, False), (1, True), (1, False), (0, True)):
        R = RayTracer(Args(), "cuda")
        R.segments_per_ray = kb
        R.record_segments = rec
        p = {k: sc[k].clone().requires_grad_(True) for k in ["points", "radii", "density", "normals", "texel_sites",
                                                             "texel_height"]}
        c = rgb.clone().requires_grad_(True)
        color, log_t, depth, normal = R.forward(cam, s, p["points"], p["radii"], p["density"], p["normals"],
                                                p["texel_sites"], c, p["texel_height"], adj, off, pm)
        ((color - tw) ** 2).sum().add(log_t.sum()).add(normal.sum()).backward()
        grads.append([p[k].grad for k in p] + [c.grad])
    for other in grads[1:]:
        for a, b in zip(grads[0], other):
            assert torch.isfinite(b).all()
            assert ((a - b).norm() / a.norm().clamp_min(1e-30)).item() <= 1e-5


def test_trace_backward_workspace_checks():
    """The adjoint's C entry rejects a missing, short or misaligned workspace
    and an out-of-range segment count before launching anything."""
    sc = np_scene(90, 200, -0.6, 0.6, 0.05, 0.15)
    cam = np_camera((0.2, 0.1, 2.2), (0, 0, 0), 16, 12, 55.0)
    tp = {k: to_t(v) for k, v in sc.items()}
    adj, off = build_power_adjacency(tp["points"], tp["radii"])
    pm = power_adjacency_diff(tp["points"], tp["radii"], adj, off)
    s = start_cell(tp["points"], tp["radii"], torch.from_numpy(cam["eye"]))
    R = RayTracer(Args(), "cuda")
    args = R._prep(tp["points"], tp["radii"], tp["density"], tp["normals"], tp["texel_sites"], tp["texel_rgb"],
                   tp["texel_height"], adj, off, pm)
    inp = R._inputs(torch_cam(cam), s, *args, 1e-3, 1 << 16, 0.5)
    nbytes = _lib.ctypes.c_size_t(0)
    _lib.call("pf_trace_backward_workspace_size", _lib.ctypes.byref(inp), 8, _lib.ctypes.byref(nbytes))
    assert nbytes.value >= 8 * 48 * 16 * 12
    for kb in (-1, 65536):
        with pytest.raises(_lib.PfError):
            _lib.call("pf_trace_backward_workspace_size", _lib.ctypes.byref(inp), kb, _lib.ctypes.byref(nbytes))
    _lib.call("pf_trace_backward_workspace_size", _lib.ctypes.byref(inp), 8, _lib.ctypes.byref(nbytes))
    n, S = tp["points"].shape[0], tp["texel_sites"].shape[1]
    color = torch.zeros((12, 16, 3), device="cuda")
    g = torch.zeros_like(color)
    out = [torch.zeros(sh, device="cuda") for sh in ((n, 3), (n,), (n, 3), (n,), (n, S, 3), (n, S, 3), (n, S))]
    ws = torch.empty(nbytes.value + 512, dtype=torch.uint8, device="cuda")
    base = (ws.data_ptr() + 255) & ~255
    for ptr, size in ((None, nbytes.value), (base, nbytes.value - 1), (base + 16, nbytes.value)):
        with pytest.raises(_lib.PfError):
            _lib.call("pf_trace_backward", _lib.ctypes.byref(inp), _lib.ptr(color), None, None, None, _lib.ptr(g),
                      None, None, None, *[_lib.ptr(t) for t in out], 8, ptr, size, _lib.stream_ptr())
    _lib.call("pf_trace_backward", _lib.ctypes.byref(inp), _lib.ptr(color), None, None, None, _lib.ptr(g), None,
              None, None, *[_lib.ptr(t) for t in out], 8, base, nbytes.value, _lib.stream_ptr())
    torch.cuda.synchronize()


@pytest.mark.parametrize("cycle_density", [0.0, 3.0])
def test_cycle_guard_matches_oracle(cycle_density):
    """Face records that send the rays round two cells: without hits in the
    cycle every walk ends where it comes back to a saved cell (the reference
    would loop for ever); with hits it walks on until the transmittance
    ends it.  Visited cells bit-exact against the oracle."""
    from tests.helpers import cycle_scene

    sc, adj, off, faces, cam = cycle_scene(cycle_density)
    tp = {k: to_t(v) for k, v in sc.items()}
    R = RayTracer(Args(), "cuda")
    r = R.trace(torch_cam(cam), 0, tp["points"], tp["radii"], tp["density"], tp["normals"], tp["texel_sites"],
                tp["texel_rgb"], tp["texel_height"], to_t(adj), to_t(off), to_t(faces), 1e-3, visit_cap=64)
    sph, nsig, _ = packed(sc)
    o = orc.trace_forward(orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj, off,
                          faces.view(np.uint16), 0, thr=1e-3, visit_cap=64)
    assert (o["status"] == 0).all()
    assert np.array_equal(r.visit_count.cpu().numpy(), o["visit_count"])
    assert np.array_equal(r.visits.cpu().numpy(), o["visits"])
    assert max_abs(r.color.cpu(), o["color"]) <= 1e-5


@pytest.mark.parametrize("kb,rec", [(None, True), (1, True), (1, False), (0, True)])
@pytest.mark.parametrize("cycle_density", [0.0, 3.0])
def test_cycle_guard_adjoint_matches_oracle(cycle_density, kb, rec):
    """The adjoint's walks apply the same guard, including the resume launch
    that takes over a ray's saved walk state (kb = 0, 1)."""
    from tests.helpers import assert_close_rel, cycle_scene

    sc, adj, off, faces, cam = cycle_scene(cycle_density)
    tp = {k: to_t(v).requires_grad_(True) for k, v in sc.items()}
    R = RayTracer(Args(), "cuda")
    R.segments_per_ray = kb
    R.record_segments = rec
    color, log_t, depth, normal = R.forward(torch_cam(cam), 0, tp["points"], tp["radii"], tp["density"],
                                            tp["normals"], tp["texel_sites"], tp["texel_rgb"], tp["texel_height"],
                                            to_t(adj), to_t(off), to_t(faces), 1e-3)
    H, W = cam["height"], cam["width"]
    rng = np.random.default_rng(3)
    wC, wL = rng.standard_normal((H, W, 3)).astype(np.float32), rng.standard_normal((H, W)).astype(np.float32)
    ((color * to_t(wC)).sum() + (log_t * to_t(wL)).sum()).backward()
    sph, nsig, _ = packed(sc)
    f = orc.trace_forward(orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj, off,
                          faces.view(np.uint16), 0, thr=1e-3)
    assert max_abs(color.detach().cpu(), f["color"]) <= 1e-5
    g = orc.trace_backward(orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"], adj, off,
                           faces.view(np.uint16), f, wC, wL, None, None, 0, thr=1e-3)
    assert_close_rel(tp["density"].grad.cpu().numpy(), g["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(tp["texel_rgb"].grad.cpu().numpy(), g["texel_rgb"], 1e-4, "rgb")
    assert_close_rel(tp["points"].grad.cpu().numpy(), g["spheres"][:, :3], 1e-4, "points")
    assert float(tp["density"].grad[0].abs()) > 0


def test_sync_free_forward_reports_the_step_cap_on_check():
    """host_sync=False: the differentiable forward does not read its status
    back; a walk stopped by the step cap raises at check(), which clears the
    word."""
    sc = np_scene(62, 300, -0.6, 0.6, 0.05, 0.15)
    cam = np_camera((0.0, 0.0, 2.2), (0, 0, 0), 24, 16, 55.0)
    tp = {k: to_t(v).requires_grad_(True) for k, v in sc.items()}
    adj, off = build_power_adjacency(tp["points"].detach(), tp["radii"].detach())
    pm = power_adjacency_diff(tp["points"].detach(), tp["radii"].detach(), adj, off)
    s = start_cell(tp["points"].detach(), tp["radii"].detach(), torch.from_numpy(cam["eye"]))
    R = RayTracer(Args(), "cuda")
    R.host_sync = False
    args = (torch_cam(cam), s, tp["points"], tp["radii"], tp["density"], tp["normals"], tp["texel_sites"],
            tp["texel_rgb"], tp["texel_height"], adj, off, pm, 1e-3)
    color, _, _, _ = R.forward(*args)
    color.sum().backward()
    assert R.check()
    R.forward(*args, max_steps=2)
    with pytest.raises(_lib.PfError) as e:
        R.check()
    assert e.value.code == _lib.PF_ERR_STEP_CAP
    assert R.check()
