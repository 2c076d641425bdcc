"""Ray-proposal network (pf_mlp.cu) and the proposal-seeded walk, against the
CPU oracles (oracle/mlp_oracle.py, oracle/pf_oracle.c).

Tolerances: tensor-core GEMMs normwise relative 1e-4 against float64 products
of the same BF16 operands; network outputs max-abs 2e-3 (BF16 rounding of an
intermediate can flip when the FP32 accumulation order differs); gradients
normwise relative 1e-2 per layer; Adam relative 1e-6; tracer labels and cell
location bit-exact; seeded image >= 50 dB PSNR against the plain walk."""

import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo
from oracle import oracle as orc
from powerfoam_b200 import _lib
from oracle.power_hull import build_power_adjacency
from powerfoam_b200.adjacency import power_adjacency_diff, start_cell
from powerfoam_b200.proposal import (CellLocator, ProposalNet, SeededTracer, camera_rays, make_training_rays,
                                     trace_labels)
from powerfoam_b200.raytrace import RayTracer
from tests.helpers import assert_close_rel, np_camera, np_scene, orc_cam, to_t, torch_cam

pytestmark = pytest.mark.gpu


def bf16_tensor(x):
    return torch.from_numpy(mo.bf16_bits(x).view(np.int16)).cuda()


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_tensor_core_gemm_layouts(mode):
    rng = np.random.default_rng(mode)
    a = mo.bf16(rng.standard_normal((128, 128)).astype(np.float32))
    b = mo.bf16(rng.standard_normal((80, 128)).astype(np.float32))
    d = torch.empty((128, 80), dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    ta, tb = bf16_tensor(a), bf16_tensor(b)  # held until the kernel has run
    _lib.call("pf_mlp_gemm_selftest", _lib.ptr(ta), _lib.ptr(tb), mode, _lib.ptr(d), _lib.ptr(st),
              _lib.stream_ptr())
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    assert_close_rel(d.cpu().numpy(), ref, 1e-4, f"mode {mode}")


def random_params(seed):
    p = mo.init_params(seed)
    rng = np.random.default_rng(seed + 50)
    ws = mo.layers(p)
    for li, w in enumerate(ws):  # nonzero biases exercise the constant-1 input column
        rows = 64 if li < 3 else 2
        w[:rows, mo.ONES[li]] = rng.uniform(-0.2, 0.2, rows)
    return np.concatenate([w.reshape(-1) for w in ws]).astype(np.float32)


def random_rays(n, seed, with_labels=False):
    rng = np.random.default_rng(seed)
    o = rng.standard_normal((n, 3))
    o = 3.0 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = -o / 3.0 + 0.4 * rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.concatenate([o, d], 1).astype(np.float32)
    if not with_labels:
        return r
    t = rng.uniform(1.0, 4.0, n)
    t[rng.uniform(size=n) < 0.3] = -1.0
    flag = (t >= 0) & (rng.uniform(size=n) < 0.25)  # no-hit rays labelled where they leave the box
    return np.concatenate([r, t[:, None], flag[:, None]], 1).astype(np.float32)


def test_forward_matches_oracle():
    p = random_params(1)
    net = ProposalNet("cuda")
    net.load_weights(torch.from_numpy(p))
    rays = random_rays(1000, 2)  # 8 tiles, the last partial
    t, c = net.forward(rays=to_t(rays))
    torch.cuda.synchronize()
    net.check()
    t_ref, c_ref = mo.forward(p, rays)
    err_t = np.abs(t.cpu().numpy() - t_ref)
    assert err_t.max() <= 2e-3 and np.median(err_t) <= 1e-5
    assert np.abs(c.cpu().numpy() - c_ref).max() <= 2e-3


def test_forward_camera_rays_match_explicit_rays():
    p = random_params(3)
    net = ProposalNet("cuda")
    net.load_weights(torch.from_numpy(p))
    cam = torch_cam(np_camera((0.5, 1.0, 2.7), (0, 0, 0), 37, 29, 50.0))
    t_cam, c_cam = net.forward(camera=cam)
    t_r, c_r = net.forward(rays=camera_rays(cam))
    # the two paths round the ray direction differently (kernel vs torch op
    # order); the 32 pi encoding frequency amplifies that into BF16 flips
    dt = np.abs(t_cam.reshape(-1).cpu().numpy() - t_r.cpu().numpy())
    assert dt.max() <= 2e-2 and np.median(dt) <= 1e-3
    assert np.abs(c_cam.reshape(-1).cpu().numpy() - c_r.cpu().numpy()).max() <= 2e-2


@pytest.mark.parametrize("batch", [300, 1024])
def test_train_step_gradient_matches_oracle(batch):
    p = random_params(4)
    net = ProposalNet("cuda")
    net.load_weights(torch.from_numpy(p))
    rays = random_rays(1000, 5, with_labels=True)
    seed = 77
    net.grad.zero_()
    net.loss.zero_()
    rays_dev = to_t(rays)  # held until the kernel has run
    _lib.call("pf_mlp_train_step", _lib.ptr(net.image), _lib.ptr(rays_dev), rays.shape[0], batch,
              _lib.ptr(net.step), seed, 10.0, 0.02, _lib.ptr(net.grad), _lib.ptr(net.loss), _lib.ptr(net.status),
              _lib.stream_ptr())
    torch.cuda.synchronize()
    net.check()
    g_ref, (lt, lc), _, _ = mo.train_grad(p, rays, batch, 0, seed, 10.0, 0.02)
    g = net.grad.cpu().numpy()
    o = 0
    for li, out in enumerate(mo.OUTS):
        n = out * mo.K_IN
        assert_close_rel(g[o:o + n], g_ref[o:o + n], 1e-2, f"layer {li}")
        o += n
    loss = net.loss.cpu().numpy()
    assert abs(loss[0] - lt) <= 1e-3 * max(lt, 1e-6)
    assert abs(loss[1] - lc) <= 1e-3 * lc


def test_adam_matches_oracle_and_repacks():
    p = random_params(6)
    net = ProposalNet("cuda")
    net.load_weights(torch.from_numpy(p))
    rng = np.random.default_rng(7)
    g = (rng.standard_normal(p.shape[0]) * 1e-2).astype(np.float32)
    m0 = (rng.standard_normal(p.shape[0]) * 1e-3).astype(np.float32)
    v0 = (rng.uniform(0, 1e-4, p.shape[0])).astype(np.float32)
    net.grad.copy_(to_t(g))
    net.m.copy_(to_t(m0))
    net.v.copy_(to_t(v0))
    net.step.fill_(3)
    _lib.call("pf_mlp_adam", _lib.ptr(net.weights), _lib.ptr(net.m), _lib.ptr(net.v), _lib.ptr(net.grad),
              _lib.ptr(net.image), _lib.ptr(net.step), _lib.ptr(net.done), 1e-3, 0.9, 0.999, 1e-8, _lib.stream_ptr())
    torch.cuda.synchronize()
    w_ref, m_ref, v_ref = mo.adam(p, m0, v0, g, 3)
    assert_close_rel(net.weights.cpu().numpy(), w_ref, 1e-6, "w")
    assert_close_rel(net.m.cpu().numpy(), m_ref, 1e-6, "m")
    assert_close_rel(net.v.cpu().numpy(), v_ref, 1e-6, "v")
    assert int(net.step.item()) == 4 and int(net.done.item()) == 0
    assert float(net.grad.abs().max()) == 0.0
    img = net.image.clone()
    net.pack()
    assert torch.equal(img, net.image)


class TArgs:
    num_texel_sites = 8


def test_trace_labels_match_oracle():
    sc = np_scene(31, 3000, -0.7, 0.7, 0.02, 0.08)
    t = {k: to_t(v) for k, v in sc.items()}
    adj, off = build_power_adjacency(t["points"], t["radii"])
    pm = power_adjacency_diff(t["points"], t["radii"], adj, off)
    cam = np_camera((0.4, 0.9, 2.4), (0, 0, 0), 48, 40, 55.0)
    tc = torch_cam(cam)
    st = start_cell(t["points"], t["radii"], tc.eye)
    tr = RayTracer(TArgs(), "cuda")
    args = (t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"], t["texel_rgb"], t["texel_height"],
            adj, off, pm)
    lab = trace_labels(tr, tc, st, args)
    torch.cuda.synchronize()
    sph = np.concatenate([sc["points"], sc["radii"][:, None]], -1).astype(np.float32)
    nsig = np.concatenate([sc["normals"], sc["density"][:, None]], -1).astype(np.float32)
    o = orc.trace_labels(orc_cam(cam), sph, nsig, sc["texel_sites"], sc["texel_rgb"], sc["texel_height"],
                         adj.cpu().numpy(), off.cpu().numpy(), pm.cpu().numpy().view(np.uint16), start_idx=st)
    assert np.array_equal(lab["label_cell"].cpu().numpy(), o["label_cell"])
    assert np.array_equal(lab["label_step"].cpu().numpy(), o["label_step"])
    assert np.array_equal(lab["label_t"].cpu().numpy(), o["label_t"])
    assert np.array_equal(lab["visit_count"].cpu().numpy(), o["visit_count"])
    assert np.abs(lab["color"].cpu().numpy() - o["color"]).max() <= 1e-5
    assert (o["label_cell"] >= 0).any() and (o["label_cell"] < 0).any()


def test_locate_cells_match_brute_force():
    sc = np_scene(41, 5000, -0.8, 0.8, 0.01, 0.06)
    pts, rad = sc["points"], sc["radii"]
    rng = np.random.default_rng(42)
    q = np.concatenate([rng.uniform(-1.2, 1.2, (3000, 3)), pts[:500] + 1e-4,  # near sites
                        rng.uniform(-3, 3, (200, 3))]).astype(np.float32)  # far outside the bounds
    loc = CellLocator(to_t(pts), to_t(rad))
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    got = loc.locate(to_t(q), st).cpu().numpy()
    assert int(st.item()) == 0
    dx = q[:, None, 0] - pts[None, :, 0]
    dy = q[:, None, 1] - pts[None, :, 1]
    dz = q[:, None, 2] - pts[None, :, 2]
    pd = ((dx * dx + dy * dy) + dz * dz) - (rad * rad)[None, :]
    assert np.array_equal(got, np.argmin(pd, axis=1).astype(np.int32))


@pytest.mark.parametrize("res", [8, 64])
def test_voxel_map_location_matches_brute_force(res):
    """Points located from the voxel map (their voxel's cell, then a walk
    across power faces) are in the cell of least power distance: the same
    cell, or one whose power distance equals it to float32 rounding (a point
    on a face).  Coarse (8^3, long walks) and fine (64^3) maps; points inside,
    near sites and far outside the primitives' box."""
    from powerfoam_b200.adjacency import power_adjacency
    from powerfoam_b200.proposal import VoxelLocator

    sc = np_scene(43, 5000, -0.8, 0.8, 0.01, 0.06)
    pts, rad = sc["points"], sc["radii"]
    adj, off = power_adjacency(to_t(pts), to_t(rad))
    rng = np.random.default_rng(44)
    q = np.concatenate([rng.uniform(-1.0, 1.0, (4000, 3)), pts[:500] + 1e-4,
                        rng.uniform(-3, 3, (300, 3))]).astype(np.float32)
    loc = VoxelLocator(to_t(pts), to_t(rad), adj, off, res=res, max_walk_steps=256)
    got = loc.locate(to_t(q)).cpu().numpy()
    assert (got >= 0).all()
    d = q[:, None, :].astype(np.float64) - pts[None, :, :].astype(np.float64)
    pd = (d * d).sum(-1) - (rad.astype(np.float64) ** 2)[None, :]
    rows = np.arange(q.shape[0])
    best = np.argmin(pd, axis=1)
    same = got == best
    gap = pd[rows, got] - pd[rows, best]
    assert same.mean() >= 0.999
    assert (gap[~same] <= 1e-5 * (1.0 + np.abs(pd[rows, best][~same]))).all()


def psnr(a, b):
    mse = float(((a.double() - b.double()) ** 2).mean())
    return 10 * np.log10(1.0 / max(mse, 1e-20))


def test_trained_proposal_seeds_at_50db():
    """Train on plain-walk labels of 2M rays (2048 small random views of a
    scene of opaque shells in empty space; rays
    that never reach a significant cell labelled with the distance at which
    they leave the primitives' box), calibrate the confidence gate on 256
    more, evaluate on held-out views: the network seeds a real share of the
    rays, the seeded walk visits fewer cells than the plain walk and keeps
    >= 50 dB PSNR against it.  Seeding from the plain walk's own labels
    through the same voxel-map location shows the headroom a perfect
    proposal would have (>= 50 dB with fewer cells)."""
    from powerfoam_b200.proposal import box_exit
    from powerfoam_b200 import synthetic

    # opaque shells in empty space: most rays never reach a significant cell, so a proposal has
    # something to skip (on the cloud scene of the 6.3M-primitive workload even seeding from the
    # plain walk's own labels saves no time: bench.py --workload proposal)
    n = 60000
    scale = (6291456 / n) ** (1 / 3)
    sc = synthetic.make_scene(n, seed=4, mixture=16, sigma=0.1, r_range=(0.001 * scale, 0.01 * scale),
                              shells=(0.12, 0.02, 30.0))
    rgb = synthetic.texel_rgb(sc, synthetic.front_camera(64, 64, 50.0))
    adj, off = build_power_adjacency(sc["points"], sc["radii"])
    pm = power_adjacency_diff(sc["points"], sc["radii"], adj, off)
    args = (sc["points"], sc["radii"], sc["density"], sc["normals"], sc["texel_sites"], rgb, sc["texel_height"], adj,
            off, pm)
    tr = RayTracer(TArgs(), "cuda")

    def views(seed0, k, w, h):
        cams = [synthetic.orbit_camera(seed0 + i, w, h, 50.0) for i in range(k)]
        return cams, [start_cell(sc["points"], sc["radii"], c.eye) for c in cams]

    box = (sc["points"].min(0).values, sc["points"].max(0).values)

    def labelled(seed0, k):
        cams, starts = views(seed0, k, 32, 32)
        return make_training_rays(tr, cams, args, starts, label_transmittance=0.999, box=box)

    rays8 = labelled(10000, 2048)
    val = labelled(50000, 256)
    net = ProposalNet("cuda", seed=1)
    hist = net.train(rays8, steps=5000, batch=65536, lr=1e-3, overshoot_weight=100.0, margin=0.1, graph_steps=100)
    # the entry-distance loss falls; the confidence targets move with the predictions (a seed's
    # safety depends on the predicted t), so that loss is only required to be well below chance (ln 2)
    assert hist[-1][0] < hist[0][0] and hist[-1][1] < 0.3
    # strict gate: no held-out seed past its first significant cell, nor within one margin of it
    # (a budget of 1e-4 of the held-out rays, or the gate without that slack, let eval views drop
    # below 50 dB: training differs from run to run in the order of its float atomics)
    thr = net.calibrate(val, t_slack=net.margin)
    print(f"calibrated threshold {thr:.5f}: {net.seed_fraction(val, thr):.3f} of the held-out rays seeded")
    seeded_tr = SeededTracer(tr, net, sc["points"], sc["radii"], conf_threshold=thr, adjacency=adj,
                             adjacency_offsets=off)
    for ev in (synthetic.orbit_camera(900 + i, 256, 192, 50.0) for i in range(2)):
        st = start_cell(sc["points"], sc["radii"], ev.eye)
        plain = tr.trace(ev, st, *args)
        seeded_tr.n_seeded.zero_()
        seeded = seeded_tr.render(ev, st, args)
        lab = trace_labels(tr, ev, st, args, label_transmittance=0.999)
        hit = lab["label_cell"] >= 0
        one = torch.ones_like(lab["label_t"])
        t_exit = box_exit(camera_rays(ev), box[0], box[1]).view_as(lab["label_t"])
        t_lab = (torch.where(hit, lab["label_t"], t_exit) - net.margin).contiguous()
        ideal_start = seeded_tr.locator.seed(ev, t_lab, one.contiguous(), 0.5, st)
        ideal = tr.trace(ev, ideal_start, *args)
        torch.cuda.synchronize()
        v_plain, v_seed, v_ideal = (int(r.visit_count.sum()) for r in (plain, seeded, ideal))
        p, p_ideal = psnr(seeded.color, plain.color), psnr(ideal.color, plain.color)
        print(f"threshold {seeded_tr.conf_threshold:.5f}: seeded {int(seeded_tr.n_seeded.item())}/{256 * 192} "
              f"rays, {p:.1f} dB, cells {v_seed}/{v_plain}; label seeding {p_ideal:.1f} dB, cells {v_ideal}")
        assert int(seeded_tr.n_seeded.item()) >= 0.02 * 256 * 192
        assert p >= 50.0 and v_seed < v_plain
        assert p_ideal >= 50.0 and v_ideal < v_plain
