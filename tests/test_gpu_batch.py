"""Batched multi-view step (pf_batch_render through powerfoam_b200.batch):
per view bit-identical to the single-view rasterizer, gradients equal to the
sum over views, images and gradients against the CPU oracle, CUDA-graph
replay, the SH pre-step adjoint and the autotuner's cache.

Tolerances: images, early-stop indices and dL/dcolor bit-exact against the
single-view kernels (same tile code); images max-abs 1e-5 against the oracle;
gradients normwise relative 1e-4 against the oracle and 1e-5 against the sum
of single-view gradients (only the order of the float additions differs)."""

import json

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from powerfoam_b200 import _lib
from powerfoam_b200.batch import BatchStep, autotune, tune_key
from powerfoam_b200.rasterize import Rasterizer
from tests.helpers import assert_close_rel, cech_np, max_abs, np_camera, np_scene, orc_cam, packed, to_t, torch_cam

pytestmark = pytest.mark.gpu


class Args:
    is_pinhole = True
    render_objective = "volume"
    num_texel_sites = 8


# uneven resolutions, ragged tiles at every width
VIEW_SPECS = [((0.2, 0.5, 2.3), 61, 37, 55.0), ((-1.6, 0.3, 1.5), 40, 30, 60.0), ((1.2, -0.8, 1.9), 96, 54, 50.0)]


def make_case(seed=3, n=500, views=VIEW_SPECS):
    sc = np_scene(seed, n, -0.6, 0.6, 0.03, 0.15)
    adj, adj_off = cech_np(sc["points"], sc["radii"])
    cams = [np_camera(eye, (0, 0, 0), W, H, fov) for eye, W, H, fov in views]
    rng = np.random.default_rng(seed + 100)
    rgbs = [rng.uniform(0, 1, sc["texel_rgb"].shape).astype(np.float32) for _ in cams]
    targets = [rng.uniform(0, 1, (c["height"], c["width"], 3)).astype(np.float32) for c in cams]
    return sc, adj, adj_off, cams, rgbs, targets


def bind_kwargs(sc, adj, adj_off, rgbs, targets):
    return dict(points=to_t(sc["points"]), radii=to_t(sc["radii"]), density=to_t(sc["density"]),
                normals=to_t(sc["normals"]), texel_sites=to_t(sc["texel_sites"]),
                texel_height=to_t(sc["texel_height"]), adjacency=to_t(adj), adjacency_offsets=to_t(adj_off),
                targets=[to_t(t) for t in targets], texel_rgb=[to_t(r) for r in rgbs])


def single_view(sc, adj, adj_off, cam, rgb, target, tw):
    R = Rasterizer(Args(), "cuda", tile_width=tw)
    t = {k: to_t(sc[k]).requires_grad_(True) for k in ["points", "radii", "density", "normals", "texel_sites",
                                                         "texel_height"]}
    rgb_t = to_t(rgb).requires_grad_(True)
    out = R.forward(torch_cam(cam), None, t["points"], t["radii"], t["density"], t["normals"], t["texel_sites"],
                    rgb_t, t["texel_height"], to_t(adj), to_t(adj_off), None, False)
    loss = ((out[0] - to_t(target)) ** 2).sum()
    loss.backward()
    return out, loss, {k: v.grad for k, v in t.items()}, rgb_t.grad, R


@pytest.mark.parametrize("tw,chunk,order,split", [(8, 1, "longest", False), (8, 3, "view", True),
                                                  (16, 2, "longest", False), (16, 1, "view", True),
                                                  (32, 1, "longest", False), (32, 5, "view", True)])
def test_batch_matches_single_view_kernels(tw, chunk, order, split):
    sc, adj, adj_off, cams, rgbs, targets = make_case()
    step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=tw, chunk=chunk, order=order, split=split)
    step.bind(**bind_kwargs(sc, adj, adj_off, rgbs, targets))
    loss = step.run().clone()
    step.check()
    gsum = None
    for v, cam in enumerate(cams):
        out, l1, grads, g_rgb, R = single_view(sc, adj, adj_off, cam, rgbs[v], targets[v], tw)
        color, opacity, nd, normal = out[0], out[1], out[2], out[3]
        assert torch.equal(step.color[v], color.detach())
        assert torch.equal(step.log_t[v].exp().neg().add(1), opacity.detach())
        assert torch.equal(step.normal_distance[v], nd.detach())
        assert torch.equal(step.normal[v], normal.detach())
        assert torch.equal(step.grad_color[v], 2 * (color.detach() - to_t(targets[v])))
        assert abs(float(loss[v]) - float(l1.detach())) <= 1e-5 * float(l1.detach())
        assert_close_rel(step.grad_texel_rgb[v].cpu().numpy(), g_rgb.cpu().numpy(), 1e-5, f"rgb view {v}")
        gsum = grads if gsum is None else {k: gsum[k] + grads[k] for k in gsum}
    for k in gsum:
        assert_close_rel(step.grads[k].cpu().numpy(), gsum[k].cpu().numpy(), 1e-5, k)


@pytest.mark.parametrize("tw", [8, 32])
def test_batch_matches_oracle(tw):
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=7)
    step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=tw, chunk=2)
    step.bind(**bind_kwargs(sc, adj, adj_off, rgbs, targets))
    step.run()
    step.check()
    N, S = sc["points"].shape[0], sc["texel_sites"].shape[1]
    acc = dict(spheres=np.zeros((N, 4)), nsigmas=np.zeros((N, 4)), texel_sites=np.zeros((N, S, 3)),
               texel_height=np.zeros((N, S)))
    for v, cam in enumerate(cams):
        scv = dict(sc, texel_rgb=rgbs[v])
        sph, nsig, rgbh = packed(scv)
        oc = orc_cam(cam)
        keys, prims, offs, _ = orc.bin(oc, sph, tw)
        ad = orc.prefetch_adjacency(sph, adj, adj_off)
        o = orc.raster_forward(oc, tw, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims, None, None,
                               1e-3, False)
        assert max_abs(step.color[v].cpu(), o["color"]) <= 1e-5
        assert max_abs(step.log_t[v].cpu(), o["log_t"]) <= 1e-5
        assert np.array_equal(step.early_stop[v].cpu().numpy(), o["early_stop"])
        H, W = cam["height"], cam["width"]
        g_c = (2 * (o["color"] - targets[v])).astype(np.float32)
        z = np.zeros((H, W), np.float32)
        gr = orc.raster_backward(oc, tw, sph, nsig, sc["texel_sites"], rgbh, adj, adj_off, ad, offs, prims,
                                 o["early_stop"], o["log_t"], g_c, z, z, np.zeros((H, W, 3), np.float32),
                                 np.zeros(N, np.float32))
        for k in acc:
            acc[k] += gr[k]
        assert_close_rel(step.grad_texel_rgb[v].cpu().numpy(), gr["texel_rgb"], 1e-4, f"rgb view {v}")
    g = step.grads
    assert_close_rel(g["points"].cpu().numpy(), acc["spheres"][:, :3], 1e-4, "points")
    assert_close_rel(g["radii"].cpu().numpy(), acc["spheres"][:, 3], 1e-4, "radii")
    assert_close_rel(g["normals"].cpu().numpy(), acc["nsigmas"][:, :3], 1e-4, "normals")
    assert_close_rel(g["density"].cpu().numpy(), acc["nsigmas"][:, 3], 1e-4, "density")
    assert_close_rel(g["texel_sites"].cpu().numpy(), acc["texel_sites"], 1e-4, "sites")
    assert_close_rel(g["texel_height"].cpu().numpy(), acc["texel_height"], 1e-4, "height")


def test_batch_graph_replay_tracks_in_place_updates():
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=11)
    kw = bind_kwargs(sc, adj, adj_off, rgbs, targets)
    step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=16, chunk=2)
    step.bind(**kw)
    step.capture()
    with torch.no_grad():
        kw["density"].mul_(1.3)
        kw["points"].add_(0.01)
    step.run()
    torch.cuda.synchronize()
    step.check()
    replay = [c.clone() for c in step.color] + [step.grads[k].clone() for k in sorted(step.grads)]
    ref = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=16, chunk=2)
    ref.bind(**kw)
    ref.run()
    eager = [c.clone() for c in ref.color] + [ref.grads[k].clone() for k in sorted(ref.grads)]
    for a, b in zip(replay[:3], eager[:3]):
        assert torch.equal(a, b)
    for a, b in zip(replay[3:], eager[3:]):
        assert_close_rel(a.cpu().numpy(), b.cpu().numpy(), 1e-5, "grad")
    # the update changed the images
    base = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=16, chunk=2)
    base.bind(**bind_kwargs(sc, adj, adj_off, rgbs, targets))
    base.run()
    assert not torch.equal(base.color[0], replay[0])


def test_batch_sh_prestep_and_adjoint():
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=5)
    rng = np.random.default_rng(9)
    sh = (rng.standard_normal((sc["points"].shape[0], 16, 3)) * 0.3).astype(np.float32)
    kw = bind_kwargs(sc, adj, adj_off, rgbs, targets)
    kw.pop("texel_rgb")
    step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=8)
    step.bind(**kw, sh=to_t(sh))
    step.run()
    step.check()
    g_sh = np.zeros_like(sh)
    for v, cam in enumerate(cams):
        rgb = orc.sh_texel_rgb(sc["points"], sh, cam["eye"], S=sc["texel_sites"].shape[1])
        assert max_abs(step.texel_rgb[v].cpu(), rgb) <= 1e-6
        orc.sh_texel_rgb_backward(sc["points"], sh, cam["eye"], step.grad_texel_rgb[v].cpu().numpy(), g_sh)
    assert_close_rel(step.grad_sh.cpu().numpy(), g_sh, 1e-5, "sh")


def test_batch_argument_errors():
    sc, adj, adj_off, cams, rgbs, targets = make_case(n=50)
    with pytest.raises(ValueError):
        BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=12)
    step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=8)
    kw = bind_kwargs(sc, adj, adj_off, rgbs, targets)
    with pytest.raises(ValueError):
        step.bind(**dict(kw, targets=kw["targets"][:2]))
    step.bind(**kw)
    step.set_schedule(chunk=0)
    with pytest.raises(_lib.PfError):
        step.run()


def test_autotune_sweeps_and_caches(tmp_path):
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=13, n=300)
    tcams = [torch_cam(c) for c in cams]
    kw = bind_kwargs(sc, adj, adj_off, rgbs, targets)
    path = str(tmp_path / "tune.json")
    step, table = autotune("cuda", tcams, kw, tile_widths=(8, 16), chunks=(1, 2), orders=("longest",), iters=1,
                           warmup=1, cache_path=path, prune=0)
    assert len(table) == 8 and all(r["render_ms"] > 0 for r in table)
    for tw in (8, 16):  # each width's step was timed with its fastest render schedule
        rows = [r for r in table if r["tile_width"] == tw]
        timed = [r for r in rows if r["step_ms"] is not None]
        assert len(timed) == 1 and timed[0]["render_ms"] == min(r["render_ms"] for r in rows)
    best = min((r for r in table if r["step_ms"] is not None), key=lambda r: r["step_ms"])
    assert (step.tile_width, step.chunk, step.order, step.split) == (best["tile_width"], best["chunk"],
                                                                     best["order"], best["split"])
    cache = json.load(open(path))
    key = tune_key(torch.device("cuda"), tcams, sc["points"].shape[0], sc["texel_sites"].shape[1])
    assert cache[key]["tile_width"] == best["tile_width"]
    step2, table2 = autotune("cuda", tcams, kw, tile_widths=(8, 16), chunks=(1, 2), orders=("longest",),
                             cache_path=path, prune=0)
    assert table2 == cache[key]["table"]
    assert (step2.tile_width, step2.chunk) == (step.tile_width, step.chunk)
    step2.run()
    step2.check()


def test_schedule_tuner_through_the_c_abi():
    """pf_batch_autotune times every schedule, picks the fastest, and leaves
    the outputs of a valid render (equal to a plain run's image)."""
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=14, n=300)
    tcams = [torch_cam(c) for c in cams]
    step = BatchStep("cuda", tcams, 8, 1, "longest")
    step.bind(**bind_kwargs(sc, adj, adj_off, rgbs, targets))
    step.run()
    ref = [c.clone() for c in step.color]
    scheds = [(1, "longest", False), (4, "view", False), (2, "longest", True)]
    times, best = step.tune_schedules(scheds, iters=2, warmup=1)
    assert len(times) == 3 and all(t > 0 for t in times) and times[best] == min(times)
    torch.cuda.synchronize()
    for a, b in zip(ref, step.color):
        assert torch.equal(a, b)
    with pytest.raises(ValueError):
        step.tune_schedules([(1, "random", False)])


@pytest.mark.parametrize("tw,split", [(8, False), (8, True), (16, False), (16, True)])
def test_batch_segment_records_give_the_clipping_adjoint(tw, split):
    """The batch launch with segment records (the forward stores each hit
    pixel's interval and plane result, the adjoint reads them) against the
    one that clips again: the same images and losses, gradients equal up to
    the order of the float atomics; so do a budget that holds the intervals
    only, a record buffer too small for most pairs (those are clipped again),
    and every view in a record group of its own (the groups render one after
    the other, reusing the buffer).  check() counts again and grows a buffer
    that a group's count outran."""
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=13)
    kw = bind_kwargs(sc, adj, adj_off, rgbs, targets)
    res = []
    for case in ("clip", "records", "small", "intervals", "groups"):
        step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=tw, chunk=2, split=split,
                         record_segments=case != "clip")
        step.bind(**kw)
        if case != "clip":
            n_rec = sum(step.view_records)
            assert n_rec > 0 and step.segs is not None and step.segs[2] is True
            assert step.seg_groups == [0] * len(cams)  # the whole batch fits one group
        if case == "intervals":
            step.segment_bytes = 16 * step.rec_capacity
            step._size_records()
            assert step.segs[2] is False
        if case == "small":  # a buffer for an eighth of the records
            step.rec_capacity = max(n_rec // 8, 1)
            step._size_records()
        if case == "groups":
            step.seg_groups = list(range(len(cams)))
            step._size_records()
        loss = step.run().clone()
        res.append((loss, [c.clone() for c in step.color], {k: g.clone() for k, g in step.grads.items()},
                    [g.clone() for g in step.grad_texel_rgb]))
        if case == "groups":
            assert step.rec_count.tolist() == step.view_records  # one counter per group, here per view
        step.check()
        if case == "small":  # counted again and grown
            assert step.rec_capacity >= n_rec and step.graph is None
    loss0, col0, g0, rgb0 = res[0]
    for loss, col, g, rgb in res[1:]:
        assert torch.equal(loss, loss0)
        for a, b in zip(col, col0):
            assert torch.equal(a, b)
        for k in g0:
            assert_close_rel(g[k].cpu().numpy(), g0[k].cpu().numpy(), 1e-5, k)
        for a, b in zip(rgb, rgb0):
            assert_close_rel(a.cpu().numpy(), b.cpu().numpy(), 1e-5, "rgb")


def test_batch_record_groups_through_the_c_abi():
    """Record groups as pf_batch_render takes them: 0 for the first view,
    then the previous view's group or the next; anything else is refused with
    PF_ERR_ARGS before any launch."""
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=17)
    step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=8)
    step.bind(**bind_kwargs(sc, adj, adj_off, rgbs, targets))
    for bad in ([0, 1, 0], [0, 2, 2], [1, 1, 1]):
        step.seg_groups = bad
        step._size_records()
        with pytest.raises(_lib.PfError):
            step.run()
    step.seg_groups = [0, 1, 1]
    step._size_records()
    step.run()
    step.check()


def test_batch_segment_records_with_an_empty_view_and_ragged_tiles():
    """A view that looks away from the scene (no sphere hits, no records) between
    two ragged views, every view in a record group of its own and all in one:
    the same images and gradients as without records."""
    views = [((0.2, 0.5, 2.3), 61, 37, 55.0), ((0.0, 0.0, 3.0), 23, 19, 40.0), ((1.2, -0.8, 1.9), 45, 27, 50.0)]
    sc, adj, adj_off, cams, rgbs, targets = make_case(seed=19, views=views)
    cams[1] = np_camera((0.0, 0.0, 3.0), (0.0, 0.0, 6.0), 23, 19, 40.0)  # facing away
    kw = bind_kwargs(sc, adj, adj_off, rgbs, targets)
    res = []
    for rec, groups in ((False, None), (True, None), (True, [0, 1, 2])):
        step = BatchStep("cuda", [torch_cam(c) for c in cams], tile_width=8, split=True, record_segments=rec)
        step.bind(**kw)
        if rec:
            assert step.view_records[1] == 0 and step.view_records[0] > 0 and step.view_records[2] > 0
        if groups:
            step.seg_groups = groups
            step._size_records()
        step.run()
        step.check()
        res.append(([c.clone() for c in step.color], {k: g.clone() for k, g in step.grads.items()}))
    for col, g in res[1:]:
        for a, b in zip(col, res[0][0]):
            assert torch.equal(a, b)
        for k in g:
            assert_close_rel(g[k].cpu().numpy(), res[0][1][k].cpu().numpy(), 1e-5, k)
