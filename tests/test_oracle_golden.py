"""The CPU oracle against golden vectors produced by executing the
reference's own kernel source (tests/golden/make_golden.py)."""

import numpy as np
import pytest

from oracle import oracle as orc
from tests.helpers import assert_close_rel, max_abs, packed

RASTER_CASES = ["raster_small", "raster_edge", "raster_dense"]


def _cam(g):
    return orc.camera(g["cam_eye"], g["cam_right"], g["cam_up"], g["width"], g["height"])


def test_binning_bit_exact_large(golden):
    g = golden("bin_large")
    keys, prims, offs, _ = orc.bin(_cam(g), g["spheres"], 8)
    assert np.array_equal(keys, g["sort_keys"])
    assert np.array_equal(prims, g["tile_prims"])
    assert np.array_equal(offs, g["tile_offsets"])


@pytest.mark.parametrize("case", RASTER_CASES)
def test_binning_and_encodings(golden, case):
    g = golden(case)
    sph, _, _ = packed(g)
    keys, prims, offs, _ = orc.bin(_cam(g), sph, 8)
    assert np.array_equal(keys, g["sort_keys"])
    assert np.array_equal(prims, g["tile_prims"])
    assert np.array_equal(offs, g["tile_offsets"])
    assert np.array_equal(orc.prefetch_adjacency(sph, g["adjacency"], g["adjacency_offsets"]), g["adjacency_diff"])
    pm = orc.power_adjacency_diff(g["points"], g["radii"], g["adjacency"], g["adjacency_offsets"])
    assert np.array_equal(pm, g["adjacency_diff_pm"])


@pytest.mark.parametrize("case", RASTER_CASES)
def test_forward(golden, case):
    g = golden(case)
    sph, nsig, rgbh = packed(g)
    o = orc.raster_forward(_cam(g), 8, sph, nsig, g["texel_sites"], rgbh, g["adjacency"], g["adjacency_offsets"],
                           g["adjacency_diff"], g["tile_offsets"], g["tile_prims"], g["depth_quantiles"], g["ray_gt"],
                           float(g["thr"]), True)
    assert np.array_equal(o["early_stop"], g["early_stop"])
    for k in ["color", "normal_distance", "normal", "quantile_depths"]:
        assert max_abs(o[k], g[k]) <= 1e-5, k
    # log transmittance reaches -600 in opaque tiles (float32 ulp 6e-5 there):
    # the returned opacity 1 - exp(log_t) within 1e-5, log_t itself relative
    assert max_abs(1 - np.exp(o["log_t"]), 1 - np.exp(g["log_t"])) <= 1e-5
    assert_close_rel(o["log_t"], g["log_t"], 1e-5, "log_t")
    for k in ["contrib", "point_err"]:
        assert_close_rel(o[k], g[k], 1e-5, k)


@pytest.mark.parametrize("case", RASTER_CASES)
def test_backward(golden, case):
    g = golden(case)
    sph, nsig, rgbh = packed(g)
    gr = orc.raster_backward(_cam(g), 8, sph, nsig, g["texel_sites"], rgbh, g["adjacency"], g["adjacency_offsets"],
                             g["adjacency_diff"], g["tile_offsets"], g["tile_prims"], g["early_stop"], g["log_t"],
                             g["grad_color"], g["grad_log_t"], g["grad_normal_distance"], g["grad_normal"],
                             g["grad_contrib"], g["depth_quantiles"], g["grad_quantile_depths"])
    for a, b in [("spheres", "spheres_grad"), ("nsigmas", "nsigmas_grad"), ("texel_sites", "texel_sites_grad"),
                 ("texel_rgb", "texel_rgb_grad"), ("texel_height", "texel_height_grad")]:
        assert_close_rel(gr[a], g[b], 1e-4, a)


@pytest.mark.parametrize("case", RASTER_CASES)
def test_benchmark_and_viewer_paths(golden, case):
    g = golden(case)
    sph, nsig, _ = packed(g)
    c = orc.raster_benchmark(_cam(g), 8, sph, nsig, g["texel_sites"], g["texel_rgb"], g["texel_height"],
                             g["adjacency_offsets"], g["adjacency_diff_pm"], g["tile_offsets"], g["tile_prims"],
                             float(g["bench_thr"]))
    assert max_abs(c, g["bench_color"]) <= 1e-5
    v = orc.raster_visualize(_cam(g), 8, sph, nsig, g["texel_sites"], g["texel_rgb"], g["texel_height"],
                             g["adjacency_offsets"], g["adjacency_diff"], g["tile_offsets"], g["tile_prims"])
    for k in ["color", "depth", "normal", "alpha"]:
        assert max_abs(v[k], g["vis_" + k]) <= 1e-5, k
    assert np.array_equal(v["intersections"], g["vis_intersections"])


def test_tracer_cell_sequences(golden):
    g = golden("trace_small")
    sph, nsig, _ = packed(g)
    assert orc.start_cell(g["points"], g["radii"], g["cam_eye"]) == int(g["start_idx"])
    assert np.array_equal(orc.power_adjacency_diff(g["points"], g["radii"], g["adjacency"], g["adjacency_offsets"]),
                          g["adjacency_diff_pm"])
    t = orc.trace_forward(_cam(g), sph, nsig, g["texel_sites"], g["texel_rgb"], g["texel_height"], g["adjacency"],
                          g["adjacency_offsets"], g["adjacency_diff_pm"], int(g["start_idx"]), thr=float(g["thr"]),
                          visit_cap=g["visits"].shape[-1])
    assert np.array_equal(t["visit_count"], g["visit_count"])
    assert np.array_equal(t["visits"], g["visits"])
    assert max_abs(t["color"], g["color"]) <= 1e-5


def test_f16_rounding_matches_numpy():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(2000) * 10 ** rng.uniform(-9, 5, 2000),
                        [0.0, -0.0, 65504.0, 65520.0, 1e-8, 6.1e-5, np.inf, -np.inf]]).astype(np.float32)
    assert np.array_equal(orc.f2h(x), x.astype(np.float16).view(np.uint16))


# ---------------------------------------------------------------------------
# generic camera (is_pinhole=False): cone-hierarchy binning and per-pixel rays


def test_generic_binning_and_cones_bit_exact(golden):
    g = golden("raster_generic")
    sph, _, _ = packed(g)
    keys, prims, offs, _, cones = orc.bin_generic(_cam(g), g["ray_maps"], sph, 8)
    assert np.array_equal(cones.view(np.uint32), g["cones"].view(np.uint32))
    assert np.array_equal(keys, g["sort_keys"])
    assert np.array_equal(prims, g["tile_prims"])
    assert np.array_equal(offs, g["tile_offsets"])


def test_generic_forward_and_backward(golden):
    g = golden("raster_generic")
    sph, nsig, rgbh = packed(g)
    o = orc.raster_forward(_cam(g), 8, sph, nsig, g["texel_sites"], rgbh, g["adjacency"], g["adjacency_offsets"],
                           g["adjacency_diff"], g["tile_offsets"], g["tile_prims"], g["depth_quantiles"], g["ray_gt"],
                           float(g["thr"]), True, ray_maps=g["ray_maps"])
    assert np.array_equal(o["early_stop"], g["early_stop"])
    for k in ["color", "normal_distance", "normal", "quantile_depths", "log_t"]:
        assert max_abs(o[k], g[k]) <= 1e-5, k
    for k in ["contrib", "point_err"]:
        assert_close_rel(o[k], g[k], 1e-5, k)
    gr = orc.raster_backward(_cam(g), 8, sph, nsig, g["texel_sites"], rgbh, g["adjacency"], g["adjacency_offsets"],
                             g["adjacency_diff"], g["tile_offsets"], g["tile_prims"], g["early_stop"], g["log_t"],
                             g["grad_color"], g["grad_log_t"], g["grad_normal_distance"], g["grad_normal"],
                             g["grad_contrib"], g["depth_quantiles"], g["grad_quantile_depths"],
                             ray_maps=g["ray_maps"])
    for a, b in [("spheres", "spheres_grad"), ("nsigmas", "nsigmas_grad"), ("texel_sites", "texel_sites_grad"),
                 ("texel_rgb", "texel_rgb_grad"), ("texel_height", "texel_height_grad")]:
        assert_close_rel(gr[a], g[b], 1e-4, a)


# ---------------------------------------------------------------------------
# spherical-Voronoi texel colour (color_fn.py:54-184)


def test_spherical_voronoi_forward_and_backward(golden):
    g = golden("sv_small")
    args = (g["points"], g["origin"], g["forward"], float(g["cutoff"]), g["sites"], g["values"], g["temps"])
    v, w = orc.sv_forward(*args)
    assert max_abs(v, g["value"]) <= 1e-6
    assert_close_rel(w, g["wsum"], 1e-6, "weight sum")
    assert np.array_equal(w == 0, g["wsum"] == 0)  # the same points fall outside the cone
    gs, gv, gt = orc.sv_backward(*args, g["wsum"], g["value"], g["grad_value"])
    for a, k in [(gs, "grad_sites"), (gv, "grad_values"), (gt, "grad_temps")]:
        assert_close_rel(a, g[k], 1e-5, k)
