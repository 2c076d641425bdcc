"""ctypes front end of the CPU oracle (oracle/pf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.  Arrays are numpy;
every function mirrors one reference kernel (see pf_oracle.c for citations).
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

F32 = np.float32


class OrcCamera(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("right", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("width", ctypes.c_int32), ("height", ctypes.c_int32)]


def build(force=False):
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "pf_oracle.c")):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.c_void_p)


def camera(eye, right, up, width, height):
    c = OrcCamera()
    for i in range(3):
        c.eye[i] = float(eye[i])
        c.right[i] = float(right[i])
        c.up[i] = float(up[i])
    c.width = int(width)
    c.height = int(height)
    return c


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _fn(name, prec):
    return getattr(lib(), f"{name}_{prec}")


def bin(cam, spheres, tile_width=8, prec="f32"):
    """Sorted (key, prim) pairs, per-tile offsets and per-prim tile counts."""
    spheres = _c(spheres, F32)
    N = spheres.shape[0]
    T = (1 + (cam.height - 1) // tile_width) * (1 + (cam.width - 1) // tile_width)
    n = ctypes.c_int64(0)
    counts = np.zeros(N, np.int32)
    offs = np.zeros(T + 1, np.int64)
    f = _fn("orc_bin", prec)
    f(ctypes.byref(cam), _p(spheres), ctypes.c_int64(N), ctypes.c_int(tile_width), ctypes.c_int64(0), None, None,
      _p(offs), _p(counts), ctypes.byref(n))
    keys = np.zeros(max(n.value, 1), np.int64)
    prims = np.zeros(max(n.value, 1), np.int32)
    rc = f(ctypes.byref(cam), _p(spheres), ctypes.c_int64(N), ctypes.c_int(tile_width), ctypes.c_int64(n.value),
           _p(keys), _p(prims), _p(offs), _p(counts), ctypes.byref(n))
    assert rc == 0
    return keys[: n.value], prims[: n.value], offs, counts


def f2h(x):
    """float32 -> float16 bits, round to nearest even."""
    f = lib().orc_f2h_f32
    f.restype = ctypes.c_uint16
    return np.array([f(ctypes.c_float(float(v))) for v in np.asarray(x, F32).ravel()], np.uint16)


def prefetch_adjacency(spheres, adj, adj_off):
    spheres = _c(spheres, F32)
    adj = _c(adj, np.int32)
    adj_off = _c(adj_off, np.int32)
    out = np.zeros((adj.shape[0], 4), np.uint16)
    lib().orc_prefetch_adjacency_f32(_p(spheres), _p(adj), _p(adj_off), ctypes.c_int64(spheres.shape[0]), _p(out))
    return out


def power_adjacency_diff(points, radii, adj, adj_off):
    points = _c(points, F32)
    radii = _c(radii, F32)
    adj = _c(adj, np.int32)
    adj_off = _c(adj_off, np.int32)
    out = np.zeros((adj.shape[0], 4), np.uint16)
    lib().orc_power_adjacency_diff_f32(_p(points), _p(radii), _p(adj), _p(adj_off),
                                       ctypes.c_int64(points.shape[0]), _p(out))
    return out


def _cam_args(cam, ray_maps, name, prec):
    """(function, leading camera arguments): the generic-camera variant takes
    the ray maps (H,W,6) after the camera."""
    if ray_maps is None:
        return _fn(name, prec), [ctypes.byref(cam)]
    rm = _c(ray_maps, F32)
    return _fn(name + "_generic", prec), [ctypes.byref(cam), _p(rm), rm]


def bin_generic(cam, ray_maps, spheres, tile_width=8, prec="f32"):
    """Generic-camera binning through the cone hierarchy: sorted (key, prim)
    pairs, per-tile offsets, per-prim tile counts and the cones (n, 4)."""
    spheres = _c(spheres, F32)
    rm = _c(ray_maps, F32)
    N = spheres.shape[0]
    T = (1 + (cam.height - 1) // tile_width) * (1 + (cam.width - 1) // tile_width)
    n = ctypes.c_int64(0)
    nc = ctypes.c_int64(0)
    counts = np.zeros(N, np.int32)
    offs = np.zeros(T + 1, np.int64)
    R = np.float64 if prec == "f64" else F32
    f = _fn("orc_bin_generic", prec)
    f(ctypes.byref(cam), _p(rm), _p(spheres), ctypes.c_int64(N), ctypes.c_int(tile_width), ctypes.c_int64(0), None,
      None, _p(offs), _p(counts), ctypes.byref(n), None, ctypes.byref(nc))
    keys = np.zeros(max(n.value, 1), np.int64)
    prims = np.zeros(max(n.value, 1), np.int32)
    cones = np.zeros((nc.value, 4), R)
    rc = f(ctypes.byref(cam), _p(rm), _p(spheres), ctypes.c_int64(N), ctypes.c_int(tile_width),
           ctypes.c_int64(n.value), _p(keys), _p(prims), _p(offs), _p(counts), ctypes.byref(n), _p(cones),
           ctypes.byref(nc))
    assert rc == 0
    return keys[: n.value], prims[: n.value], offs, counts, cones


def raster_forward(cam, tile_width, spheres, nsigmas, sites, rgbh, adj, adj_off, adj_diff, tile_offsets,
                   tile_prims, depth_q=None, ray_gt=None, thr=1e-3, return_point_err=False, surface=False,
                   prec="f32", ray_maps=None):
    """ray_maps (H,W,6): per-pixel origin and direction (generic camera)."""
    N = spheres.shape[0]
    S = sites.shape[1]
    H, W = cam.height, cam.width
    T = tile_offsets.shape[0] - 1
    Q = 0 if depth_q is None else depth_q.shape[-1]
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbh, F32), _c(adj, np.int32),
            _c(adj_off, np.int32), None if adj_diff is None else _c(adj_diff, np.uint16), _c(tile_offsets, np.int64),
            _c(tile_prims, np.int32)]
    dq = None if depth_q is None else _c(depth_q, F32)
    gt = None if ray_gt is None else _c(ray_gt, F32)
    R = np.float64 if prec == "f64" else F32
    out = dict(color=np.zeros((H, W, 3), R), log_t=np.zeros((H, W), R), normal_distance=np.zeros((H, W), R),
               normal=np.zeros((H, W, 3), R), quantile_depths=-np.ones((H, W, max(Q, 1)), R),
               contrib=np.zeros(N, R), point_err=np.zeros(N, R), early_stop=np.zeros(T, np.int32),
               err=np.zeros((H, W), R) if surface else None)
    fn, lead = _cam_args(cam, ray_maps, "orc_raster_forward", prec)
    rc = fn(
        *lead[:2], ctypes.c_int(tile_width), ctypes.c_int64(N), *[_p(a) for a in args[:4]], ctypes.c_int(S),
        *[_p(a) for a in args[4:]], _p(dq), ctypes.c_int(Q), _p(gt), ctypes.c_float(thr),
        ctypes.c_int(int(return_point_err)), _p(out["color"]), _p(out["log_t"]), _p(out["normal_distance"]),
        _p(out["normal"]), _p(out["quantile_depths"]), _p(out["err"]), _p(out["contrib"]), _p(out["point_err"]),
        _p(out["early_stop"]))
    assert rc == 0
    if Q == 0:
        out["quantile_depths"] = None
    return out


def raster_backward(cam, tile_width, spheres, nsigmas, sites, rgbh, adj, adj_off, adj_diff, tile_offsets,
                    tile_prims, early_stop, log_t, grad_color, grad_log_t, grad_nd, grad_normal, grad_contrib,
                    depth_q=None, grad_qd=None, prec="f32", ray_maps=None):
    N = spheres.shape[0]
    S = sites.shape[1]
    Q = 0 if depth_q is None else depth_q.shape[-1]
    g = dict(spheres=np.zeros((N, 4), F32), nsigmas=np.zeros((N, 4), F32), texel_sites=np.zeros((N, S, 3), F32),
             texel_rgb=np.zeros((N, S, 3), F32), texel_height=np.zeros((N, S), F32))
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbh, F32)]
    args2 = [_c(adj, np.int32), _c(adj_off, np.int32), None if adj_diff is None else _c(adj_diff, np.uint16),
             _c(tile_offsets, np.int64), _c(tile_prims, np.int32), _c(early_stop, np.int32)]
    dq = None if depth_q is None else _c(depth_q, F32)
    gq = None if grad_qd is None else _c(grad_qd, F32)
    ins = [_c(log_t, F32), _c(grad_color, F32), _c(grad_log_t, F32), _c(grad_nd, F32), _c(grad_normal, F32)]
    adj_diff = None if adj_diff is None else _c(adj_diff, np.uint16)
    fn, lead = _cam_args(cam, ray_maps, "orc_raster_backward", prec)
    rc = fn(
        *lead[:2], ctypes.c_int(tile_width), ctypes.c_int64(N), *[_p(a) for a in args], ctypes.c_int(S),
        *[_p(a) for a in args2], _p(dq), ctypes.c_int(Q), *[_p(a) for a in ins], _p(gq),
        _p(_c(grad_contrib, F32)), _p(g["spheres"]), _p(g["nsigmas"]), _p(g["texel_sites"]), _p(g["texel_rgb"]),
        _p(g["texel_height"]))
    assert rc == 0
    return g


def raster_benchmark(cam, tile_width, spheres, nsigmas, sites, rgbs, heights, adj_off, adj_diff_pm, tile_offsets,
                     tile_prims, thr=1e-3, prec="f32"):
    H, W = cam.height, cam.width
    S = sites.shape[1]
    color = np.zeros((H, W, 3), F32)
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbs, F32), _c(heights, F32)]
    rc = _fn("orc_raster_benchmark", prec)(
        ctypes.byref(cam), ctypes.c_int(tile_width), *[_p(a) for a in args], ctypes.c_int(S),
        _p(_c(adj_off, np.int32)), _p(_c(adj_diff_pm, np.uint16)), _p(_c(tile_offsets, np.int64)),
        _p(_c(tile_prims, np.int32)), ctypes.c_float(thr), _p(color))
    assert rc == 0
    return color


def raster_visualize(cam, tile_width, spheres, nsigmas, sites, rgbs, heights, adj_off, adj_diff, tile_offsets,
                     tile_prims, thr=1e-3, max_intersections=1024, depth_quantile=0.5, bkgd=(0.0, 0.0, 0.0),
                     prec="f32"):
    H, W = cam.height, cam.width
    S = sites.shape[1]
    out = dict(color=np.zeros((H, W, 3), F32), depth=np.zeros((H, W), F32), normal=np.zeros((H, W, 3), F32),
               alpha=np.zeros((H, W), F32), intersections=np.zeros((H, W), np.int32))
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbs, F32), _c(heights, F32)]
    rc = _fn("orc_raster_visualize", prec)(
        ctypes.byref(cam), ctypes.c_int(tile_width), *[_p(a) for a in args], ctypes.c_int(S),
        _p(_c(adj_off, np.int32)), _p(_c(adj_diff, np.uint16)), _p(_c(tile_offsets, np.int64)),
        _p(_c(tile_prims, np.int32)), ctypes.c_float(thr), ctypes.c_int(max_intersections),
        ctypes.c_float(depth_quantile), _p(np.asarray(bkgd, F32)), _p(out["color"]), _p(out["depth"]),
        _p(out["normal"]), _p(out["alpha"]), _p(out["intersections"]))
    assert rc == 0
    return out


def trace_forward(cam, spheres, nsigmas, sites, rgbs, heights, adj, adj_off, adj_diff_pm, start_idx=0,
                  start_cells=None, thr=1e-3, max_steps=1 << 16, depth_quantile=0.5, visit_cap=0, prec="f32"):
    H, W = cam.height, cam.width
    S = sites.shape[1]
    R = np.float64 if prec == "f64" else F32
    out = dict(color=np.zeros((H, W, 3), R), log_t=np.zeros((H, W), R), depth=np.zeros((H, W), R),
               normal=np.zeros((H, W, 3), R), depth_seg=np.zeros((H, W), np.int32),
               depth_sigma=np.zeros((H, W), R), visit_count=np.zeros((H, W), np.int32),
               status=np.zeros((H, W), np.int32))
    vl = np.full((H, W, max(visit_cap, 1)), -1, np.int32) if visit_cap else None
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbs, F32), _c(heights, F32)]
    sc = None if start_cells is None else _c(start_cells, np.int32)
    rc = _fn("orc_trace_forward", prec)(
        ctypes.byref(cam), *[_p(a) for a in args], ctypes.c_int(S), _p(_c(adj, np.int32)),
        _p(_c(adj_off, np.int32)), _p(None if adj_diff_pm is None else _c(adj_diff_pm, np.uint16)),
        ctypes.c_int32(start_idx), _p(sc), ctypes.c_float(thr), ctypes.c_int(max_steps),
        ctypes.c_float(depth_quantile), _p(out["color"]),
        _p(out["log_t"]), _p(out["depth"]), _p(out["normal"]), _p(out["depth_seg"]), _p(out["depth_sigma"]),
        _p(vl), ctypes.c_int(visit_cap), _p(out["visit_count"]), _p(out["status"]))
    out["rc"] = rc
    out["visits"] = vl
    return out


def trace_forward_pixels(cam, spheres, nsigmas, sites, rgbs, heights, adj, adj_off, adj_diff_pm, pixels,
                         start_idx=0, start_cells=None, thr=1e-3, max_steps=1 << 16, depth_quantile=0.5,
                         visit_cap=0, prec="f32"):
    """trace_forward for the camera pixels listed in ``pixels`` (row-major
    indices); every output is indexed like ``pixels``."""
    pixels = _c(pixels, np.int64)
    n = pixels.shape[0]
    S = sites.shape[1]
    R = np.float64 if prec == "f64" else F32
    out = dict(color=np.zeros((n, 3), R), log_t=np.zeros(n, R), depth=np.zeros(n, R), normal=np.zeros((n, 3), R),
               depth_seg=np.zeros(n, np.int32), depth_sigma=np.zeros(n, R), visit_count=np.zeros(n, np.int32),
               status=np.zeros(n, np.int32))
    vl = np.full((n, max(visit_cap, 1)), -1, np.int32) if visit_cap else None
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbs, F32), _c(heights, F32)]
    sc = None if start_cells is None else _c(start_cells, np.int32)
    rc = _fn("orc_trace_forward_pixels", prec)(
        ctypes.byref(cam), *[_p(a) for a in args], ctypes.c_int(S), _p(_c(adj, np.int32)),
        _p(_c(adj_off, np.int32)), _p(None if adj_diff_pm is None else _c(adj_diff_pm, np.uint16)),
        ctypes.c_int32(start_idx), _p(sc), ctypes.c_float(thr), ctypes.c_int(max_steps),
        ctypes.c_float(depth_quantile), _p(pixels), ctypes.c_int64(n), _p(out["color"]), _p(out["log_t"]),
        _p(out["depth"]), _p(out["normal"]), _p(out["depth_seg"]), _p(out["depth_sigma"]), _p(vl),
        ctypes.c_int(visit_cap), _p(out["visit_count"]), _p(out["status"]))
    out["rc"] = rc
    out["visits"] = vl
    return out


def trace_labels(cam, spheres, nsigmas, sites, rgbs, heights, adj, adj_off, adj_diff_pm, start_idx=0,
                 start_cells=None, thr=1e-3, max_steps=1 << 16, label_thr=0.99):
    """Proposal-network labels of every camera ray: entry t / cell / step of
    the first cell after which the transmittance is below label_thr (-1 when
    never), with the colour and the number of cells walked."""
    H, W = cam.height, cam.width
    S = sites.shape[1]
    out = dict(color=np.zeros((H, W, 3), F32), label_t=np.zeros((H, W), F32),
               label_cell=np.zeros((H, W), np.int32), label_step=np.zeros((H, W), np.int32),
               visit_count=np.zeros((H, W), np.int32), status=np.zeros((H, W), np.int32))
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbs, F32), _c(heights, F32)]
    sc = None if start_cells is None else _c(start_cells, np.int32)
    rc = lib().orc_trace_labels_f32(
        ctypes.byref(cam), *[_p(a) for a in args], ctypes.c_int(S), _p(_c(adj, np.int32)),
        _p(_c(adj_off, np.int32)), _p(_c(adj_diff_pm, np.uint16)), ctypes.c_int32(start_idx), _p(sc),
        ctypes.c_float(thr), ctypes.c_int(max_steps), ctypes.c_float(label_thr), _p(out["color"]),
        _p(out["label_t"]), _p(out["label_cell"]), _p(out["label_step"]), _p(out["visit_count"]),
        _p(out["status"]))
    out["rc"] = rc
    return out


def start_cell(points, radii, eye):
    f = lib().orc_start_cell_f32
    f.restype = ctypes.c_int32
    points = _c(points, F32)
    return int(f(_p(points), _p(_c(radii, F32)), ctypes.c_int64(points.shape[0]), _p(np.asarray(eye, F32))))


def sh_texel_rgb(points, sh, eye, S=8):
    points = _c(points, F32)
    N = points.shape[0]
    out = np.zeros((N, S, 3), F32)
    lib().orc_sh_texel_rgb_f32(_p(points), _p(_c(sh, F32)), ctypes.c_int64(N), ctypes.c_int(S),
                               _p(np.asarray(eye, F32)), _p(out))
    return out


def sh_texel_rgb_backward(points, sh, eye, grad_texel_rgb, grad_sh=None):
    """Adds the coefficient gradient of sh_texel_rgb into grad_sh (N,16,3)."""
    points = _c(points, F32)
    N = points.shape[0]
    g = _c(grad_texel_rgb, F32)
    out = np.zeros((N, 16, 3), F32) if grad_sh is None else grad_sh
    lib().orc_sh_texel_rgb_backward_f32(_p(points), _p(_c(sh, F32)), ctypes.c_int64(N), ctypes.c_int(g.shape[1]),
                                        _p(np.asarray(eye, F32)), _p(g), _p(out))
    return out


def interpenetration(spheres, adj, adj_off, prec="f32", rows=None):
    """areas (N,) of interpenetration_kernel (geometry.py:88-117); with
    ``rows`` only the first rows are evaluated (the rest stay 0)."""
    sph = _c(spheres, F32)
    N = sph.shape[0]
    R = np.float64 if prec == "f64" else F32
    out = np.zeros(N, R)
    getattr(lib(), f"orc_interpenetration_{prec}")(_p(sph), _p(_c(adj, np.int32)), _p(_c(adj_off, np.int32)),
                                                   ctypes.c_int64(N if rows is None else rows), _p(out))
    return out


def interpenetration_backward(spheres, adj, adj_off, grad_areas, prec="f32", rows=None):
    """dL/dspheres (N,4) given dL/dareas (geometry.py:158-189); with ``rows``
    only the lists of the first rows are replayed."""
    sph = _c(spheres, F32)
    N = sph.shape[0]
    R = np.float64 if prec == "f64" else F32
    out = np.zeros((N, 4), R)
    getattr(lib(), f"orc_interpenetration_backward_{prec}")(_p(sph), _p(_c(adj, np.int32)), _p(_c(adj_off, np.int32)),
                                                            ctypes.c_int64(N if rows is None else rows),
                                                            _p(_c(grad_areas, F32)), _p(out))
    return out


def sv_forward(points, origin, forward, cutoff, sites, values, temps, prec="f32"):
    """Spherical-Voronoi colour and weight sum (color_fn.py:54-101)."""
    pts = _c(points, F32)
    N = pts.shape[0]
    dof = sites.shape[0]
    R = np.float64 if prec == "f64" else F32
    v = np.zeros((N, 3), R)
    w = np.zeros(N, R)
    getattr(lib(), f"orc_sv_forward_{prec}")(_p(pts), _p(np.asarray(origin, F32)), _p(np.asarray(forward, F32)),
                                             ctypes.c_float(cutoff), _p(_c(sites, F32)), _p(_c(values, F32)),
                                             _p(_c(temps, F32)), ctypes.c_int64(N), ctypes.c_int(dof), _p(v), _p(w))
    return v, w


def sv_backward(points, origin, forward, cutoff, sites, values, temps, wsum, value, grad_value, prec="f32"):
    """Site gradients of sv_forward (color_fn.py:105-182)."""
    pts = _c(points, F32)
    N = pts.shape[0]
    dof = sites.shape[0]
    R = np.float64 if prec == "f64" else F32
    gs = np.zeros((dof, N, 3), R)
    gv = np.zeros((dof, N, 3), R)
    gt = np.zeros((dof, N), R)
    getattr(lib(), f"orc_sv_backward_{prec}")(_p(pts), _p(np.asarray(origin, F32)), _p(np.asarray(forward, F32)),
                                              ctypes.c_float(cutoff), _p(_c(sites, F32)), _p(_c(values, F32)),
                                              _p(_c(temps, F32)), _p(_c(wsum, F32)), _p(_c(value, F32)),
                                              _p(_c(grad_value, F32)), ctypes.c_int64(N), ctypes.c_int(dof), _p(gs),
                                              _p(gv), _p(gt))
    return gs, gv, gt


def num_threads():
    return int(lib().orc_num_threads_f32())


def trace_backward(cam, spheres, nsigmas, sites, rgbs, heights, adj, adj_off, adj_diff_pm, fwd, g_color=None,
                   g_log_t=None, g_depth=None, g_normal=None, start_idx=0, start_cells=None, thr=1e-3,
                   max_steps=1 << 16, depth_quantile=0.5, prec="f32"):
    """Exact adjoint of trace_forward (see pf_oracle.c).  ``fwd`` is the dict
    returned by trace_forward with the same arguments."""
    N = spheres.shape[0]
    S = sites.shape[1]
    R = np.float64 if prec == "f64" else F32
    g = dict(spheres=np.zeros((N, 4), F32), nsigmas=np.zeros((N, 4), F32), texel_sites=np.zeros((N, S, 3), F32),
             texel_rgb=np.zeros((N, S, 3), F32), texel_height=np.zeros((N, S), F32))
    args = [_c(spheres, F32), _c(nsigmas, F32), _c(sites, F32), _c(rgbs, F32), _c(heights, F32)]
    sc = None if start_cells is None else _c(start_cells, np.int32)
    opt = lambda a: None if a is None else _c(a, F32)
    rc = _fn("orc_trace_backward", prec)(
        ctypes.byref(cam), *[_p(a) for a in args], ctypes.c_int(S), _p(_c(adj, np.int32)), _p(_c(adj_off, np.int32)),
        _p(None if adj_diff_pm is None else _c(adj_diff_pm, np.uint16)), ctypes.c_int32(start_idx), _p(sc),
        ctypes.c_float(thr),
        ctypes.c_int(max_steps), ctypes.c_float(depth_quantile), _p(_c(fwd["color"], R)),
        _p(_c(fwd["normal"], R)), _p(_c(fwd["depth_seg"], np.int32)), _p(_c(fwd["depth_sigma"], R)),
        _p(opt(g_color)), _p(opt(g_log_t)), _p(opt(g_depth)), _p(opt(g_normal)), _p(g["spheres"]),
        _p(g["nsigmas"]), _p(g["texel_sites"]), _p(g["texel_rgb"]), _p(g["texel_height"]))
    assert rc == 0
    return g


def cech_adjacency(points, radii):
    """Čech adjacency of bvh.py:7-69 / build_cech_complex (bvh.py:96-123):
    (adjacency int32 (E), offsets int32 (N+1)), lists ascending."""
    pts = _c(points, F32)
    rad = _c(radii, F32)
    N = pts.shape[0]
    off = np.zeros(N + 1, np.int32)
    ne = ctypes.c_int64(0)
    f = lib().orc_cech_adjacency_f32
    assert f(_p(pts), _p(rad), ctypes.c_int64(N), _p(off), None, ctypes.byref(ne)) == 0
    adj = np.zeros(max(ne.value, 1), np.int32)
    assert f(_p(pts), _p(rad), ctypes.c_int64(N), _p(off), _p(adj), ctypes.byref(ne)) == 0
    return adj[: ne.value], off
