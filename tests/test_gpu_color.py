"""Spherical-Voronoi texel colour (powerfoam/color_fn.py) on the GPU against
the golden run of the reference's kernels and the oracle: float32 colours
within 1e-6, gradients within 1e-5 (relative); float16 attributes within
float16 rounding; the autograd mirror's returns."""

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from powerfoam_b200 import _lib
from tests.helpers import assert_close_rel, max_abs, torch_cam

pytestmark = pytest.mark.gpu


def _v3(a):
    return (_lib.ctypes.c_float * 3)(*[float(x) for x in a])


def _run(g, half=False):
    dt = torch.float16 if half else torch.float32
    d = "cuda"
    pts = torch.from_numpy(g["points"]).to(d)
    sites, values, temps = (torch.from_numpy(g[k]).to(d, dt).contiguous() for k in ("sites", "values", "temps"))
    n, dof = pts.shape[0], sites.shape[0]
    v = torch.empty(n, 3, device=d, dtype=dt)
    w = torch.empty(n, device=d, dtype=dt)
    _lib.call("pf_sv_forward", _lib.ptr(pts), _v3(g["origin"]), _v3(g["forward"]), float(g["cutoff"]),
              _lib.ptr(sites), _lib.ptr(values), _lib.ptr(temps), n, dof, int(half), _lib.ptr(v), _lib.ptr(w),
              _lib.stream_ptr())
    gv_in = torch.from_numpy(g["grad_value"]).to(d, dt).contiguous()
    gs, gvv, gt = torch.full_like(sites, 7), torch.full_like(values, 7), torch.full_like(temps, 7)
    _lib.call("pf_sv_backward", _lib.ptr(pts), _v3(g["origin"]), _v3(g["forward"]), float(g["cutoff"]),
              _lib.ptr(sites), _lib.ptr(values), _lib.ptr(temps), _lib.ptr(w), _lib.ptr(v), _lib.ptr(gv_in), n, dof,
              int(half), _lib.ptr(gs), _lib.ptr(gvv), _lib.ptr(gt), _lib.stream_ptr())
    torch.cuda.synchronize()
    return [t.float().cpu().numpy() for t in (v, w, gs, gvv, gt)]


def test_sv_float_matches_golden_and_oracle(golden):
    g = golden("sv_small")
    v, w, gs, gv, gt = _run(g)
    assert max_abs(v, g["value"]) <= 1e-6
    assert_close_rel(w, g["wsum"], 1e-6, "weight sum")
    for a, k in [(gs, "grad_sites"), (gv, "grad_values"), (gt, "grad_temps")]:
        assert_close_rel(a, g[k], 1e-5, k)
    args = (g["points"], g["origin"], g["forward"], float(g["cutoff"]), g["sites"], g["values"], g["temps"])
    # exp differs between CUDA and the host library by an ulp or two
    ov, ow = orc.sv_forward(*args)
    assert max_abs(v, ov) <= 1e-6
    assert_close_rel(w, ow, 1e-6, "weight sum")
    assert np.array_equal(w == 0, ow == 0)
    ogs, ogv, ogt = orc.sv_backward(*args, ow, ov, g["grad_value"])
    for a, b, k in [(gs, ogs, "sites"), (gv, ogv, "values"), (gt, ogt, "temps")]:
        assert_close_rel(a, b, 1e-5, k)


def test_sv_half_attributes(golden):
    g = golden("sv_small")
    v, w, gs, gv, gt = _run(g, half=True)
    assert max_abs(v, g["value"]) <= 4e-3
    assert_close_rel(w, g["wsum"], 4e-3, "weight sum")
    assert_close_rel(gv, g["grad_values"], 2e-2, "grad values")


def test_sv_autograd_mirror(golden):
    from powerfoam_b200.color_fn import SphericalVoronoi

    g = golden("sv_small")
    cam = torch_cam(dict(eye=g["cam_eye"], right=g["cam_right"], up=g["cam_up"], width=int(g["width"]),
                         height=int(g["height"])))

    class A:
        sv_dof = g["sites"].shape[0]

    sv = SphericalVoronoi(A(), "cuda")
    origin, forward, cutoff = sv._camera_frame(cam)
    sites, values, temps = (torch.from_numpy(g[k]).cuda().requires_grad_(True) for k in ("sites", "values", "temps"))
    pts = torch.from_numpy(g["points"]).cuda()
    out = sv.forward(pts, cam, sites, values, temps)
    gval = torch.from_numpy(g["grad_value"]).cuda()
    (out * gval).sum().backward()
    o = origin.cpu().numpy()
    f = forward.cpu().numpy()
    ov, ow = orc.sv_forward(g["points"], o, f, float(np.float32(cutoff)), g["sites"], g["values"], g["temps"])
    assert max_abs(out.detach().cpu().numpy(), ov) <= 1e-6
    ogs, ogv, ogt = orc.sv_backward(g["points"], o, f, float(np.float32(cutoff)), g["sites"], g["values"],
                                    g["temps"], ow, ov, g["grad_value"])
    assert_close_rel(sites.grad.cpu().numpy(), ogs, 1e-5, "sites")
    assert_close_rel(values.grad.cpu().numpy(), ogv, 1e-5, "values")
    assert_close_rel(temps.grad.cpu().numpy(), ogt, 1e-5, "temps")
    assert 0 < (ow == 0).sum() < ow.shape[0]  # the camera cone cuts the cloud
