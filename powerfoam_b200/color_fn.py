"""Spherical-Voronoi texel colour, mirroring powerfoam/color_fn.py.

``SphericalVoronoi(args, device, attr_dtype)`` keeps the reference's
constructor (``args.sv_dof``), ``compute_fov_cos_cutoff``, ``forward(points,
camera, att_sites, att_values, att_temps)`` through the autograd function
``SphericalVoronoiGradFn`` and its gradients (the site axes, values and
temperatures; none for the points, whose gradient the reference disables).
The kernels are pf_sv_forward / pf_sv_backward.
"""

import math

import torch

from . import _lib

# Fixed angular buffer (radians) added beyond the camera frustum diagonal
_FOV_BUFFER_RAD = math.radians(10.0)


class SphericalVoronoiGradFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, spherical_voronoi, points, camera, att_sites, att_values, att_temps):
        fov_cos_cutoff = getattr(camera, "fov_cos_cutoff", None)
        if fov_cos_cutoff is None:
            fov_cos_cutoff = spherical_voronoi.fov_cos_cutoff
        return spherical_voronoi._forward(ctx, points, camera, att_sites, att_values, att_temps, fov_cos_cutoff)

    @staticmethod
    def backward(ctx, *args):
        return ctx.spherical_voronoi._backward(ctx, *args)


def _vec3(t):
    return (_lib.ctypes.c_float * 3)(*[float(v) for v in t.detach().float().cpu().tolist()])


class SphericalVoronoi:
    fov_cos_cutoff = None

    @staticmethod
    def compute_fov_cos_cutoff(camera):
        """color_fn.py:28-36."""
        K = camera.intrinsics_matrix()
        fx, fy = K[0, 0], K[1, 1]
        cx, cy = K[0, 2], K[1, 2]
        x_max = max(float(cx), float(camera.width) - float(cx)) / float(fx)
        y_max = max(float(cy), float(camera.height) - float(cy)) / float(fy)
        tan_theta = float((x_max**2 + y_max**2) ** 0.5 * 1.1)
        return 1.0 / ((1.0 + tan_theta**2) ** 0.5)

    def __init__(self, args, device, attr_dtype="float"):
        self.device = torch.device(device)
        self.args = args
        self.sv_dof = args.sv_dof
        if attr_dtype == "float":
            self.tscalar = torch.float32
        elif attr_dtype == "half":
            self.tscalar = torch.float16
        else:
            raise ValueError(f"Unsupported attribute dtype: {attr_dtype}")
        _lib.load()

    def _camera_frame(self, camera):
        """Origin, unit forward and the cone cutoff of the frustum diagonal
        plus 10 degrees (color_fn.py:204-214)."""
        forward = torch.cross(camera.up, camera.right, dim=-1)
        forward = forward / torch.norm(forward, dim=-1, keepdim=True)
        right_norm = float(torch.linalg.norm(camera.right).item())
        up_norm = float(torch.linalg.norm(camera.up).item())
        tan_diag = math.sqrt(right_norm**2 + up_norm**2)
        return camera.eye, forward, math.cos(math.atan(tan_diag) + _FOV_BUFFER_RAD)

    def _attrs(self, att_sites, att_values, att_temps):
        return [a.detach().to(self.tscalar).contiguous() for a in (att_sites, att_values, att_temps)]

    def _forward(self, grad_ctx, points, camera, att_sites, att_values, att_temps, fov_cos_cutoff):
        n = points.shape[0]
        pts = points.detach().float().contiguous()
        sites, vals, temps = self._attrs(att_sites, att_values, att_temps)
        values_out = torch.empty(n, 3, device=self.device, dtype=self.tscalar)
        weights_sum_out = torch.empty(n, device=self.device, dtype=self.tscalar)
        origin, forward, cutoff = self._camera_frame(camera)
        _lib.call("pf_sv_forward", _lib.ptr(pts), _vec3(origin), _vec3(forward), float(cutoff), _lib.ptr(sites),
                  _lib.ptr(vals), _lib.ptr(temps), n, self.sv_dof, int(self.tscalar == torch.float16),
                  _lib.ptr(values_out), _lib.ptr(weights_sum_out), _lib.stream_ptr())
        grad_ctx.spherical_voronoi = self
        grad_ctx.fov_cos_cutoff = cutoff
        grad_ctx.frame = (origin.detach(), forward.detach())
        grad_ctx.save_for_backward(pts, sites, vals, temps, values_out, weights_sum_out)
        return values_out

    def forward(self, points, camera, att_sites, att_values, att_temps):
        return SphericalVoronoiGradFn.apply(self, points, camera, att_sites, att_values, att_temps)

    def _backward(self, grad_ctx, grad_values):
        pts, sites, vals, temps, values_in, weights_sum_in = grad_ctx.saved_tensors
        origin, forward = grad_ctx.frame
        g = grad_values.detach().to(self.tscalar).contiguous()
        gs = torch.empty_like(sites)
        gv = torch.empty_like(vals)
        gt = torch.empty_like(temps)
        _lib.call("pf_sv_backward", _lib.ptr(pts), _vec3(origin), _vec3(forward), float(grad_ctx.fov_cos_cutoff),
                  _lib.ptr(sites), _lib.ptr(vals), _lib.ptr(temps), _lib.ptr(weights_sum_in), _lib.ptr(values_in),
                  _lib.ptr(g), pts.shape[0], self.sv_dof, int(self.tscalar == torch.float16), _lib.ptr(gs),
                  _lib.ptr(gv), _lib.ptr(gt), _lib.stream_ptr())
        return None, None, None, gs, gv, gt
