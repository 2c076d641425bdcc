"""Cell-walk ray tracer: drop-in for powerfoam/raytrace.py.

``RayTracer(args, device, attr_dtype).benchmark(...)`` keeps the reference's
signature and returns the colour image (raytrace.py:247-309).  ``trace``
exposes the extensions of the walk kernel: per-ray start cells, a step cap,
depth / normal / log transmittance and the visited-cell log.  ``forward``
is differentiable (``RayTraceGradFn``): its adjoint has no counterpart in the
reference, whose tracer is forward-only.
"""

from dataclasses import dataclass

import torch

from . import _lib

DEFAULT_MAX_STEPS = 1 << 16
# bound on the adjoint's segment records when segments_per_ray is left to the tracer
RECORD_BYTES = 4 << 30


@dataclass
class TraceResult:
    color: torch.Tensor
    log_t: torch.Tensor
    depth: torch.Tensor
    normal: torch.Tensor
    depth_seg: torch.Tensor
    depth_sigma: torch.Tensor
    visit_count: torch.Tensor
    visits: torch.Tensor = None
    status: int = 0
    records: tuple = None  # (workspace, segments_per_ray) of a recording walk


class RayTraceGradFn(torch.autograd.Function):
    """(color, log_t, depth, normal) of the walk; gradients for points, radii,
    density, normals, texel_sites, texel_rgb, texel_height."""

    @staticmethod
    def forward(ctx, tracer, camera, start, points, radii, density, normals, texel_sites, texel_rgb, texel_height,
                adjacency, adjacency_offsets, adjacency_diff, transmittance_threshold=1e-3, max_steps=None,
                depth_quantile=0.5):
        return tracer._forward(ctx, camera, start, points, radii, density, normals, texel_sites, texel_rgb,
                               texel_height, adjacency, adjacency_offsets, adjacency_diff, transmittance_threshold,
                               max_steps, depth_quantile)

    @staticmethod
    def backward(ctx, g_color, g_log_t, g_depth, g_normal):
        return ctx.tracer._backward(ctx, g_color, g_log_t, g_depth, g_normal)


class RayTracer:
    def __init__(self, args, device, attr_dtype="float"):
        self.device = torch.device(device)
        self.args = args
        if attr_dtype == "float":
            self.tscalar = torch.float32
        elif attr_dtype == "half":
            self.tscalar = torch.float16
        else:
            raise ValueError(f"Unsupported attribute dtype: {attr_dtype}")
        self.attr_dtype = attr_dtype
        self.num_texel_sites = args.num_texel_sites
        # segments per ray the adjoint records for its gradient launch (rays
        # with more are walked on by its slower resume launch; any value
        # gives the same gradients), 48 bytes per pixel each; None: 96,
        # lowered so the records stay within RECORD_BYTES
        self.segments_per_ray = None
        # the differentiable forward writes the adjoint's segment records
        # (pf_trace_forward_record), so the adjoint does not walk again; False:
        # plain forward, and the adjoint repeats the walk (pf_trace_backward)
        self.record_segments = True
        # host_sync (default True): the differentiable forward reads its status
        # word back and raises at once (step cap, bad cell index); False: the
        # forward never waits on the host (a training loop queues steps ahead),
        # the kernels raise the persistent device word ``status`` and check()
        # reports it
        self.host_sync = True
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        _lib.load()

    def check(self):
        """Raise PfError if a forward since the last check stopped a walk
        early (host_sync=False mode; one host read); clears the word."""
        st = int(self.status.item())
        if st != _lib.PF_OK:
            self.status.zero_()
            raise _lib.PfError(st, "cell walk stopped early (step cap or invalid cell index)")
        return True

    def _inputs(self, camera, start, spheres, nsig, sites, rgb, height, adjacency, adjacency_offsets,
                adjacency_diff, thr, max_steps, depth_quantile):
        inp = _lib.PfTraceInputs()
        inp.cam = camera.to_pf()
        inp.n_sites = sites.shape[1]
        inp.attr_half = int(self.attr_dtype == "half")
        inp.n_prims = spheres.shape[0]
        inp.spheres = _lib.ptr(spheres)
        inp.nsigmas = _lib.ptr(nsig)
        inp.texel_sites = _lib.ptr(sites)
        inp.texel_rgb = _lib.ptr(rgb)
        inp.texel_height = _lib.ptr(height)
        inp.adjacency = _lib.ptr(adjacency)
        inp.adjacency_offsets = _lib.ptr(adjacency_offsets)
        inp.adjacency_diff = _lib.ptr(adjacency_diff)
        if isinstance(start, torch.Tensor) and start.numel() > 1:
            inp.start_idx = 0
            inp.start_cells = _lib.ptr(start)
        else:
            inp.start_idx = int(start)
            inp.start_cells = None
        inp.transmittance_threshold = float(thr)
        inp.max_steps = int(max_steps)
        inp.depth_quantile = float(depth_quantile)
        return inp

    def _prep(self, points, radii, density, normals, texel_sites, texel_rgb, texel_height, adjacency,
              adjacency_offsets, adjacency_diff):
        spheres = torch.cat([points, radii[:, None]], dim=-1).to(torch.float32).contiguous()
        nsig = torch.cat([normals, density[:, None]], dim=-1).to(self.tscalar).contiguous()
        return (spheres, nsig, texel_sites.to(self.tscalar).contiguous(), texel_rgb.to(self.tscalar).contiguous(),
                texel_height.to(self.tscalar).contiguous(), adjacency.to(torch.int32).contiguous(),
                adjacency_offsets.to(torch.int32).contiguous(), adjacency_diff.contiguous())

    def _segments_per_ray(self, camera):
        kb = self.segments_per_ray
        if kb is None:
            slots = ((int(camera.height) + 7) // 8) * ((int(camera.width) + 7) // 8) * 64
            kb = max(1, min(96, RECORD_BYTES // (48 * slots)))
        return int(kb)

    def _records(self, inp, kb):
        """The adjoint's segment-record workspace (256-byte aligned)."""
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_trace_backward_workspace_size", _lib.ctypes.byref(inp), kb, _lib.ctypes.byref(nbytes))
        ws = torch.empty(nbytes.value + 256, dtype=torch.uint8, device=self.device)
        return ws, (ws.data_ptr() + 255) & ~255, nbytes.value

    def trace(self, camera, start, points, radii, density, normals, texel_sites, texel_rgb, texel_height, adjacency,
              adjacency_offsets, adjacency_diff, transmittance_threshold=1e-3, max_steps=DEFAULT_MAX_STEPS,
              depth_quantile=0.5, visit_cap=0, check_status=True, record=False, status=None):
        """Walk every pixel's ray.  ``start`` is one cell index or an (H, W)
        int32 tensor of per-ray start cells.  ``record``: also write the
        adjoint's segment records (pf_trace_forward_record; f32, no visit
        log), returned in ``records`` for the backward.  ``status``: a device
        int32 word the kernels raise (not cleared here); a fresh one when None."""
        H, W = camera.height, camera.width
        dev = self.device
        args = self._prep(points, radii, density, normals, texel_sites, texel_rgb, texel_height, adjacency,
                          adjacency_offsets, adjacency_diff)
        if isinstance(start, torch.Tensor) and start.numel() > 1:
            start = start.to(torch.int32).contiguous()
        r = TraceResult(
            color=torch.empty((H, W, 3), dtype=torch.float32, device=dev),
            log_t=torch.empty((H, W), dtype=torch.float32, device=dev),
            depth=torch.empty((H, W), dtype=torch.float32, device=dev),
            normal=torch.empty((H, W, 3), dtype=torch.float32, device=dev),
            depth_seg=torch.empty((H, W), dtype=torch.int32, device=dev),
            depth_sigma=torch.empty((H, W), dtype=torch.float32, device=dev),
            visit_count=torch.empty((H, W), dtype=torch.int32, device=dev),
            visits=torch.empty((H, W, visit_cap), dtype=torch.int32, device=dev) if visit_cap else None,
        )
        if status is None:
            status = torch.zeros(1, dtype=torch.int32, device=dev)
        inp = self._inputs(camera, start, *args, transmittance_threshold, max_steps, depth_quantile)
        if record:
            if visit_cap:
                raise ValueError("a recording walk keeps no visit log")
            kb = self._segments_per_ray(camera)
            ws, ws_ptr, nbytes = self._records(inp, kb)
            _lib.call("pf_trace_forward_record", _lib.ctypes.byref(inp), _lib.ptr(r.color), _lib.ptr(r.log_t),
                      _lib.ptr(r.depth), _lib.ptr(r.normal), _lib.ptr(r.depth_seg), _lib.ptr(r.depth_sigma),
                      _lib.ptr(r.visit_count), _lib.ptr(status), kb, ws_ptr, nbytes, _lib.stream_ptr())
            r.records = (ws, ws_ptr, nbytes, kb)
        else:
            _lib.call("pf_trace_forward", _lib.ctypes.byref(inp), _lib.ptr(r.color), _lib.ptr(r.log_t),
                      _lib.ptr(r.depth), _lib.ptr(r.normal), _lib.ptr(r.depth_seg), _lib.ptr(r.depth_sigma),
                      _lib.ptr(r.visits), int(visit_cap), _lib.ptr(r.visit_count), _lib.ptr(status),
                      _lib.stream_ptr())
        if check_status:
            r.status = int(status.item())
            if r.status != _lib.PF_OK:
                raise _lib.PfError(r.status, "cell walk stopped early (step cap or invalid cell index)")
        return r

    # ------------------------------------------------------------------
    def forward(self, camera, start, points, radii, density, normals, texel_sites, texel_rgb, texel_height,
                adjacency, adjacency_offsets, adjacency_diff, transmittance_threshold=1e-3, max_steps=None,
                depth_quantile=0.5):
        """Differentiable walk: returns (color, log_t, depth, normal)."""
        return RayTraceGradFn.apply(self, camera, start, points, radii, density, normals, texel_sites, texel_rgb,
                                    texel_height, adjacency, adjacency_offsets, adjacency_diff,
                                    transmittance_threshold, max_steps, depth_quantile)

    def _forward(self, ctx, camera, start, points, radii, density, normals, texel_sites, texel_rgb, texel_height,
                 adjacency, adjacency_offsets, adjacency_diff, thr, max_steps, depth_quantile):
        if self.attr_dtype != "float":
            raise ValueError("Forward pass only supports float precision")
        max_steps = DEFAULT_MAX_STEPS if max_steps is None else max_steps
        # with gradients wanted, the walk writes the adjoint's segment records (the adjoint then does not
        # walk again); ctx.needs_input_grad follows the apply() arguments: points ... texel_height are 3-9
        record = self.record_segments and any(ctx.needs_input_grad[3:10])
        r = self.trace(camera, start, points.detach(), radii.detach(), density.detach(), normals.detach(),
                       texel_sites.detach(), texel_rgb.detach(), texel_height.detach(), adjacency, adjacency_offsets,
                       adjacency_diff, thr, max_steps, depth_quantile, record=record, check_status=self.host_sync,
                       status=None if self.host_sync else self.status)
        ctx.records = r.records
        ctx.tracer = self
        ctx.camera = camera
        ctx.start = start
        ctx.cfg = (thr, max_steps, depth_quantile)
        ctx.save_for_backward(points, radii, density, normals, texel_sites, texel_rgb, texel_height, adjacency,
                              adjacency_offsets, adjacency_diff, r.color, r.normal, r.depth_seg, r.depth_sigma)
        return r.color, r.log_t, r.depth, r.normal

    def _backward(self, ctx, g_color, g_log_t, g_depth, g_normal):
        (points, radii, density, normals, texel_sites, texel_rgb, texel_height, adjacency, adjacency_offsets,
         adjacency_diff, color, normal, depth_seg, depth_sigma) = ctx.saved_tensors
        thr, max_steps, depth_quantile = ctx.cfg
        args = self._prep(points.detach(), radii.detach(), density.detach(), normals.detach(), texel_sites.detach(),
                          texel_rgb.detach(), texel_height.detach(), adjacency, adjacency_offsets, adjacency_diff)
        start = ctx.start
        if isinstance(start, torch.Tensor) and start.numel() > 1:
            start = start.to(torch.int32).contiguous()
        inp = self._inputs(ctx.camera, start, *args, thr, max_steps, depth_quantile)
        n = points.shape[0]
        S = texel_sites.shape[1]
        dev = self.device
        out = [torch.empty(s, dtype=torch.float32, device=dev) for s in ((n, 3), (n,), (n, 3), (n,), (n, S, 3),
                                                                         (n, S, 3), (n, S))]
        c = lambda t: None if t is None else t.float().contiguous()
        grads_in = (_lib.ptr(c(g_color)), _lib.ptr(c(g_log_t)), _lib.ptr(c(g_depth)), _lib.ptr(c(g_normal)))
        if ctx.records is not None:  # the forward's segment records
            ws, ws_ptr, nbytes, kb = ctx.records
            _lib.call("pf_trace_backward_recorded", _lib.ctypes.byref(inp), _lib.ptr(color), _lib.ptr(normal),
                      _lib.ptr(depth_seg), _lib.ptr(depth_sigma), *grads_in, *[_lib.ptr(t) for t in out], kb,
                      ws_ptr, nbytes, _lib.stream_ptr())
        else:
            kb = self._segments_per_ray(ctx.camera)
            ws, ws_ptr, nbytes = self._records(inp, kb)
            _lib.call("pf_trace_backward", _lib.ctypes.byref(inp), _lib.ptr(color), _lib.ptr(normal),
                      _lib.ptr(depth_seg), _lib.ptr(depth_sigma), *grads_in, *[_lib.ptr(t) for t in out], kb,
                      ws_ptr, nbytes, _lib.stream_ptr())
        del ctx.tracer, ctx.camera, ctx.start, ctx.records
        g_pts, g_rad, g_nrm, g_den, g_sites, g_rgb, g_h = out
        return (None, None, None, g_pts, g_rad, g_den, g_nrm, g_sites, g_rgb, g_h, None, None, None, None, None,
                None)

    def benchmark(self, camera, start_point_idx, points, radii, density, normals, texel_sites, texel_rgb,
                  texel_height, adjacency, adjacency_offsets, adjacency_diff, transmittance_threshold=1e-3):
        """raytrace.py:247-309: colour of every ray walked from start_point_idx."""
        r = self.trace(camera, start_point_idx, points, radii, density, normals, texel_sites, texel_rgb,
                       texel_height, adjacency, adjacency_offsets, adjacency_diff, transmittance_threshold,
                       check_status=False)
        return r.color
