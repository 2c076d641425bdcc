"""Tile rasterizer: drop-in for powerfoam/rasterize.py.

``Rasterizer(args, device, attr_dtype)`` keeps the reference's constructor,
``forward`` (through the ``RasterGradFn`` autograd function), ``benchmark`` and
``visualize`` signatures, return tuples and error behaviour
(rasterize.py:23-2285).  Every step runs in libpfoam (hand-written sm_100a
CUDA) on torch's current stream; there is no CPU path.

Differences from the reference, all deliberate:
* equal sort keys are ordered by primitive index (the reference leaves them
  in atomic order), so outputs are deterministic up to float atomics;
* tile edge ``tile_width`` may be 8 (the reference's constant), 16 or 32.

Generic cameras (``args.is_pinhole`` False) follow the reference: binning
through the ray-cone hierarchy built from ``camera.ray_maps``
(rasterize.py:202-291, 365-569, 1518-1585; pinhole ray maps are built when
the camera has none, as TorchCamera.to_warp does) and per-pixel ray origins
and directions in the forward and backward; ``benchmark`` and ``visualize``
composite pinhole rays over those bins, as the reference's kernels do.
"""

from dataclasses import dataclass, field

import torch

from . import _lib

TILE_WIDTH = 8
TILE_SIZE = TILE_WIDTH * TILE_WIDTH
# device bytes the forward may use for the adjoint's segment records (64 per
# hit pixel with the texture-plane results, 16 without); larger buffers keep
# the intervals only, or none (the adjoint then clips again)
SEGMENT_BYTES = 24 << 30

# Optional instrumentation: when set, called as hook(name, "begin" | "end")
# around every library call of the forward / backward (bench.py records CUDA
# events there).  It never changes the work done.
PROFILE_HOOK = None


def _timed_call(name, *args):
    hook = PROFILE_HOOK
    if hook is not None:
        hook(name, "begin")
    _lib.call(name, *args)
    if hook is not None:
        hook(name, "end")


@dataclass
class VisOptions:
    """rasterize.py:15-20"""

    transmittance_threshold: float = 1e-3
    max_intersections: int = 1024
    depth_quantile: float = 0.5
    bkgd_color: tuple = field(default_factory=lambda: (0.0, 0.0, 0.0))


class RasterGradFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rasterizer, *args):
        return rasterizer._forward(ctx, *args)

    @staticmethod
    def backward(ctx, *args):
        return ctx.rasterizer._backward(ctx, *args)


def _f32(t, name):
    if t.dtype != torch.float32:
        raise ValueError(f"{name} must be float32, got {t.dtype}")
    return t.contiguous()


class TileBins:
    """Result of binning: per-tile offsets (T+1, int64) and sorted primitive
    ids.  ``n_pairs`` is an int after a synchronous binning and a device
    scalar (int64) after a sync-free one, whose ``tile_prims`` / ``sort_keys``
    then keep the buffer's full capacity (only the first n_pairs entries are
    meaningful; the kernels read the lists through ``tile_offsets``)."""

    def __init__(self, tile_offsets, tile_prims, n_pairs, prim_visible, sort_keys=None, tile_order=None):
        self.tile_order = tile_order
        self.tile_offsets = tile_offsets
        self.tile_prims = tile_prims
        self.n_pairs = n_pairs
        self.prim_visible = prim_visible
        self.sort_keys = sort_keys


class Binner:
    """Owns the binning workspace and the pair capacity estimate.

    Synchronous (``sync=True``, the reference's behaviour: offsets[-1].item(),
    rasterize.py:1714): one host read of the pair count and the status word
    per call, re-binning with a larger capacity when the estimate was too
    small, and PfError(PF_ERR_NONFINITE) when the status reports a NaN or
    infinite attribute.  Sync-free (``sync=False``): the first call sizes the
    pair buffer with one read (1.25x headroom, rounded up to a multiple of
    65,536 pairs); later calls
    read nothing back, so they can be captured in a CUDA graph; an overflow
    then empties the tile lists and raises PF_ERR_OVERFLOW in the caller's
    persistent ``status`` word, which the caller checks when it chooses."""

    def __init__(self, device, headroom=1.25):
        self.device = torch.device(device)
        self.capacity = 0
        self.headroom = headroom
        self.ws = None

    @staticmethod
    def _round(n):
        return ((int(n) + 65535) >> 16) << 16

    def _ensure(self, n_prims, cap, num_tiles):
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_bin_workspace_size", n_prims, cap, num_tiles, _lib.ctypes.byref(nbytes))
        if self.ws is None or self.ws.numel() < nbytes.value:
            self.ws = torch.empty(max(nbytes.value, 256), dtype=torch.uint8, device=self.device)

    def _ensure_generic(self, n_prims, cap, cam_pf, tile_width):
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_bin_generic_workspace_size", n_prims, cap, cam_pf.width, cam_pf.height, tile_width,
                  _lib.ctypes.byref(nbytes))
        if self.ws is None or self.ws.numel() < nbytes.value:
            self.ws = torch.empty(max(nbytes.value, 256), dtype=torch.uint8, device=self.device)

    def _launch(self, cam_pf, tile_width, spheres, n_prims, num_tiles, cap, return_keys, ray_maps, status):
        if ray_maps is None:
            self._ensure(n_prims, cap, num_tiles)
        else:
            self._ensure_generic(n_prims, cap, cam_pf, tile_width)
        tile_offsets = torch.empty(num_tiles + 1, dtype=torch.int64, device=self.device)
        tile_order = torch.empty(num_tiles, dtype=torch.int32, device=self.device)
        tile_prims = torch.empty(max(cap, 1), dtype=torch.int32, device=self.device)
        keys = torch.empty(max(cap, 1), dtype=torch.int64, device=self.device) if return_keys else None
        visible = torch.empty(n_prims, dtype=torch.uint8, device=self.device)
        n_pairs = torch.zeros(1, dtype=torch.int64, device=self.device)
        outs = (_lib.ptr(self.ws), self.ws.numel(), cap, _lib.ptr(tile_offsets), _lib.ptr(tile_prims), _lib.ptr(keys),
                _lib.ptr(visible), _lib.ptr(tile_order), _lib.ptr(n_pairs), _lib.ptr(status), _lib.stream_ptr())
        if ray_maps is None:
            _lib.call("pf_bin", _lib.ctypes.byref(cam_pf), tile_width, _lib.ptr(spheres), n_prims, *outs)
        else:
            _lib.call("pf_bin_generic", _lib.ctypes.byref(cam_pf), _lib.ptr(ray_maps), tile_width,
                      _lib.ptr(spheres), n_prims, *outs)
        return tile_offsets, tile_order, tile_prims, keys, visible, n_pairs

    def __call__(self, cam_pf, tile_width, spheres, n_prims, num_tiles, return_keys=False, capacity=None,
                 ray_maps=None, status=None, sync=True):
        """ray_maps (H,W,6) f32: bin a generic camera through its ray cones.
        status: device int32 word the kernels raise (pf_pack_prims' non-finite
        flag may already be in it); a fresh one when None."""
        own_status = status is None
        if own_status:
            status = torch.zeros(1, dtype=torch.int32, device=self.device)
        if not sync and self.capacity > 0 and capacity is None:
            t_off, t_ord, t_prims, keys, vis, n_pairs = self._launch(cam_pf, tile_width, spheres, n_prims, num_tiles,
                                                                     self.capacity, return_keys, ray_maps, status)
            return TileBins(t_off, t_prims, n_pairs[0], vis.bool(), keys, t_ord)
        cap = capacity if capacity is not None else max(self.capacity, 4 * n_prims, 1 << 14)
        while True:
            t_off, t_ord, t_prims, keys, vis, n_pairs = self._launch(cam_pf, tile_width, spheres, n_prims, num_tiles,
                                                                     cap, return_keys, ray_maps, status)
            n, st = (int(v) for v in torch.stack([n_pairs[0], status[0].long()]).tolist())
            if st == _lib.PF_ERR_NONFINITE:
                raise _lib.PfError(st, "a primitive attribute is NaN or infinite")
            if n <= cap:
                break
            cap = self._round(n * self.headroom)
            status.zero_()
        self.capacity = max(self.capacity, cap)
        if not sync:  # sized: later calls read nothing back
            self.capacity = max(self.capacity, self._round(max(n, 1) * self.headroom))
        return TileBins(t_off, t_prims[:n], n, vis.bool(), keys[:n] if return_keys else None, t_ord)


class Rasterizer:
    """``host_sync`` (default True) keeps the reference's one host read per
    call (the pair count, rasterize.py:1714), here together with the status
    word, so overflow is handled and non-finite attributes raise at once.
    With ``host_sync=False`` only the first call reads back (to size the pair
    buffer); later forward / backward calls never wait on the host and can be
    captured in a CUDA graph, and overflow (PF_ERR_OVERFLOW) or non-finite
    attributes (PF_ERR_NONFINITE) accumulate in the device word ``status``,
    raised by ``check()``."""

    def __init__(self, args, device, attr_dtype="float", tile_width=TILE_WIDTH, host_sync=True):
        self.device = torch.device(device)
        self.host_sync = bool(host_sync)
        self.args = args
        if attr_dtype == "float":
            self.tscalar = torch.float32
        elif attr_dtype == "half":
            self.tscalar = torch.float16
        else:
            raise ValueError(f"Unsupported attribute dtype: {attr_dtype}")
        self.attr_dtype = attr_dtype
        self.loss_accumulation = args.render_objective == "surface"
        self.num_texel_sites = args.num_texel_sites
        self.generic = not getattr(args, "is_pinhole", True)
        if tile_width not in (8, 16, 32):
            raise ValueError("tile_width must be 8, 16 or 32")
        self.tile_width = tile_width
        self.binner = Binner(self.device)
        self.collect_stats = False
        self.last_stats = None
        # device scratch of the compositing kernels' tile work queue; one
        # Rasterizer serves one stream at a time
        self.scratch = torch.zeros(64, dtype=torch.int32, device=self.device)
        # persistent device status word of the sync-free mode (see class docstring)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        # optional multiview.GradBuffer with multiview.raster_fields: the
        # adjoint then writes the gradients into its views (the cross-GPU
        # exchange runs on the buffer with no copies)
        self.grad_buffer = None
        # tile widths 8 and 16: when gradients are wanted, the forward writes
        # each hit (primitive, pixel) pair's clipped sphere interval and
        # bounding-surface ids, and its texture-plane result (a 64-byte
        # record; up to SEGMENT_BYTES), which the adjoint reads instead of
        # clipping and evaluating the plane again.  The record buffer is sized
        # from the last count read back (host_sync: every call; sync-free: the
        # first call and check()); pairs beyond a full buffer are clipped
        # again in the adjoint.
        self.record_segments = True
        self.rec_capacity = 0
        self.rec_count = torch.zeros(1, dtype=torch.int64, device=self.device)
        _lib.load()

    def check(self):
        """Raise PfError if a sync-free call reported overflow or non-finite
        attributes since the last check (one host read); clears the word."""
        st, n_rec = (int(v) for v in torch.stack([self.status[0].long(), self.rec_count[0]]).tolist())
        self._grow_records(n_rec)
        if st != _lib.PF_OK:
            self.status.zero_()
            raise _lib.PfError(st, "a sync-free rasterizer call overflowed its pair buffer (re-run it: the "
                                   "capacity is re-sized) or met a non-finite attribute")
        return True

    def _grow_records(self, n_rec):
        if n_rec > self.rec_capacity:
            self.rec_capacity = min(Binner._round(n_rec * 1.25), (1 << 31) - (1 << 16))

    def _segment_buffers(self, pairs):
        """Record buffer, hit masks, offsets and counter for a forward over
        `pairs` listed pairs, or None when the budget holds none."""
        per_pair = self.tile_width * self.tile_width
        if self.host_sync and self.rec_capacity > 0:
            self._grow_records(int(self.rec_count.item()))  # the previous call's count
        if self.rec_capacity == 0:  # first call: a quarter of the listed pixels
            self.rec_capacity = min(Binner._round(max(pairs * per_pair // 4, 1)), (1 << 31) - (1 << 16))
        cap = self.rec_capacity
        planes = cap * 64 <= SEGMENT_BYTES
        if pairs <= 0 or (not planes and cap * 16 > SEGMENT_BYTES):
            return None
        dev = self.device
        self.rec_count.zero_()
        return (torch.empty((cap * (4 if planes else 1), 4), dtype=torch.float32, device=dev),
                torch.empty(pairs * per_pair // 32, dtype=torch.int32, device=dev),
                torch.empty(pairs * per_pair // 32, dtype=torch.int32, device=dev), self.rec_count, pairs, cap,
                planes)

    def _call_status(self):
        return torch.zeros(1, dtype=torch.int32, device=self.device) if self.host_sync else self.status

    # ------------------------------------------------------------------
    def num_tiles(self, camera):
        tw = self.tile_width
        return (1 + (camera.height - 1) // tw) * (1 + (camera.width - 1) // tw)

    def pack(self, points, radii, normals=None, density=None, status=None):
        """(N,4) spheres (centre, radius) and (N,4) normal+density, as
        rasterize.py:1619-1620 builds them; a NaN or infinite value raises
        PF_ERR_NONFINITE in ``status`` (device int32, optional)."""
        n = points.shape[0]
        spheres = torch.empty((n, 4), dtype=torch.float32, device=self.device)
        nsig = torch.empty((n, 4), dtype=torch.float32, device=self.device) if normals is not None else None
        _lib.call("pf_pack_prims", _lib.ptr(_f32(points, "points")), _lib.ptr(_f32(radii, "radii")),
                  _lib.ptr(None if normals is None else _f32(normals, "normals")),
                  _lib.ptr(None if density is None else _f32(density, "density")), n, _lib.ptr(spheres),
                  _lib.ptr(nsig), _lib.ptr(status), _lib.stream_ptr())
        return spheres, nsig

    def ray_maps(self, camera):
        """The (H,W,6) f32 ray maps of a generic camera (pinhole ones if it
        has none, as the reference's TorchCamera.to_warp builds), else None."""
        if not self.generic:
            return None
        rm = camera.ray_maps if camera.ray_maps is not None else camera.build_pinhole_ray_maps()
        if rm.shape != (camera.height, camera.width, 6):
            raise ValueError("ray_maps must have shape (height, width, 6)")
        if not rm.is_cuda:
            raise ValueError("Only CUDA tensors are supported as inputs")
        return rm.detach().to(torch.float32).contiguous()

    def bin(self, camera, spheres, return_keys=False, ray_maps=None, status=None):
        if self.generic and ray_maps is None:
            ray_maps = self.ray_maps(camera)
        return self.binner(camera.to_pf(), self.tile_width, spheres, spheres.shape[0], self.num_tiles(camera),
                           return_keys=return_keys, ray_maps=ray_maps, status=status, sync=self.host_sync)

    def prefetch_adjacency(self, spheres, adjacency, adjacency_offsets):
        """(E,4) float16 (c_j - c_i, r_j): rasterize.py:580-606."""
        adj_diff = torch.empty((adjacency.shape[0], 4), dtype=torch.float16, device=self.device)
        _lib.call("pf_adjacency_prefetch", _lib.ptr(spheres), _lib.ptr(adjacency), _lib.ptr(adjacency_offsets),
                  spheres.shape[0], _lib.ptr(adj_diff), _lib.stream_ptr())
        return adj_diff

    @staticmethod
    def _set_segments(inp, segs):
        seg, mask, offs, count, pairs, cap, planes = segs
        inp.segments = _lib.ptr(seg)
        inp.segment_masks = _lib.ptr(mask)
        inp.segment_offsets = _lib.ptr(offs)
        inp.segment_count = _lib.ptr(count)
        inp.segment_pairs = int(pairs)
        inp.segment_capacity = int(cap)
        inp.segment_planes = int(planes)

    def _inputs(self, camera, spheres, nsig, sites, rgb, height, adjacency, adjacency_offsets, adj_diff, bins,
                depth_quantiles=None, ray_gt=None, thr=1e-3, attr_half=False, ray_maps=None):
        inp = _lib.PfRasterInputs()
        inp.ray_maps = _lib.ptr(ray_maps)
        inp.cam = camera.to_pf()
        inp.tile_width = self.tile_width
        inp.n_sites = sites.shape[1]
        inp.n_prims = spheres.shape[0]
        inp.spheres = _lib.ptr(spheres)
        inp.nsigmas = _lib.ptr(nsig)
        inp.texel_sites = _lib.ptr(sites)
        inp.texel_rgb = _lib.ptr(rgb)
        inp.texel_height = _lib.ptr(height)
        inp.attr_half = int(attr_half)
        inp.adjacency = _lib.ptr(adjacency)
        inp.adjacency_offsets = _lib.ptr(adjacency_offsets)
        inp.adjacency_diff = _lib.ptr(adj_diff)
        inp.tile_offsets = _lib.ptr(bins.tile_offsets)
        inp.tile_prims = _lib.ptr(bins.tile_prims) if bins.tile_prims.numel() > 0 else _lib.ptr(bins.tile_offsets)
        inp.depth_quantiles = _lib.ptr(depth_quantiles)
        inp.n_quantiles = 0 if depth_quantiles is None else depth_quantiles.shape[-1]
        inp.ray_gt = _lib.ptr(ray_gt)
        inp.transmittance_threshold = float(thr)
        inp.tile_order = _lib.ptr(bins.tile_order)
        inp.scratch = _lib.ptr(self.scratch)
        return inp

    # ------------------------------------------------------------------
    def _forward(self, grad_ctx, camera, depth_quantiles, points, radii, density, normals, texel_sites, texel_rgb,
                 texel_height, adjacency, adjacency_offsets, ray_gt, return_point_err,
                 transmittance_threshold=1e-3):
        if self.attr_dtype != "float":
            raise ValueError("Forward pass only supports float precision")
        if ray_gt is None and self.loss_accumulation:
            raise ValueError("Ground truth rays must be provided for surface loss accumulation")
        if ray_gt is None and return_point_err:
            raise ValueError("Ground truth rays must be provided to return point error")
        H, W = camera.height, camera.width
        dev = self.device
        n = points.shape[0]
        status = self._call_status()
        spheres, nsig = self.pack(points.detach(), radii.detach(), normals.detach(), density.detach(), status)
        sites = _f32(texel_sites.detach(), "texel_sites")
        rgb = _f32(texel_rgb.detach(), "texel_rgb")
        height = _f32(texel_height.detach(), "texel_height")
        adjacency = adjacency.to(torch.int32).contiguous()
        adjacency_offsets = adjacency_offsets.to(torch.int32).contiguous()
        dq = None if depth_quantiles is None else _f32(depth_quantiles.detach(), "depth_quantiles")
        gt = None if ray_gt is None else _f32(ray_gt.detach(), "ray_gt")

        ray_maps = self.ray_maps(camera)
        bins = self.bin(camera, spheres, ray_maps=ray_maps, status=status)
        adj_diff = self.prefetch_adjacency(spheres, adjacency, adjacency_offsets)

        color = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
        log_t = torch.empty((H, W), dtype=torch.float32, device=dev)
        nd = torch.empty((H, W), dtype=torch.float32, device=dev)
        normal = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
        contrib = torch.empty(n, dtype=torch.float32, device=dev)
        qd = torch.empty(dq.shape, dtype=torch.float32, device=dev) if dq is not None else None
        perr = torch.empty(n, dtype=torch.float32, device=dev) if return_point_err else None
        err = torch.empty((H, W), dtype=torch.float32, device=dev) if self.loss_accumulation else None
        early_stop = torch.empty(self.num_tiles(camera), dtype=torch.int32, device=dev)
        stats = torch.empty(self.num_tiles(camera), dtype=torch.int32, device=dev) if self.collect_stats else None
        inp = self._inputs(camera, spheres, nsig, sites, rgb, height, adjacency, adjacency_offsets, adj_diff, bins,
                           dq, gt, transmittance_threshold, ray_maps=ray_maps)
        segs = None
        if (grad_ctx is not None and self.record_segments and self.tile_width in (8, 16)
                and any(grad_ctx.needs_input_grad[3:10])):
            segs = self._segment_buffers(bins.tile_prims.numel())  # the pair buffer's capacity or count
            if segs is not None:
                self._set_segments(inp, segs)
        _timed_call("pf_raster_forward", _lib.ctypes.byref(inp), int(bool(return_point_err)), _lib.ptr(color),
                    _lib.ptr(log_t), _lib.ptr(nd), _lib.ptr(normal), _lib.ptr(qd), _lib.ptr(err), _lib.ptr(contrib),
                    _lib.ptr(perr), _lib.ptr(early_stop), _lib.ptr(stats), _lib.stream_ptr())
        if self.collect_stats:
            self.last_stats = dict(bins=bins, early_stop=early_stop, contrib_pairs=stats,
                                   adjacency_offsets=adjacency_offsets, camera=camera, n_prims=n, segments=segs,
                                   tile_width=self.tile_width)

        if grad_ctx is not None:
            grad_ctx.rasterizer = self
            grad_ctx.camera = camera
            grad_ctx.n_inputs = 14 if transmittance_threshold == 1e-3 else 15
            grad_ctx.thr = transmittance_threshold
            grad_ctx.bins = bins
            grad_ctx.ray_maps = ray_maps
            grad_ctx.segments = segs
            grad_ctx.save_for_backward(dq, spheres, nsig, sites, rgb, height, adjacency, adjacency_offsets,
                                       adj_diff, early_stop, log_t)
        opacity = 1.0 - torch.exp(log_t)
        return color, opacity, nd, normal, qd, err, contrib, perr, bins.prim_visible

    def forward(self, *args):
        return RasterGradFn.apply(self, *args)

    def _backward(self, grad_ctx, grad_color_in, grad_opacity_in, grad_normal_distance_in, grad_normal_in,
                  grad_quantile_depths_in, grad_err_in, grad_contrib_in, grad_point_err_in,
                  grad_prim_visible_mask_in):
        del grad_point_err_in, grad_prim_visible_mask_in
        if self.attr_dtype != "float":
            raise ValueError("Backward pass only supports float precision")
        if self.loss_accumulation:
            raise NotImplementedError()
        (dq, spheres, nsig, sites, rgb, height, adjacency, adjacency_offsets, adj_diff, early_stop,
         log_t) = grad_ctx.saved_tensors
        camera = grad_ctx.camera
        n = spheres.shape[0]
        S = sites.shape[1]
        dev = self.device

        def g(t, shape):
            return torch.zeros(shape, dtype=torch.float32, device=dev) if t is None else _f32(t, "grad")

        H, W = camera.height, camera.width
        gc = g(grad_color_in, (H, W, 3))
        go = g(grad_opacity_in, (H, W))
        gnd = None if grad_normal_distance_in is None else _f32(grad_normal_distance_in, "grad")
        gn = None if grad_normal_in is None else _f32(grad_normal_in, "grad")
        gq = None if (grad_quantile_depths_in is None or dq is None) else _f32(grad_quantile_depths_in, "grad")
        gcon = None if grad_contrib_in is None else _f32(grad_contrib_in, "grad")
        gb = self.grad_buffer
        if gb is not None:
            if gb.n != n or tuple(gb.layout["texel_sites"][2]) != (n, S, 3):
                raise ValueError("grad_buffer does not match the primitive count / texel sites")
            v = gb.views()
            out = dict(points=v["points"], radii=v["radii"], normals=v["normals"], density=v["density"],
                       sites=v["texel_sites"], rgb=v["texel_rgb"], height=v["texel_height"])
        else:
            out = dict(points=torch.empty((n, 3), dtype=torch.float32, device=dev),
                       radii=torch.empty(n, dtype=torch.float32, device=dev),
                       normals=torch.empty((n, 3), dtype=torch.float32, device=dev),
                       density=torch.empty(n, dtype=torch.float32, device=dev),
                       sites=torch.empty((n, S, 3), dtype=torch.float32, device=dev),
                       rgb=torch.empty((n, S, 3), dtype=torch.float32, device=dev),
                       height=torch.empty((n, S), dtype=torch.float32, device=dev))
        inp = self._inputs(camera, spheres, nsig, sites, rgb, height, adjacency, adjacency_offsets, adj_diff,
                           grad_ctx.bins, dq, None, grad_ctx.thr, ray_maps=grad_ctx.ray_maps)
        if grad_ctx.segments is not None:
            self._set_segments(inp, grad_ctx.segments)
        _timed_call("pf_raster_backward", _lib.ctypes.byref(inp), _lib.ptr(early_stop), _lib.ptr(log_t), _lib.ptr(gc),
                    _lib.ptr(go), _lib.ptr(gnd), _lib.ptr(gn), _lib.ptr(gq), _lib.ptr(gcon), _lib.ptr(out["points"]),
                    _lib.ptr(out["radii"]), _lib.ptr(out["normals"]), _lib.ptr(out["density"]),
                    _lib.ptr(out["sites"]), _lib.ptr(out["rgb"]), _lib.ptr(out["height"]), _lib.stream_ptr())
        del grad_ctx.rasterizer, grad_ctx.camera, grad_ctx.bins, grad_ctx.segments
        grads = (None, None, None, out["points"], out["radii"], out["density"], out["normals"], out["sites"],
                 out["rgb"], out["height"], None, None, None, None)
        return grads + (None,) * (grad_ctx.n_inputs - 14)

    # ------------------------------------------------------------------
    def benchmark(self, camera, points, radii, density, normals, texel_sites, texel_rgb, texel_height, adjacency,
                  adjacency_offsets, adjacency_diff, transmittance_threshold=1e-3):
        """Forward colour only, (dc, dpm)-encoded neighbours, attributes in
        attr_dtype (rasterize.py:1982-2131)."""
        H, W = camera.height, camera.width
        status = self._call_status()
        spheres, _ = self.pack(points.float().contiguous(), radii.float().contiguous(), status=status)
        nsig = torch.cat([normals, density[:, None]], dim=-1).to(self.tscalar).contiguous()
        sites = texel_sites.to(self.tscalar).contiguous()
        rgb = texel_rgb.to(self.tscalar).contiguous()
        height = texel_height.to(self.tscalar).contiguous()
        bins = self.bin(camera, spheres, status=status)
        color = torch.empty((H, W, 3), dtype=torch.float32, device=self.device)
        inp = self._inputs(camera, spheres, nsig, sites, rgb, height, adjacency.to(torch.int32).contiguous(),
                           adjacency_offsets.to(torch.int32).contiguous(), adjacency_diff.contiguous(), bins,
                           thr=transmittance_threshold, attr_half=self.attr_dtype == "half")
        _lib.call("pf_raster_benchmark", _lib.ctypes.byref(inp), _lib.ptr(color), _lib.stream_ptr())
        return color

    def visualize(self, camera, points, radii, density, normals, texel_sites, texel_rgb, texel_height, adjacency,
                  adjacency_offsets, vis_options=None):
        """(color, depth, normal, alpha, intersections), rasterize.py:2133-2285;
        written to device buffers (no graphics API)."""
        if vis_options is None:
            vis_options = VisOptions()
        H, W = camera.height, camera.width
        dev = self.device
        status = self._call_status()
        spheres, _ = self.pack(points.float().contiguous(), radii.float().contiguous(), status=status)
        nsig = torch.cat([normals, density[:, None]], dim=-1).to(self.tscalar).contiguous()
        sites = texel_sites.to(self.tscalar).contiguous()
        rgb = texel_rgb.to(self.tscalar).contiguous()
        height = texel_height.to(self.tscalar).contiguous()
        adjacency = adjacency.to(torch.int32).contiguous()
        adjacency_offsets = adjacency_offsets.to(torch.int32).contiguous()
        bins = self.bin(camera, spheres, status=status)
        adj_diff = self.prefetch_adjacency(spheres, adjacency, adjacency_offsets)
        color = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
        depth = torch.empty((H, W), dtype=torch.float32, device=dev)
        normal = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
        alpha = torch.empty((H, W), dtype=torch.float32, device=dev)
        inter = torch.empty((H, W), dtype=torch.int32, device=dev)
        inp = self._inputs(camera, spheres, nsig, sites, rgb, height, adjacency, adjacency_offsets, adj_diff, bins,
                           thr=vis_options.transmittance_threshold, attr_half=self.attr_dtype == "half")
        b = [float(x) for x in vis_options.bkgd_color]
        _lib.call("pf_raster_visualize", _lib.ctypes.byref(inp), int(vis_options.max_intersections),
                  float(vis_options.depth_quantile), b[0], b[1], b[2], _lib.ptr(color), _lib.ptr(depth),
                  _lib.ptr(normal), _lib.ptr(alpha), _lib.ptr(inter), _lib.stream_ptr())
        return color, depth, normal, alpha, inter
