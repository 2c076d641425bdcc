"""Batched multi-view training step: many views of uneven resolution, one
persistent launch (pf_batch_render), captured with everything around it in
one CUDA graph, with tile width and work-queue chunking picked by an
autotuner.

No counterpart in the reference, whose scene renders one view per
Rasterizer.forward call (powerfoam/scene.py:314-353).  Per view the step is
the reference's forward + L2 loss + adjoint; the gradients of all views are
summed.

``BatchStep`` owns every buffer the step touches (static addresses, as graph
replay needs): packed primitives, the fp16 neighbour table, per-view tile
lists, images, texel colours and gradients.  The caller updates the bound
parameter tensors in place between steps.  Texel colours are either given per
view (``texel_rgb``: a list of (N,S,3) tensors, gradients per view in
``grad_texel_rgb``) or produced from SH coefficients (``sh``: (N,16,3)) by
the SH pre-step inside the step, whose adjoint then fills ``grad_sh``.

Sizing without host syncs: the first run bins every view eagerly and reads
the pair counts once to size the per-view pair buffers (1.25x headroom,
rounded to a power of two); later runs and graph replays never read them
back.  ``check()`` reads the device status words (overflow, wait limit) when
the caller chooses.
"""

import json
import os
import time

import torch

from . import _lib

TILE_WIDTHS = (8, 16, 32)
CHUNKS = (1, 2, 4, 8)
ORDERS = {"longest": _lib.PF_BATCH_ORDER_LONGEST, "view": _lib.PF_BATCH_ORDER_VIEW}


def _pow2_at_least(n):
    return 1 << max(int(n) - 1, 1).bit_length()


class BatchStep:
    def __init__(self, device, cameras, tile_width=8, chunk=1, order="longest", transmittance_threshold=1e-3,
                 headroom=1.25, split=False, world=1, record_segments=True, segment_bytes=None):
        if not 1 <= len(cameras) <= _lib.PF_BATCH_MAX_VIEWS:
            raise ValueError(f"1..{_lib.PF_BATCH_MAX_VIEWS} views per batch")
        if tile_width not in TILE_WIDTHS:
            raise ValueError("tile_width must be 8, 16 or 32")
        if order not in ORDERS:
            raise ValueError(f"order must be one of {sorted(ORDERS)}")
        self.device = torch.device(device)
        self.cameras = list(cameras)
        self.tile_width = tile_width
        self.chunk = int(chunk)
        self.order = order
        self.split = bool(split)
        self.world = int(world)  # ranks exchanging grad_buffer (its fields are padded to a multiple)
        self.thr = float(transmittance_threshold)
        self.headroom = headroom
        self.graph = None
        self.bound = False
        self.kernel_events = None  # a list: eager runs append (start, end) events around pf_batch_render
        # segment records (tile widths 8 and 16), as Rasterizer keeps them: the
        # forward stores every hit pixel's interval and plane result, the
        # adjoint reads them instead of clipping again.  One buffer for the
        # batch, sized by a counting launch at bind() and grown by check();
        # pairs past a full buffer are clipped again in the adjoint.
        self.record_segments = bool(record_segments) and tile_width in (8, 16)
        self.segment_bytes = segment_bytes
        self.rec_capacity = 0
        self.segs = None  # (record buffer, capacity in records, plane results stored)
        self.seg_masks = self.seg_offs = None
        self.seg_groups = [0] * len(self.cameras)  # record group per view (non-decreasing)
        self.view_records = None  # records per view, from the counting launch
        _lib.load()
        tw = tile_width
        self.n_tiles = [(1 + (c.height - 1) // tw) * (1 + (c.width - 1) // tw) for c in self.cameras]
        self.cams_pf = [c.to_pf() for c in self.cameras]
        self.eyes = [(_lib.c_f * 3)(*[float(x) for x in c.eye.float().cpu().tolist()]) for c in self.cameras]

    # ------------------------------------------------------------------
    def bind(self, points, radii, density, normals, texel_sites, texel_height, adjacency, adjacency_offsets,
             targets, texel_rgb=None, sh=None):
        """Bind the step's inputs (kept by reference: update them in place)."""
        if (texel_rgb is None) == (sh is None):
            raise ValueError("give exactly one of texel_rgb (per view) or sh")
        if len(targets) != len(self.cameras):
            raise ValueError("one target image per view")
        dev = self.device
        f32 = lambda t, name: _check(t, name, torch.float32)
        self.points = f32(points, "points")
        self.radii = f32(radii, "radii")
        self.density = f32(density, "density")
        self.normals = f32(normals, "normals")
        self.texel_sites = f32(texel_sites, "texel_sites")
        self.texel_height = f32(texel_height, "texel_height")
        self.adjacency = _check(adjacency, "adjacency", torch.int32)
        self.adjacency_offsets = _check(adjacency_offsets, "adjacency_offsets", torch.int32)
        self.targets = [f32(t, "target") for t in targets]
        for t, c in zip(self.targets, self.cameras):
            if tuple(t.shape) != (c.height, c.width, 3):
                raise ValueError("target shape must be (H, W, 3) of its view")
        n = self.points.shape[0]
        S = self.texel_sites.shape[1]
        self.n, self.S = n, S
        V = len(self.cameras)
        self.sh = None if sh is None else f32(sh, "sh")
        if texel_rgb is not None:
            if len(texel_rgb) != V:
                raise ValueError("one texel_rgb tensor per view")
            self.texel_rgb = [f32(t, "texel_rgb") for t in texel_rgb]
        else:
            self.texel_rgb = [torch.empty((n, S, 3), dtype=torch.float32, device=dev) for _ in range(V)]
        # every per-primitive gradient in one flat buffer (multiview.GradBuffer): a multi-GPU step
        # exchanges it in place
        from .multiview import GradBuffer

        fields = {"points": (n, 3), "radii": (n,), "normals": (n, 3), "density": (n,), "texel_sites": (n, S, 3),
                  "texel_height": (n, S)}
        if sh is not None:
            fields["sh"] = (n, 16, 3)
        self.grad_buffer = GradBuffer(fields, dev, world=self.world)
        self.grad_sh = self.grad_buffer.view("sh") if sh is not None else None
        self.spheres = torch.empty((n, 4), dtype=torch.float32, device=dev)
        self.nsigmas = torch.empty((n, 4), dtype=torch.float32, device=dev)
        self.adj_diff = torch.empty((self.adjacency.shape[0], 4), dtype=torch.float16, device=dev)
        e = lambda *s, dt=torch.float32: torch.empty(s, dtype=dt, device=dev)
        self.color = [e(c.height, c.width, 3) for c in self.cameras]
        self.log_t = [e(c.height, c.width) for c in self.cameras]
        self.normal_distance = [e(c.height, c.width) for c in self.cameras]
        self.normal = [e(c.height, c.width, 3) for c in self.cameras]
        self.grad_color = [e(c.height, c.width, 3) for c in self.cameras]
        self.contrib = e(n)  # summed over views
        self.early_stop = [e(T, dt=torch.int32) for T in self.n_tiles]
        self.tile_contrib_pairs = [e(T, dt=torch.int32) for T in self.n_tiles]
        self.grad_texel_rgb = [e(n, S, 3) for _ in range(V)]
        self.grads = {k: self.grad_buffer.view(k) for k in ("points", "radii", "normals", "density", "texel_sites",
                                                             "texel_height")}
        self.tile_loss = e(sum(self.n_tiles))
        self.loss = e(V)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.bin_scalars = torch.zeros((V, 2), dtype=torch.int64, device=dev)  # n_pairs, status
        self.tile_offsets = [e(T + 1, dt=torch.int64) for T in self.n_tiles]
        self.tile_prims = [None] * V
        self.capacity = [0] * V
        self.rec_count = torch.zeros(V, dtype=torch.int64, device=dev)  # one counter per record group
        self._size_bins()
        self._build_structs()
        self._size_records()
        self.bound = True
        self.graph = None

    # ------------------------------------------------------------------
    def _bin_ws(self, cap):
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_bin_workspace_size", self.n, cap, max(self.n_tiles), _lib.ctypes.byref(nbytes))
        return nbytes.value

    def _size_bins(self):
        """Eager binning of every view to size the pair buffers (one host read)."""
        self._pack()
        caps = [max(4 * self.n, 1 << 14)] * len(self.cameras)
        while True:
            self.bin_ws = torch.empty(max(self._bin_ws(max(caps)), 256), dtype=torch.uint8, device=self.device)
            self.tile_prims = [torch.empty(max(c, 1), dtype=torch.int32, device=self.device) for c in caps]
            self.capacity = caps
            self._bin_all()
            counts = self.bin_scalars[:, 0].tolist()
            if all(n <= c for n, c in zip(counts, caps)):
                break
            caps = [max(c, _pow2_at_least(n * self.headroom)) for n, c in zip(counts, caps)]
        self.bin_scalars.zero_()  # statuses are sticky: clear the sizing runs' overflows
        caps = [_pow2_at_least(max(n, 1) * self.headroom) for n in counts]
        if caps != self.capacity:
            self.bin_ws = torch.empty(max(self._bin_ws(max(caps)), 256), dtype=torch.uint8, device=self.device)
            self.tile_prims = [torch.empty(max(c, 1), dtype=torch.int32, device=self.device) for c in caps]
            self.capacity = caps
        ws = _lib.ctypes.c_size_t(0)
        self._views = (_lib.PfBatchView * len(self.cameras))()
        self._fill_views()
        _lib.call("pf_batch_workspace_size", self._views, len(self.cameras), self.tile_width, _lib.ctypes.byref(ws))
        self.batch_ws = torch.empty(max(ws.value, 256), dtype=torch.uint8, device=self.device)

    def _record_budget(self):
        """segment_bytes when given; else half the device memory still free
        (a batch of many views needs more records than one frame)."""
        if self.segment_bytes is not None:
            return int(self.segment_bytes)
        free, _ = torch.cuda.mem_get_info(self.device)
        free += torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        return free // 2

    def _size_records(self):
        """Masks and offsets for every view's pair capacity and the record
        buffer: capacity and record groups from a counting launch when none is
        set, 64 bytes a record with the plane results, 16 without (intervals
        only), none when even that exceeds the budget."""
        self.segs = None
        if not self.record_segments:
            self._build_structs()
            return
        dev = self.device
        n = max(sum(self.capacity) * (self.tile_width * self.tile_width // 32), 1)
        if self.seg_masks is None or self.seg_masks.numel() != n:
            self.seg_masks = torch.empty(n, dtype=torch.int32, device=dev)
            self.seg_offs = torch.empty(n, dtype=torch.int32, device=dev)
        if self.rec_capacity == 0:
            self._count_records()
        cap = self.rec_capacity
        budget = self._record_budget()
        planes = cap * 64 <= budget
        if planes or cap * 16 <= budget:
            self.segs = (torch.empty((cap * (4 if planes else 1), 4), dtype=torch.float32, device=dev), cap, planes)
        self._build_structs()

    def _count_records(self):
        """One step with every view in its own record group and capacity 0
        (every reservation is refused and counted): the records per view, then
        the groups (record_groups) and the capacity, the largest group."""
        from .rasterize import Binner

        V = len(self.cameras)
        self.seg_groups = list(range(V))
        self.segs = (torch.empty((1, 4), dtype=torch.float32, device=self.device), 0, True)
        self._build_structs()
        self._launch()
        self.view_records = [int(c) for c in self.rec_count[:V].tolist()]
        self.segs = None
        need = [max(int(c * self.headroom), 1) for c in self.view_records]
        budget = self._record_budget()
        limit = (1 << 31) - (1 << 16)
        # the largest group that fits, less the rounding of the capacity
        size = lambda per: min(budget // per, limit) - (1 << 16)
        per = 64 if max(need) <= size(64) else 16
        self.seg_groups, sums = record_groups(need, max(size(per), 1))
        self.rec_capacity = min(Binner._round(max(sums)), limit)

    def _fill_views(self):
        base = 0
        for v, c in enumerate(self.cameras):
            w = self._views[v]
            w.segment_pair_base = base
            w.segment_pairs = self.capacity[v]
            w.segment_group = self.seg_groups[v]
            base += self.capacity[v]
            w.cam = self.cams_pf[v]
            w.tile_offsets = _lib.ptr(self.tile_offsets[v])
            w.tile_prims = _lib.ptr(self.tile_prims[v])
            w.texel_rgb = _lib.ptr(self.texel_rgb[v])
            w.target = _lib.ptr(self.targets[v])
            w.color = _lib.ptr(self.color[v])
            w.log_t = _lib.ptr(self.log_t[v])
            w.normal_distance = _lib.ptr(self.normal_distance[v])
            w.normal = _lib.ptr(self.normal[v])
            w.grad_color = _lib.ptr(self.grad_color[v])
            w.contrib = _lib.ptr(self.contrib)
            w.early_stop = _lib.ptr(self.early_stop[v])
            w.tile_contrib_pairs = _lib.ptr(self.tile_contrib_pairs[v])
            w.grad_texel_rgb = _lib.ptr(self.grad_texel_rgb[v])

    def _build_structs(self):
        self._fill_views()
        sc = _lib.PfBatchScene()
        sc.n_sites = self.S
        sc.n_prims = self.n
        sc.spheres = _lib.ptr(self.spheres)
        sc.nsigmas = _lib.ptr(self.nsigmas)
        sc.texel_sites = _lib.ptr(self.texel_sites)
        sc.texel_height = _lib.ptr(self.texel_height)
        sc.adjacency = _lib.ptr(self.adjacency)
        sc.adjacency_offsets = _lib.ptr(self.adjacency_offsets)
        sc.adjacency_diff = _lib.ptr(self.adj_diff)
        sc.transmittance_threshold = self.thr
        if self.segs is not None:
            seg, cap, planes = self.segs
            sc.segments = _lib.ptr(seg)
            sc.segment_masks = _lib.ptr(self.seg_masks)
            sc.segment_offsets = _lib.ptr(self.seg_offs)
            sc.segment_count = _lib.ptr(self.rec_count)
            sc.segment_capacity = int(cap)
            sc.segment_planes = int(planes)
        self._scene = sc

    # ------------------------------------------------------------------
    def _pack(self):
        st = _lib.stream_ptr()
        _lib.call("pf_pack_prims", _lib.ptr(self.points), _lib.ptr(self.radii), _lib.ptr(self.normals),
                  _lib.ptr(self.density), self.n, _lib.ptr(self.spheres), _lib.ptr(self.nsigmas),
                  _lib.ptr(self.status), st)

    def _bin_all(self):
        st = _lib.stream_ptr()
        for v in range(len(self.cameras)):
            sc = self.bin_scalars[v]
            _lib.call("pf_bin", _lib.ctypes.byref(self.cams_pf[v]), self.tile_width, _lib.ptr(self.spheres), self.n,
                      _lib.ptr(self.bin_ws), self.bin_ws.numel(), self.capacity[v], _lib.ptr(self.tile_offsets[v]),
                      _lib.ptr(self.tile_prims[v]), None, None, None, _lib.ptr(sc[:1]),
                      _lib.ptr(sc[1:].view(torch.int32)[:1]), st)

    def _launch(self):
        """The whole step, on the current stream, without host syncs."""
        st = _lib.stream_ptr()
        self._pack()
        _lib.call("pf_adjacency_prefetch", _lib.ptr(self.spheres), _lib.ptr(self.adjacency),
                  _lib.ptr(self.adjacency_offsets), self.n, _lib.ptr(self.adj_diff), st)
        if self.sh is not None:
            for v in range(len(self.cameras)):
                _lib.call("pf_sh_texel_rgb", _lib.ptr(self.points), _lib.ptr(self.sh), self.n, self.S, self.eyes[v],
                          _lib.ptr(self.texel_rgb[v]), st)
        self._bin_all()
        g = self.grads
        if self.kernel_events is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
        _lib.call("pf_batch_render", _lib.ctypes.byref(self._scene), self._views, len(self.cameras), self.tile_width,
                  self.chunk, ORDERS[self.order], int(self.split), _lib.ptr(self.batch_ws), self.batch_ws.numel(),
                  _lib.ptr(self.tile_loss), _lib.ptr(g["points"]), _lib.ptr(g["radii"]), _lib.ptr(g["normals"]),
                  _lib.ptr(g["density"]), _lib.ptr(g["texel_sites"]), _lib.ptr(g["texel_height"]),
                  _lib.ptr(self.status), st)
        if self.kernel_events is not None:
            ev[1].record()
            self.kernel_events.append(ev)
        if self.sh is not None:
            self.grad_sh.zero_()
            for v in range(len(self.cameras)):
                _lib.call("pf_sh_texel_rgb_backward", _lib.ptr(self.points), _lib.ptr(self.sh), self.n, self.S,
                          self.eyes[v], _lib.ptr(self.grad_texel_rgb[v]), _lib.ptr(self.grad_sh), st)
        torch.stack([s.sum() for s in self.tile_loss.split(self.n_tiles)], out=self.loss)

    def run(self):
        """One step; returns the (V,) per-view loss tensor (device)."""
        if not self.bound:
            raise RuntimeError("bind() the inputs first")
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch()
        return self.loss

    def capture(self):
        """Record the step into a CUDA graph; run() then replays it."""
        if not self.bound:
            raise RuntimeError("bind() the inputs first")
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self._launch()  # warm-up outside the graph (kernel attributes, allocator)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch()
        self.graph = g
        return g

    def tune_schedules(self, schedules, iters=3, warmup=1):
        """Time the render launch (pf_batch_autotune) for every (chunk, order,
        split) in `schedules` on this step's bins; returns (mean ms per
        schedule, index of the fastest).  One eager step first brings the
        bins and colours up to date; the host waits for the timings."""
        if not self.bound:
            raise RuntimeError("bind() the inputs first")
        self._launch()
        cands = (_lib.PfBatchSchedule * len(schedules))()
        for c, (ch, order, split) in zip(cands, schedules):
            if order not in ORDERS:
                raise ValueError(f"order must be one of {sorted(ORDERS)}")
            c.chunk, c.order, c.split, c.ms = int(ch), ORDERS[order], int(bool(split)), 0.0
        best = _lib.c_i32(-1)
        g = self.grads
        _lib.call("pf_batch_autotune", _lib.ctypes.byref(self._scene), self._views, len(self.cameras),
                  self.tile_width, cands, len(schedules), int(warmup), int(iters), _lib.ptr(self.batch_ws),
                  self.batch_ws.numel(), _lib.ptr(self.tile_loss), _lib.ptr(g["points"]), _lib.ptr(g["radii"]),
                  _lib.ptr(g["normals"]), _lib.ptr(g["density"]), _lib.ptr(g["texel_sites"]),
                  _lib.ptr(g["texel_height"]), _lib.ptr(self.status), _lib.ctypes.byref(best), _lib.stream_ptr())
        return [float(c.ms) for c in cands], int(best.value)

    def set_schedule(self, chunk=None, order=None, split=None):
        """Change the work-queue chunk / order / fused-or-split schedule (drops
        a captured graph)."""
        if chunk is not None:
            self.chunk = int(chunk)
        if split is not None:
            self.split = bool(split)
        if order is not None:
            if order not in ORDERS:
                raise ValueError(f"order must be one of {sorted(ORDERS)}")
            self.order = order
        self.graph = None

    def check(self):
        """Raise if any device status word reports a problem (host sync).  A
        record group whose count outran the record buffer makes it count the
        records again and size the groups and the buffer anew (and drop a
        captured graph: capture() again)."""
        bs = self.bin_scalars.cpu()
        if self.segs is not None:
            n_groups = self.seg_groups[-1] + 1
            if max(self.rec_count[:n_groups].tolist()) > self.rec_capacity:
                self.graph = None  # it holds the old buffer
                self.rec_capacity = 0  # count again, per view
                self._size_records()
        for v in range(len(self.cameras)):
            n, st = int(bs[v, 0]), int(bs[v, 1]) & 0xffffffff  # the status is the slot's low int32 word
            if st != _lib.PF_OK:
                raise _lib.PfError(st, f"view {v}: {n} pairs exceed the capacity {self.capacity[v]}")
        s = int(self.status.item())
        if s != _lib.PF_OK:
            raise _lib.PfError(s, "batch step reported an error (a non-finite primitive attribute, or a "
                                  "compositing wait limit)")

    def pair_counts(self):
        return self.bin_scalars[:, 0].tolist()


def record_groups(need, size):
    """Contiguous record groups of the views, in order: a view joins the
    current group while the group's records stay within `size`, else it
    starts the next one (a view larger than `size` gets a group of its own).
    Returns the group of each view and the records of each group."""
    groups, sums = [], []
    for n in need:
        if not sums or (sums[-1] > 0 and sums[-1] + n > size):
            sums.append(0)
        groups.append(len(sums) - 1)
        sums[-1] += n
    return groups, sums


def _check(t, name, dtype):
    if not t.is_cuda:
        raise ValueError(f"{name}: only CUDA tensors are supported")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous (bound tensors are used in place)")
    return t


# ----------------------------------------------------------------------------
# autotuner
def default_cache_path():
    return os.environ.get("PF_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "powerfoam_b200", "autotune.json"))


def tune_key(device, cameras, n_prims, n_sites, record_segments=True):
    """Cache key: GPU name, primitive count, sites, the views' resolutions
    and, when the adjoint clips again, a "|clip" suffix."""
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    res = sorted(f"{c.width}x{c.height}" for c in cameras)
    counts = {}
    for r in res:
        counts[r] = counts.get(r, 0) + 1
    views = ",".join(f"{k}*{v}" for k, v in sorted(counts.items()))
    return f"{name}|N={n_prims}|S={n_sites}|views={views}" + ("" if record_segments else "|clip")


def time_step(step, iters=3, warmup=1):
    """Mean device milliseconds of step.run() (CUDA events on the current stream)."""
    for _ in range(warmup):
        step.run()
    st = torch.cuda.current_stream(step.device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(step.device)
    a.record(st)
    for _ in range(iters):
        step.run()
    b.record(st)
    torch.cuda.synchronize(step.device)
    return a.elapsed_time(b) / iters


def autotune(device, cameras, bind_kwargs, tile_widths=TILE_WIDTHS, chunks=CHUNKS, orders=("longest", "view"),
             splits=(False, True), iters=3, warmup=1, cache_path=None, use_cache=True, transmittance_threshold=1e-3,
             log=None, prune=1.3, record_segments=True):
    """Sweep tile width x work-queue chunk x item order x fused / split
    schedule and return (best BatchStep bound and ready, table).  Per tile
    width the views are binned at that width and pf_batch_autotune times the
    render launch for every schedule (CUDA events, `iters` runs after
    `warmup`); the width's best schedule is then timed over the whole step
    (colour pre-step, binning, render, adjoint pre-step: the binning's cost
    depends on the width), and the width with the fastest step wins.  Table
    rows: one per (width, schedule) with its render_ms, step_ms on each
    width's best row (None elsewhere).  Tile widths are swept in the given
    order; once a width's step time exceeds `prune` x the best so far, the
    remaining widths are skipped (step time grows monotonically with the width
    on these workloads).  The winner is cached in a JSON file keyed by
    tune_key(); a cached entry skips the sweep."""
    cache_path = cache_path or default_cache_path()
    n = bind_kwargs["points"].shape[0]
    S = bind_kwargs["texel_sites"].shape[1]
    key = tune_key(device, cameras, n, S, record_segments)
    cache = {}
    if os.path.exists(cache_path):
        try:
            with open(cache_path) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}

    def make(best):
        step = BatchStep(device, cameras, best["tile_width"], best["chunk"], best["order"], transmittance_threshold,
                         split=best.get("split", False), record_segments=record_segments)
        step.bind(**bind_kwargs)
        return step

    if use_cache and key in cache:
        best = cache[key]
        return make(best), best.get("table", [])
    scheds = [(ch, order, bool(split)) for split in splits for order in orders for ch in chunks]
    table = []
    best = None
    for tw in tile_widths:
        t0 = time.perf_counter()
        step = BatchStep(device, cameras, tw, 1, "longest", transmittance_threshold,
                         record_segments=record_segments)
        step.bind(**bind_kwargs)
        times, bi = step.tune_schedules(scheds, iters=iters, warmup=warmup)
        rows = [{"tile_width": tw, "chunk": ch, "order": order, "split": split, "render_ms": ms, "step_ms": None}
                for (ch, order, split), ms in zip(scheds, times)]
        ch, order, split = scheds[bi]
        step.set_schedule(chunk=ch, order=order, split=split)
        rows[bi]["step_ms"] = time_step(step, iters=iters, warmup=warmup)
        table += rows
        if log:
            for r in rows:
                log(f"autotune tile={tw} chunk={r['chunk']} order={r['order']} split={r['split']}: render "
                    f"{r['render_ms']:.3f} ms" + (f", step {r['step_ms']:.3f} ms" if r["step_ms"] else ""))
            log(f"autotune tile={tw}: {time.perf_counter() - t0:.1f} s")
        width_best = rows[bi]
        if best is None or width_best["step_ms"] < best["step_ms"]:
            best = dict(width_best)
        del step
        torch.cuda.empty_cache()
        if prune and width_best["step_ms"] > prune * best["step_ms"]:
            if log:
                log(f"autotune: tile {tw} is {width_best['step_ms'] / best['step_ms']:.2f}x the best; larger widths "
                    "skipped")
            break
    best["table"] = table
    cache[key] = best
    try:
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, cache_path)
    except OSError:
        pass
    return make(best), table
