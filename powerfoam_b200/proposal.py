"""Ray-proposal network and the proposal-seeded cell walk.

No counterpart in the reference (its tracer, powerfoam/raytrace.py:115-309,
always walks from the camera's cell).  ``ProposalNet`` holds the network of
pf_mlp.cu (positional encoding -> 3 x 64 ReLU -> entry distance and
confidence; BF16 tensor-core GEMMs, FP32 accumulation and FP32 master
weights with Adam), trains it with the library's own forward/backward/Adam
kernels on rays labelled by the plain tracer (``make_training_rays``), and
``SeededTracer`` starts each confident ray's walk at the power cell that
contains its predicted entry point, falling back to the plain walk below the
confidence threshold.
"""

import math

import torch

from . import _lib
from .raytrace import DEFAULT_MAX_STEPS

LABEL_TRANSMITTANCE = 0.99


class ProposalNet:
    def __init__(self, device, seed=0):
        self.device = torch.device(device)
        lib = _lib.load()
        self.n_params = lib.pf_mlp_param_count()
        self.image_bytes = lib.pf_mlp_image_bytes()
        dev = self.device
        self.weights = init_weights(seed).to(dev)
        self.m = torch.zeros_like(self.weights)
        self.v = torch.zeros_like(self.weights)
        self.grad = torch.zeros_like(self.weights)
        self.image = torch.zeros(self.image_bytes, dtype=torch.uint8, device=dev)
        self.step = torch.zeros(1, dtype=torch.int32, device=dev)
        self.done = torch.zeros(1, dtype=torch.int32, device=dev)
        self.loss = torch.zeros(2, dtype=torch.float32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.margin = 0.02  # seed back-off the confidence head was trained for
        self.pack()

    def pack(self):
        """BF16 image of the current master weights."""
        _lib.call("pf_mlp_pack", _lib.ptr(self.weights), _lib.ptr(self.image), _lib.stream_ptr())

    def load_weights(self, w):
        with torch.no_grad():
            self.weights.copy_(torch.as_tensor(w, dtype=torch.float32))
        self.pack()

    # ------------------------------------------------------------------
    def forward(self, rays=None, camera=None):
        """(t_entry, confidence) for rays (n, 6) = origin, unit direction, or
        for every pixel ray of `camera` ((H, W) each)."""
        if (rays is None) == (camera is None):
            raise ValueError("give rays or a camera")
        if rays is not None:
            rays = rays.to(torch.float32).contiguous()
            n = rays.shape[0]
            shape = (n,)
            cam = None
        else:
            n = camera.width * camera.height
            shape = (camera.height, camera.width)
            cam = _lib.ctypes.byref(camera.to_pf())
        t = torch.empty(shape, dtype=torch.float32, device=self.device)
        c = torch.empty(shape, dtype=torch.float32, device=self.device)
        _lib.call("pf_mlp_forward", _lib.ptr(self.image), _lib.ptr(rays), n, cam, _lib.ptr(t), _lib.ptr(c),
                  _lib.ptr(self.status), _lib.stream_ptr())
        return t, c

    def train_step(self, rays8, batch, seed=0, overshoot_weight=10.0, margin=0.02, lr=1e-3, record_loss=True):
        """One Adam step on a minibatch drawn from rays8 (n, 8) (no host sync)."""
        st = _lib.stream_ptr()
        if record_loss:
            self.loss.zero_()
        _lib.call("pf_mlp_train_step", _lib.ptr(self.image), _lib.ptr(rays8), rays8.shape[0], int(batch),
                  _lib.ptr(self.step), int(seed) & 0xFFFFFFFF, float(overshoot_weight), float(margin),
                  _lib.ptr(self.grad), _lib.ptr(self.loss) if record_loss else None, _lib.ptr(self.status), st)
        _lib.call("pf_mlp_adam", _lib.ptr(self.weights), _lib.ptr(self.m), _lib.ptr(self.v), _lib.ptr(self.grad),
                  _lib.ptr(self.image), _lib.ptr(self.step), _lib.ptr(self.done), float(lr), 0.9, 0.999, 1e-8, st)

    def train(self, rays8, steps=5000, batch=65536, lr=1e-3, seed=0, overshoot_weight=10.0, margin=0.02,
              graph_steps=50, log=None):
        """Train for `steps` Adam steps; chunks of graph_steps steps are
        replayed from one CUDA graph.  Returns the per-chunk mean losses
        (entry-distance term, confidence term) of each chunk's last step."""
        rays8 = rays8.to(torch.float32).contiguous()
        self.margin = float(margin)
        history = []
        kw = dict(seed=seed, overshoot_weight=overshoot_weight, margin=margin, lr=lr)

        def chunk(n):
            for i in range(n):
                self.train_step(rays8, batch, record_loss=(i == n - 1), **kw)

        done = 0
        g = None
        if graph_steps and steps >= 2 * graph_steps:
            s = torch.cuda.Stream(device=self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                chunk(graph_steps)  # warm-up (kernel attributes) outside the graph
            torch.cuda.current_stream(self.device).wait_stream(s)
            done += graph_steps
            history.append([x / batch for x in self.loss.tolist()])
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                chunk(graph_steps)
        while done < steps:
            n = min(graph_steps or steps, steps - done)
            if g is not None and n == graph_steps:
                g.replay()
            else:
                chunk(n)
            done += n
            history.append([x / batch for x in self.loss.tolist()])
            if log:
                log(f"proposal step {done}: loss_t {history[-1][0]:.5f} loss_conf {history[-1][1]:.4f}")
        self.check()
        return history

    def calibrate(self, rays8, max_unsafe=0, floor=0.9, max_unsafe_frac=0.0, t_slack=0.0):
        """Confidence threshold from held-out labelled rays (n, 8): the plain
        walk judges each seed, and the threshold sits just above the
        confidence of the (k + 1)-th most confident seed that would have
        started past its first significant cell, k = max(max_unsafe,
        max_unsafe_frac * n) (never below `floor`; rays flagged as never
        reaching one are safe anywhere).  t_slack > 0 counts a seed as unsafe
        already when it starts within t_slack of that cell: a more
        conservative gate for rays unlike the held-out ones."""
        rays8 = rays8.to(torch.float32).contiguous()
        t, c = self.forward(rays=rays8[:, :6].contiguous())
        lab = rays8[:, 6]
        # a ray flagged as never reaching a significant cell is safe wherever it is seeded
        unsafe = (lab >= 0) & (rays8[:, 7] == 0) & (t - self.margin + float(t_slack) > lab)
        k = max(int(max_unsafe), int(max_unsafe_frac * rays8.shape[0]))
        cu = torch.sort(c[unsafe], descending=True).values
        thr = float(cu[k]) if cu.numel() > k else 0.0
        return max(floor, math.nextafter(thr, 2.0))

    def seed_fraction(self, rays8, threshold):
        """Share of the rays (n, 8) the gate at `threshold` would seed."""
        t, c = self.forward(rays=rays8[:, :6].to(torch.float32).contiguous())
        return float(((c >= threshold) & (t - self.margin > 0)).float().mean())

    def check(self):
        s = int(self.status.item())
        if s != _lib.PF_OK:
            raise _lib.PfError(s, "proposal network kernel reported an error")


def init_weights(seed=0):
    """Uniform fan-in initialisation of the data columns (CPU, seeded); the
    bias and pad columns and the unused output rows start at zero."""
    g = torch.Generator().manual_seed(seed)
    blocks = []
    for li, out in enumerate((64, 64, 64, 16)):
        fan_in = 78 if li == 0 else 64
        bound = math.sqrt(6.0 / fan_in) if li < 3 else math.sqrt(1.0 / fan_in)
        w = torch.zeros(out, 80)
        rows = out if li < 3 else 2
        w[:rows, :fan_in] = (torch.rand(rows, fan_in, generator=g) * 2 - 1) * bound
        blocks.append(w.reshape(-1))
    return torch.cat(blocks).float()


# ----------------------------------------------------------------------------
def trace_labels(tracer, camera, start, scene_args, label_transmittance=LABEL_TRANSMITTANCE,
                 max_steps=DEFAULT_MAX_STEPS):
    """pf_trace_labels over every pixel ray of `camera`: dict of colour, label
    t / cell / step and the number of cells walked."""
    args = tracer._prep(*scene_args)
    inp = tracer._inputs(camera, start, *args, 1e-3, max_steps, 0.5)
    H, W = camera.height, camera.width
    dev = tracer.device
    out = dict(color=torch.empty((H, W, 3), dtype=torch.float32, device=dev),
               label_t=torch.empty((H, W), dtype=torch.float32, device=dev),
               label_cell=torch.empty((H, W), dtype=torch.int32, device=dev),
               label_step=torch.empty((H, W), dtype=torch.int32, device=dev),
               visit_count=torch.empty((H, W), dtype=torch.int32, device=dev))
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call("pf_trace_labels", _lib.ctypes.byref(inp), float(label_transmittance), _lib.ptr(out["color"]),
              _lib.ptr(out["label_t"]), _lib.ptr(out["label_cell"]), _lib.ptr(out["label_step"]),
              _lib.ptr(out["visit_count"]), _lib.ptr(status), _lib.stream_ptr())
    out["status"] = status
    return out


def camera_rays(camera):
    """(H*W, 6) origin and unit direction of every pixel ray (row-major)."""
    H, W = camera.height, camera.width
    d = camera.ray_directions().float()
    o = camera.eye.float()[None, None, :].expand(H, W, 3)
    return torch.cat([o, d], dim=-1).reshape(-1, 6)


def box_exit(rays, lo, hi):
    """Distance along each ray (n, 6: origin, unit direction) at which it
    leaves the box [lo, hi]; 0 for rays that miss it or leave behind."""
    o, d = rays[:, :3], rays[:, 3:6]
    inv = 1.0 / torch.where(d == 0, torch.full_like(d, 1e-30), d)
    t0, t1 = (lo - o) * inv, (hi - o) * inv
    t_near = torch.minimum(t0, t1).max(-1).values
    t_far = torch.maximum(t0, t1).min(-1).values
    return torch.where((t_far >= t_near) & (t_far > 0), t_far, torch.zeros_like(t_far))


def make_training_rays(tracer, cameras, scene_args, start_cells, label_transmittance=LABEL_TRANSMITTANCE,
                       box=None):
    """(n, 8) training rays (origin, direction, label t, no-hit flag) from the
    plain walk of every pixel of every camera.  The label is the entry t of the
    first cell after which the transmittance is below label_transmittance.
    Rays that never get there have label -1, or with ``box`` (lo, hi) of the
    primitives the t at which they leave it and flag 1: seeding them there
    skips a walk that composites next to nothing (the transmittance stays
    above label_transmittance all the way)."""
    parts = []
    for cam, start in zip(cameras, start_cells):
        lab = trace_labels(tracer, cam, start, scene_args, label_transmittance)
        r = camera_rays(cam)
        t = lab["label_t"].reshape(-1, 1)
        flag = torch.zeros_like(t)
        if box is not None:
            miss = t[:, 0] < 0
            t = torch.where(miss[:, None], box_exit(r, box[0], box[1])[:, None], t)
            flag = miss[:, None].to(t.dtype)
        parts.append(torch.cat([r, t, flag], dim=-1))
    return torch.cat(parts, 0).contiguous()


class CellLocator:
    """Power-cell point location over fixed primitives (pf_locator_build)."""

    def __init__(self, points, radii):
        self.points = points.float().contiguous()
        self.radii = radii.float().contiguous()
        n = self.points.shape[0]
        nbytes = _lib.ctypes.c_size_t(0)
        _lib.call("pf_locator_workspace_size", n, _lib.ctypes.byref(nbytes))
        self.ws = torch.empty(max(nbytes.value, 256), dtype=torch.uint8, device=self.points.device)
        _lib.call("pf_locator_build", _lib.ptr(self.points), _lib.ptr(self.radii), n, _lib.ptr(self.ws),
                  self.ws.numel(), _lib.stream_ptr())

    def locate(self, queries, status=None):
        q = queries.float().contiguous()
        out = torch.empty(q.shape[0], dtype=torch.int32, device=q.device)
        st = status if status is not None else torch.zeros(1, dtype=torch.int32, device=q.device)
        _lib.call("pf_locate_cells", _lib.ptr(self.points), _lib.ptr(self.radii), self.points.shape[0],
                  _lib.ptr(self.ws), _lib.ptr(q), q.shape[0], _lib.ptr(out), _lib.ptr(st), _lib.stream_ptr())
        return out

    def seed(self, camera, t_entry, confidence, conf_threshold, default_start, n_seeded=None):
        H, W = camera.height, camera.width
        start = torch.empty((H, W), dtype=torch.int32, device=self.points.device)
        _lib.call("pf_seed_start_cells", _lib.ptr(self.points), _lib.ptr(self.radii), self.points.shape[0],
                  _lib.ptr(self.ws), _lib.ctypes.byref(camera.to_pf()), _lib.ptr(t_entry), _lib.ptr(confidence),
                  float(conf_threshold), int(default_start), _lib.ptr(start), _lib.ptr(n_seeded), _lib.stream_ptr())
        return start


class VoxelLocator:
    """Point location through a voxel map (pf_voxel_map_build): the power cell
    of every voxel centre of a res^3 grid over the primitives' bounding box,
    located exactly once per scene; a point then walks from its voxel's cell
    across the power faces of `adjacency` to the cell that contains it (a few
    faces), where CellLocator searches a grid of primitives for every query."""

    def __init__(self, points, radii, adjacency, adjacency_offsets, res=256, max_walk_steps=64):
        self.points = points.float().contiguous()
        self.radii = radii.float().contiguous()
        self.adjacency = adjacency.to(torch.int32).contiguous()
        self.adjacency_offsets = adjacency_offsets.to(torch.int32).contiguous()
        self.res = int(res)
        self.max_walk_steps = int(max_walk_steps)
        lo = self.points.min(0).values.cpu().tolist()
        hi = self.points.max(0).values.cpu().tolist()
        self.box = ((_lib.c_f * 3)(*lo), (_lib.c_f * 3)(*hi))
        exact = CellLocator(self.points, self.radii)
        self.cells = torch.empty(self.res ** 3, dtype=torch.int32, device=self.points.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.points.device)
        _lib.call("pf_voxel_map_build", _lib.ptr(self.points), _lib.ptr(self.radii), self.points.shape[0],
                  _lib.ptr(exact.ws), self.box[0], self.box[1], self.res, _lib.ptr(self.cells), _lib.ptr(status),
                  _lib.stream_ptr())
        st = int(status.item())
        if st != _lib.PF_OK:
            raise _lib.PfError(st, "a voxel centre could not be located")

    def _common(self):
        return (_lib.ptr(self.points), _lib.ptr(self.radii), self.points.shape[0], _lib.ptr(self.adjacency),
                _lib.ptr(self.adjacency_offsets), _lib.ptr(self.cells), self.box[0], self.box[1], self.res)

    def locate(self, queries):
        """Cells containing queries (n, 3); -1 where the walk gave up."""
        q = queries.float().contiguous()
        out = torch.empty(q.shape[0], dtype=torch.int32, device=q.device)
        _lib.call("pf_locate_cells_vmap", *self._common(), _lib.ptr(q), q.shape[0], self.max_walk_steps,
                  _lib.ptr(out), _lib.stream_ptr())
        return out

    def seed(self, camera, t_entry, confidence, conf_threshold, default_start, n_seeded=None):
        H, W = camera.height, camera.width
        start = torch.empty((H, W), dtype=torch.int32, device=self.points.device)
        _lib.call("pf_seed_start_cells_vmap", *self._common(), _lib.ctypes.byref(camera.to_pf()),
                  _lib.ptr(t_entry), _lib.ptr(confidence), float(conf_threshold), int(default_start),
                  self.max_walk_steps, _lib.ptr(start), _lib.ptr(n_seeded), _lib.stream_ptr())
        return start


class OccupancySeeder:
    """A conservative proposal without a network (pf_occupancy_build,
    pf_occupancy_entry): each pixel ray starts in the cell that contains the
    point where it enters the first voxel of a res^3 grid that a primitive of
    density >= sigma_min reaches (`margin` earlier, one voxel by default), or
    where it leaves the primitives' box when it meets none.  The walk
    composites only inside spheres of density >= 1e-3, so the seeded walk
    skips only cells that add nothing; the cells are located through
    `locator` (a VoxelLocator)."""

    def __init__(self, points, radii, density, locator, res=128, sigma_min=1e-3, margin=None):
        self.locator = locator
        self.res = int(res)
        dev = locator.points.device
        words = _lib.c_i64(0)
        _lib.call("pf_occupancy_words", self.res, _lib.ctypes.byref(words))
        self.bits = torch.zeros(words.value, dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        pts = points.float().contiguous()
        rad = radii.float().contiguous()
        den = density.float().contiguous()
        # the grid holds every sphere whole: a ray can cross a sphere's part beyond its centre's box
        grow = float(rad.max()) if rad.numel() else 0.0
        lo = [a - grow for a in locator.box[0]]
        hi = [b + grow for b in locator.box[1]]
        self.h = max(max(b - a for a, b in zip(lo, hi)), 1e-6) / self.res
        lo, hi = [a - self.h for a in lo], [b + self.h for b in hi]
        self.h = max(max(b - a for a, b in zip(lo, hi)), 1e-6) / self.res
        self.box = ((_lib.c_f * 3)(*lo), (_lib.c_f * 3)(*hi))
        self.margin = self.h if margin is None else float(margin)
        _lib.call("pf_occupancy_build", _lib.ptr(pts), _lib.ptr(rad), _lib.ptr(den), pts.shape[0], self.box[0],
                  self.box[1], self.res, float(sigma_min), _lib.ptr(self.bits), _lib.ptr(self.status),
                  _lib.stream_ptr())

    def entry(self, camera):
        """(t_entry, confidence), (H, W) each, for pf_seed_start_cells_vmap."""
        H, W = camera.height, camera.width
        dev = self.bits.device
        t = torch.empty((H, W), dtype=torch.float32, device=dev)
        c = torch.empty((H, W), dtype=torch.float32, device=dev)
        _lib.call("pf_occupancy_entry", _lib.ptr(self.bits), self.box[0], self.box[1], self.res,
                  _lib.ctypes.byref(camera.to_pf()), self.margin, _lib.ptr(t), _lib.ptr(c), _lib.stream_ptr())
        return t, c

    def start_cells(self, camera, default_start, n_seeded=None):
        t, c = self.entry(camera)
        return self.locator.seed(camera, t, c, 0.5, default_start, n_seeded)

    def check(self):
        s = int(self.status.item())
        if s != _lib.PF_OK:
            raise _lib.PfError(s, "a primitive centre or radius is not finite")


class SeededTracer:
    """Proposal-seeded cell walk: network forward over the pixel rays, start
    cells from the locator where the confidence reaches the threshold, then
    the tracer's walk from those cells (plain start cell elsewhere)."""

    def __init__(self, tracer, net, points, radii, conf_threshold=0.9, adjacency=None, adjacency_offsets=None,
                 voxel_res=256, occupancy=None):
        self.tracer = tracer
        self.net = net
        self.conf_threshold = conf_threshold
        self.occupancy = occupancy  # an OccupancySeeder: rays the gate does not seed start at its safe entry
        # with the walk's adjacency: voxel-map location (a few faces per seed), else the grid search
        self.locator = (VoxelLocator(points, radii, adjacency, adjacency_offsets, voxel_res)
                        if adjacency is not None else CellLocator(points, radii))
        self.n_seeded = torch.zeros(1, dtype=torch.int32, device=tracer.device)

    def start_cells(self, camera, default_start):
        """The confidence predicts that t - margin lies before the first
        significant cell, so the seed point is backed off by the margin."""
        t, c = self.net.forward(camera=camera)
        t.sub_(self.net.margin)
        if self.occupancy is None:
            return self.locator.seed(camera, t, c, self.conf_threshold, default_start, self.n_seeded)
        # both seeds are safe: the later one of the two wherever both apply
        t_o, c_o = self.occupancy.entry(camera)
        net_ok, occ_ok = c >= self.conf_threshold, c_o > 0.5
        t = torch.where(net_ok & occ_ok, torch.maximum(t, t_o), torch.where(net_ok, t, t_o)).contiguous()
        c = (net_ok | occ_ok).float().contiguous()
        return self.locator.seed(camera, t, c, 0.5, default_start, self.n_seeded)

    def render(self, camera, default_start, scene_args, **kw):
        start = self.start_cells(camera, default_start)
        return self.tracer.trace(camera, start, *scene_args, check_status=False, **kw)
