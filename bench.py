"""Benchmark: differentiable rasterizer forward + backward at 1M primitives 1080p.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one training iteration of the rendering path on one
view): 1,048,576 primitives drawn from a 32-component Gaussian mixture
(sigma 0.15) plus 10 % uniform background, r log-uniform in [0.002, 0.02],
degree-3 SH colours; one 1920x1080 pinhole camera with a 50 degree vertical
field of view on a radius-3 orbit; the step evaluates the per-view texel
colours, rasterizes (pack, bin, neighbour encoding, composite), takes an L2
loss against a seeded uniform target image and runs the adjoint to gradients
of every primitive attribute.  Data are synthetic (seeded); the scene (256 MB
of primitive attributes) is larger than L2, so no flush is needed.

With N > 1 (torchrun, one process per GPU, NCCL) every rank renders its own
view of the same scene and the per-primitive gradients are summed across ranks
with one NCCL all-reduce per step (data-parallel over views): weak scaling.

--impl reference times the reference algorithm on the host cores: the CPU
restatement of the reference kernels (oracle/, OpenMP; the reference's Warp
kernels are not importable here), inputs built on the host, each step 1/16 of
the frame's work (binning of every 16th primitive, forward + adjoint of every
16th tile), frames/s = frames of work done / time.
"""

import argparse
import math
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

from powerfoam_b200.multiview import GradBuffer, max_over_ranks, raster_fields, shard_views  # noqa: E402

METRIC = "fwd+bwd ms/iter, FPS @1M prims 1080p; proposal vs plain trace @≥50dB PSNR"
UNIT = "frames/s (fwd+bwd iterations/s)"
WORKLOAD = "raster1m"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)  # ~1.1 s timed at raster1m: one transient stall moves it little
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--tile", type=int, default=8)
    p.add_argument("--workload", default=WORKLOAD, help="raster1m (the measured configuration), raster256k "
                   "(a quarter-size case with the same density per pixel, for profiling), batch3m (32 views of "
                   "a 3.1M-primitive scene in one graph-captured persistent step), batch256k (its small case), "
                   "trace1m (tracer forward + adjoint), interpen3m (interpenetration loss forward + adjoint), power1m "
                   "(power-diagram adjacency build), fisheye1m (raster1m through a generic fisheye camera), color1m "
                   "(spherical-Voronoi texel colour forward + adjoint) or proposal "
                   "(proposal-seeded vs plain cell walk)")
    p.add_argument("--cpu-slices", type=int, default=4, help="slices (1/16 of a frame each) the CPU baseline times")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-segment-records", action="store_true",
                   help="raster and batch workloads: the adjoint clips the sphere intervals again instead of "
                   "reading the forward's segment records (record_segments = False)")
    p.add_argument("--graph", action="store_true",
                   help="raster workloads, one GPU: time the step as CUDA graph replays (the sync-free step is "
                   "captured whole) instead of eager calls")
    p.add_argument("--host-sync", action="store_true",
                   help="raster workloads: Rasterizer(host_sync=True), the reference's host read of the pair count "
                   "per call; by default the step runs sync-free (host_sync=False: the host queues steps ahead "
                   "of the GPU, and overflow or non-finite inputs are checked once after the timed steps)")
    p.add_argument("--no-autotune", action="store_true", help="batch workloads: use --tile, chunk 1")
    p.add_argument("--proposal-prims", type=int, default=0,
                   help="proposal workload: primitive count (default 6,291,456; radii scale with the spacing)")
    p.add_argument("--proposal-scene", default="clouds", choices=["clouds", "shells"],
                   help="proposal workload: the configuration's Gaussian clouds, or opaque shells (radius 0.12, "
                   "thickness 0.02, density x30) in empty space")
    return p.parse_args()


# Per launch of the dominant kernel, from one ncu capture of the same command
# (`ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,smsp__inst_executed.sum ... -k
# regex:raster_bwd_kernel -s 1 -c 1 python bench.py --steps 2 --warmup 1 --no-cpu-baseline`, one
# pass): DRAM bytes read + written, and warp instructions for the issue roofline.  Recorded once
# per kernel change; the bench line carries them as capture metadata next to its live timings.
CAPTURES = {
    # the adjoint that reads the forward's segment records (the default)
    ("raster1m", "pf_raster_backward", True): dict(
        traffic=4.523e9 + 283.23e6, warp_instructions=6_956_738_056,
        source="ncu capture of raster_bwd_kernel<8, 0, 2, false> (the second step's adjoint, `-k regex:raster_ -s 3 "
               "-c 6` on `python bench.py --steps 2 --warmup 1 --no-cpu-baseline`), on the build before the "
               "adjoint stored its first gradient-table writes (which removed shared-memory loads, so the current "
               "launch issues fewer): dram__bytes_read.sum + dram__bytes_write.sum, smsp__inst_executed.sum"),
    # the adjoint that clips again (--no-segment-records)
    ("raster1m", "pf_raster_backward", False): dict(
        traffic=816.77e6 + 206.06e6, warp_instructions=11_715_679_565,
        source="ncu capture of raster_bwd_kernel<8, 0> (second launch of `python bench.py --steps 2 --warmup 1 "
               "--no-cpu-baseline --no-segment-records`): dram__bytes_read.sum + dram__bytes_write.sum, "
               "smsp__inst_executed.sum"),
}
SMS, SCHEDULERS_PER_SM = 148, 4


def capture_traffic(kernel, workload, records):
    c = CAPTURES.get((workload, kernel, records))
    return (c["traffic"], c["source"]) if c else None


def issue_roofline(kernel, workload, records, ms, sm_mhz):
    """Warp instructions of the captured launch / issue slots of the live
    launch time (148 SMs x 4 schedulers x clock x time)."""
    c = CAPTURES.get((workload, kernel, records))
    if not c or not ms:
        return None
    mhz = sm_mhz or 1965.0
    slots = SMS * SCHEDULERS_PER_SM * mhz * 1e6 * ms * 1e-3
    return dict(warp_instructions=c["warp_instructions"], issue_slots=slots,
                frac=c["warp_instructions"] / slots, sm_mhz=mhz, source=c["source"])


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:  # noqa: BLE001
            self.proc = None
            return
        # nvidia-smi's start-up (driver queries) must not fall inside the timed
        # region: wait for its first two samples (bounded)
        t0 = time.time()
        while len(self.lines) < 2 and time.time() - t0 < 10.0 and self.proc.poll() is None:
            time.sleep(0.05)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:  # noqa: BLE001
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nme, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nme)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
def build_workload(device, seed_offset=0, tile=8, workload=WORKLOAD):
    from powerfoam_b200 import synthetic

    return synthetic.raster_workload(workload, device, view=seed_offset)


class Args:
    is_pinhole = True
    render_objective = "volume"
    num_texel_sites = 8


class ArgsGeneric(Args):
    is_pinhole = False


def make_step(R, scene, cam, adj, adj_off, target_dev, world):
    from powerfoam_b200 import synthetic

    names = ["points", "radii", "density", "normals", "texel_sites", "texel_height"]
    params = {k: scene[k].clone().requires_grad_(True) for k in names}
    if world > 1:  # the adjoint writes into one flat buffer, all-reduced in place
        R.grad_buffer = GradBuffer(raster_fields(scene["points"].shape[0], scene["texel_sites"].shape[1]),
                                   scene["points"].device, world=world)

    def step(target=None, ready=None):
        t = target_dev if target is None else target
        for p in params.values():
            p.grad = None
        rgb = synthetic.texel_rgb(scene, cam).requires_grad_(True)
        out = R.forward(cam, None, params["points"], params["radii"], params["density"], params["normals"],
                        params["texel_sites"], rgb, params["texel_height"], adj, adj_off, None, False)
        if ready is not None:  # the target's upload, issued on a copy stream, is needed from here on
            torch.cuda.current_stream().wait_event(ready)
        loss = ((out[0] - t) ** 2).sum()
        loss.backward()
        if world > 1:
            R.grad_buffer.allreduce()
        return loss

    return step, params


def algorithmic_bytes(stats, H, W):
    """Per-launch algorithmic HBM bytes of the compositing forward and adjoint
    (the per-unit figures: 256 B of primitive record per visited (tile, prim)
    pair, 8 B per neighbour face record, 4 B per list entry; per pixel 32 B of
    forward outputs and 36 B of adjoint inputs; 2 x 256 B read-modify-write of
    the gradient record per pair with a contributing pixel)."""
    bins = stats["bins"]
    es = stats["early_stop"].long()
    offs = bins.tile_offsets
    T = es.shape[0]
    lens = offs[1:] - offs[:-1]
    tile_of = torch.repeat_interleave(torch.arange(T, device=offs.device), lens)
    n_pairs = int(bins.n_pairs)  # a device scalar after a sync-free call
    pos = torch.arange(n_pairs, device=offs.device) - offs[:-1][tile_of]
    visited = pos < es[tile_of]
    prims = bins.tile_prims[:n_pairs].long()[visited]
    ao = stats["adjacency_offsets"].long()
    deg = (ao[prims + 1] - ao[prims]).sum().item()
    V = int(visited.sum().item())
    U = int(stats["contrib_pairs"].long().sum().item())
    N = stats["n_prims"]
    fwd = 256 * V + 8 * deg + 4 * V + 8 * (T + 1) + 32 * H * W + 4 * N
    bwd = 256 * V + 8 * deg + 4 * V + 36 * H * W + 2 * 256 * U
    rec = segment_record_bytes(stats, visited)
    # the forward writes the segment records, the adjoint reads them (and skips the face records)
    if rec:
        fwd += rec["bytes"]
        bwd += rec["bytes"] - 8 * deg
    return dict(fwd=fwd, bwd=bwd, V=V, U=U, deg=deg, pairs=n_pairs, T=T, records=rec)


def segment_record_bytes(stats, visited):
    """Bytes of the segment records of the visited pairs: 8 B of hit mask and
    record offset per (pair, warp), 16 B per hit pixel with a record, 48 B of
    texture-plane result per such pixel whose clipped interval is not empty
    (counted from the records themselves)."""
    segs = stats.get("segments")
    if segs is None:
        return None
    seg, mask, offs, count, pairs, cap, planes = segs
    g = stats["tile_width"] ** 2 // 32
    vis = torch.nonzero(visited).flatten()
    m = mask.view(pairs, g)[vis].flatten().long() & 0xFFFFFFFF
    o = offs.view(pairs, g)[vis].flatten().long()
    bit = torch.arange(32, device=m.device)
    cnt = ((m[:, None] >> bit) & 1).sum(-1)
    ok = o >= 0
    clipped = int(((~ok) & (cnt > 0)).sum())  # hit (pair, warp)s the full buffer left without records
    cnt, o = cnt[ok], o[ok]
    n = int(cnt.sum())
    start = torch.cumsum(cnt, 0) - cnt
    idx = torch.repeat_interleave(o, cnt) + (torch.arange(n, device=m.device) - torch.repeat_interleave(start, cnt))
    r = seg.view(cap, -1)[idx, :3]
    ne = r[:, 0] < r[:, 1]
    ids = r[:, 2].contiguous().view(torch.int32)
    faced = int((ne & (((ids & 0xFFFF) >= 2) | ((ids >> 16) >= 2))).sum())  # a power face bounds it
    nonempty = int(ne.sum())
    b = 8 * vis.numel() * g + 16 * n + (48 * nonempty if planes else 0)
    return dict(bytes=b, hit_pixels=n, nonempty_pixels=nonempty, face_bounded_pixels=faced, capacity=cap,
                reserved=int(count.item()), clipped_again_pairs=clipped)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class OracleFrame:
    """The raster workload on the host, for the CPU baseline and the reference
    arm: scene, camera, texel colours (SH pre-step), Čech adjacency and target
    built on the CPU by the oracle (no GPU library loaded), and the oracle's
    binning + forward + adjoint timed in slices.  Slice k of S holds 1/S of a
    frame's work: the binning of every S-th primitive (k, k + S, ...) and the
    forward + adjoint of every S-th tile with its full list; S consecutive
    slices time one whole frame, every part of it once."""

    def __init__(self, workload, tile=8):
        from oracle import oracle as orc
        from powerfoam_b200 import synthetic

        self.orc = orc
        orc.build()
        cfg = synthetic.CONFIGS[workload]
        sc = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg.get("sigma", 0.15),
                                  r_range=cfg["r_range"], device="cpu")
        cam = synthetic.orbit_camera(100, cfg["width"], cfg["height"], cfg["vfov"], device="cpu")
        self.cfg, self.tile = cfg, tile
        n = {k: v.numpy() for k, v in sc.items()}
        eye = cam.eye.numpy()
        rgb = orc.sh_texel_rgb(n["points"], n["sh"], eye)
        self.sites = n["texel_sites"]
        self.sph = np.concatenate([n["points"], n["radii"][:, None]], -1).astype(np.float32)
        self.nsig = np.concatenate([n["normals"], n["density"][:, None]], -1).astype(np.float32)
        self.rgbh = np.concatenate([rgb, n["texel_height"][..., None]], -1).astype(np.float32)
        self.adj, self.adj_off = orc.cech_adjacency(n["points"], n["radii"])
        self.oc = orc.camera(eye, cam.right.numpy(), cam.up.numpy(), cam.width, cam.height)
        g = torch.Generator().manual_seed(200)
        self.target = torch.rand((cfg["height"], cfg["width"], 3), generator=g).numpy()
        # the frame's tile lists (the slices composite them); each slice re-bins its primitives in its timing
        keys, self.prims, self.offs, _ = orc.bin(self.oc, self.sph, tile)
        self.ad = orc.prefetch_adjacency(self.sph, self.adj, self.adj_off)
        self.T = self.offs.shape[0] - 1
        self.zeros = (np.zeros((cfg["height"], cfg["width"]), np.float32),
                      np.zeros((cfg["height"], cfg["width"], 3), np.float32), np.zeros(self.sph.shape[0], np.float32))

    def run_slice(self, k, S):
        """Seconds of slice k of S (binning of primitives k::S, neighbour
        records of their lists, forward + adjoint of tiles k::S)."""
        orc = self.orc
        tiles = np.arange(k, self.T, S)
        lens = np.zeros(self.T, np.int64)
        lens[tiles] = self.offs[tiles + 1] - self.offs[tiles]
        offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        prims = np.concatenate([self.prims[self.offs[t]:self.offs[t + 1]] for t in tiles]).astype(np.int32)
        sph_k = np.ascontiguousarray(self.sph[k::S])
        z, zn, zc = self.zeros
        t0 = time.perf_counter()
        orc.bin(self.oc, sph_k, self.tile)
        o = orc.raster_forward(self.oc, self.tile, self.sph, self.nsig, self.sites, self.rgbh, self.adj, self.adj_off,
                               self.ad, offs, prims)
        g_c = (2 * (o["color"] - self.target)).astype(np.float32)
        orc.raster_backward(self.oc, self.tile, self.sph, self.nsig, self.sites, self.rgbh, self.adj, self.adj_off,
                            self.ad, offs, prims, o["early_stop"], o["log_t"], g_c, z, z, zn, zc)
        return time.perf_counter() - t0


CPU_SLICES = 16


def cpu_baseline_line(frame, n_slices):
    """frames/s of the oracle over n_slices consecutive slices (1/CPU_SLICES
    of a frame each)."""
    t = sum(frame.run_slice(k % CPU_SLICES, CPU_SLICES) for k in range(n_slices))
    frac = n_slices / CPU_SLICES
    return dict(value=frac / t, unit=UNIT, cores=frame.orc.num_threads(), cpu=cpu_model(), kind="port",
                sample=(f"oracle (CPU restatement, OpenMP) binning + forward + adjoint of {n_slices}/{CPU_SLICES} "
                        f"of the frame (slices of every {CPU_SLICES}th primitive and tile), {frac:.2f} frames in "
                        f"{t:.2f} s; inputs built on the host"))


def reference_arm(args, rank, world):
    """The reference's algorithm on the host cores: the oracle (the CPU
    restatement of the reference's kernels; the reference's Warp kernels
    cannot be imported here) over slices of the frame, each timed step one
    slice (1/16 of the frame's work), frames/s = (steps / 16) / time."""
    if rank != 0:
        return
    frame = OracleFrame(args.workload, args.tile)
    for k in range(args.warmup):
        frame.run_slice(k % CPU_SLICES, CPU_SLICES)
    times = [frame.run_slice(k % CPU_SLICES, CPU_SLICES) for k in range(args.steps)]
    t = sum(times)
    v = (args.steps / CPU_SLICES) / t
    cb = dict(value=v, unit=UNIT, cores=frame.orc.num_threads(), cpu=cpu_model(), kind="port",
              sample=(f"{args.steps} steps, each 1/{CPU_SLICES} of the frame (binning of every {CPU_SLICES}th "
                      f"primitive, forward + adjoint of every {CPU_SLICES}th tile); {args.steps / CPU_SLICES:.2f} "
                      f"frames in {t:.2f} s"))
    line = dict(metric=METRIC, value=v, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=1000.0 * t / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic", impl="reference",
                config=dict(workload=args.workload, prims=frame.cfg["n"], width=frame.cfg["width"],
                            height=frame.cfg["height"], tile=args.tile, parallelism="cpu-openmp",
                            step=f"1/{CPU_SLICES} frame"),
                cpu_baseline=cb, e2e=dict(value=v, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                note=("the reference's Warp kernels are not importable on this image (no warp module); the "
                      "timed CPU implementation is the oracle, the reference's kernels restated in C"))
    print(json.dumps(line), flush=True)


def bin_launches(T, with_order=True):
    """Kernels one pf_bin call launches: count 1, depth sort 4 radix passes of 5
    kernels (histogram, 3-kernel scan, scatter), gather 1, scan 3, emit 1, tile
    sort ceil(log2(T)/8) passes, tile ranges 1; + 16 for the tile order (key
    kernel and 3 passes)."""
    bits = max(int(T - 1).bit_length(), 0)
    return 1 + 20 + 1 + 3 + 1 + 5 * ((bits + 7) // 8) + 1 + (16 if with_order else 0)


def batch_main(args, world, rank, local, dev):
    """Batched multi-view workload: 32 views of sizes drawn from {320x240,
    640x480, 1280x720, 1920x1080} of a 3,145,728-primitive scene (64-component
    mixture), one graph-captured step = SH pre-step + binning of every view +
    the persistent forward/loss/adjoint launch + SH adjoint.  Views are split
    round-robin over ranks; with N > 1 the gradients are all-reduced (NCCL)."""
    from powerfoam_b200 import synthetic
    from powerfoam_b200.adjacency import CechBuilder
    from powerfoam_b200.batch import autotune

    cfg = synthetic.CONFIGS[args.workload]
    scene = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"],
                                 r_range=cfg["r_range"], device=dev)
    cams_all = synthetic.batch_cameras(cfg["views"], cfg["seed"], cfg["vfov"], device=dev)
    mine = shard_views(len(cams_all), rank, world)
    cams = [cams_all[v] for v in mine]
    adj, adj_off = CechBuilder(dev)(scene["points"], scene["radii"])
    g = torch.Generator().manual_seed(300)
    targets_host = [torch.rand((c.height, c.width, 3), generator=g) for c in cams_all]
    targets_host = [targets_host[v].pin_memory() for v in mine]
    targets = [t.to(dev) for t in targets_host]
    kw = dict(points=scene["points"], radii=scene["radii"], density=scene["density"], normals=scene["normals"],
              texel_sites=scene["texel_sites"], texel_height=scene["texel_height"], adjacency=adj,
              adjacency_offsets=adj_off, targets=targets, sh=scene["sh"])
    t0 = time.perf_counter()
    if args.no_autotune:
        from powerfoam_b200.batch import BatchStep

        step = BatchStep(dev, cams, args.tile, 1, "longest", record_segments=not args.no_segment_records)
        step.bind(**kw)
        table = []
    else:
        step, table = autotune(dev, cams, kw, chunks=(1, 4), iters=1, warmup=1,
                               record_segments=not args.no_segment_records,
                               log=(lambda m: print(m, file=sys.stderr, flush=True)) if rank == 0 else None)
    tune_s = time.perf_counter() - t0
    step.capture()

    def run():
        loss = step.run()
        if world > 1:  # the step's gradients live in one flat buffer: summed in place
            step.grad_buffer.allreduce()
        return loss

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(max(args.warmup, 3)):
        run()
    barrier()
    step.check()
    if step.graph is None:  # check() grew the segment record buffer: capture the step again
        step.capture()
        for _ in range(max(args.warmup, 3)):
            run()
        barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        run()
    b.record()
    barrier()
    clk = clocks.stop()
    ms = a.elapsed_time(b) / args.steps
    # end to end: every view's target image from pinned host memory in, the per-view losses out
    loss_host = torch.empty((args.steps, len(cams)), dtype=torch.float32).pin_memory()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        for t_dev, t_host in zip(step.targets, targets_host):
            t_dev.copy_(t_host, non_blocking=True)
        loss = run()
        loss_host[i].copy_(loss, non_blocking=True)
    e1.record()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        ms, e2e_ms = max_over_ranks(ms, dev), max_over_ranks(e2e_ms, dev)
    # live kernel time of the persistent launch (eager runs, events around it)
    step.kernel_events = []
    for _ in range(3):
        step._launch()
    torch.cuda.synchronize()
    k_ms = statistics.mean(x.elapsed_time(y) for x, y in step.kernel_events)
    step.kernel_events = None
    # the same work as separate per-view calls (SH pre-step, Rasterizer forward, loss, backward), for comparison
    from powerfoam_b200 import rasterize

    R = rasterize.Rasterizer(Args(), dev, tile_width=step.tile_width)
    pnames = ["points", "radii", "density", "normals", "texel_sites", "texel_height"]
    params = {k: scene[k].clone().requires_grad_(True) for k in pnames}

    def per_view_pass():
        for v, c in enumerate(cams):
            rgb = synthetic.texel_rgb(scene, c).requires_grad_(True)
            out = R.forward(c, None, params["points"], params["radii"], params["density"], params["normals"],
                            params["texel_sites"], rgb, params["texel_height"], adj, adj_off, None, False)
            ((out[0] - step.targets[v]) ** 2).sum().backward()

    per_view_pass()
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    per_view_pass()
    s1.record()
    torch.cuda.synchronize()
    sequential_ms = s0.elapsed_time(s1)
    del R, params
    V = len(cams)
    n_groups = step.seg_groups[-1] + 1 if step.segs is not None else 1
    # pack 1, neighbour encoding 1, SH pre-step V, binning per view, the batch launch (work list: keys 1
    # + three 5-kernel radix passes when ordered by length; per record group the persistent kernel once
    # fused, or forward + adjoint split, the adjoint as two launches with segment records; 6 + V
    # sanitise), SH adjoint V
    per_step = 1 + 1 + V + sum(bin_launches(T, with_order=False) for T in step.n_tiles)
    per_step += 1 + (15 if step.order == "longest" else 0)
    per_step += n_groups * ((3 if step.segs else 2) if step.split else 1)
    per_step += 6 + V + V
    groups_info = None if step.segs is None else dict(groups=n_groups, capacity=step.segs[1], planes=step.segs[2],
                                                      view_records=step.view_records)
    totals = dict(alg=0, pairs=0, rec_bytes=0, rec_hits=0, rec_clipped=0)

    def add_view_bytes(s, v, c):
        """Algorithmic bytes of view v of BatchStep s (its slice of the masks
        and offsets; its group's counter)."""
        class _B:
            pass
        bins = _B()
        bins.tile_offsets = s.tile_offsets[v]
        n_p = int(s.bin_scalars[v, 0])
        bins.tile_prims = s.tile_prims[v][:n_p]
        bins.n_pairs = n_p
        totals["pairs"] += n_p
        segs = None
        if s.segs is not None:
            g = s.tile_width ** 2 // 32
            base, cap_v = sum(s.capacity[:v]), s.capacity[v]
            sl = slice(base * g, (base + cap_v) * g)
            grp = s.seg_groups[v]
            segs = (s.segs[0], s.seg_masks[sl], s.seg_offs[sl], s.rec_count[grp:grp + 1], cap_v, s.segs[1],
                    s.segs[2])
        st = algorithmic_bytes(dict(bins=bins, early_stop=s.early_stop[v], adjacency_offsets=adj_off,
                                    contrib_pairs=s.tile_contrib_pairs[v], n_prims=cfg["n"], segments=segs,
                                    tile_width=s.tile_width), c.height, c.width)
        totals["alg"] += st["fwd"] + st["bwd"]
        if st["records"]:
            totals["rec_bytes"] += st["records"]["bytes"]
            totals["rec_hits"] += st["records"]["hit_pixels"]
            totals["rec_clipped"] += st["records"]["clipped_again_pairs"]

    if n_groups == 1:
        for v, c in enumerate(cams):
            add_view_bytes(step, v, c)
    else:
        # the record buffer holds the last group's records only: each group's are counted on a
        # step over that group's views (untimed)
        from powerfoam_b200.batch import BatchStep

        groups = list(step.seg_groups)
        sched = dict(tile_width=step.tile_width, chunk=step.chunk, order=step.order, split=step.split)
        step.graph = None
        step.segs = None
        step.seg_masks = step.seg_offs = None
        torch.cuda.empty_cache()
        for g in range(n_groups):
            vs = [v for v in range(V) if groups[v] == g]
            sub = BatchStep(dev, [cams[v] for v in vs], **sched)
            sub.bind(**dict(kw, targets=[targets[v] for v in vs]))
            sub.run()
            torch.cuda.synchronize()
            groups_info.setdefault("sub_step_groups", []).append(sub.seg_groups[-1] + 1)
            for i, v in enumerate(vs):
                add_view_bytes(sub, i, cams[v])
            del sub
            torch.cuda.empty_cache()
    alg, pairs = totals["alg"], totals["pairs"]
    rec_bytes, rec_hits, rec_clipped = totals["rec_bytes"], totals["rec_hits"], totals["rec_clipped"]
    peak, peak_kind = load_peaks()
    achieved = alg / (k_ms * 1e-3) / 1e9
    n_views = len(cams_all)
    pixels = sum(c.width * c.height for c in cams_all)
    line = dict(metric="batched multi-view fwd+bwd, views/s", value=n_views * 1000.0 / ms,
                unit="views/s (32 views per step)", n_gpus=world, steps=args.steps, warmup=max(args.warmup, 3),
                ms_per_step=ms, higher_is_better=True, scaling="strong", vs_baseline=None, dtype="f32",
                data="synthetic (seeded scene, orbit cameras, uniform targets)",
                config=dict(workload=args.workload, prims=cfg["n"], views=n_views, pixels=pixels, pairs=pairs,
                            tile=step.tile_width, chunk=step.chunk, order=step.order, split=step.split,
                            autotune_s=tune_s,
                            per_view_calls_ms=sequential_ms,
                            segment_records=None if groups_info is None else dict(
                                groups_info, hit_pixels=rec_hits, bytes=rec_bytes, clipped_again_pairs=rec_clipped),
                            autotune=table, graph="one CUDA graph per step",
                            l2="inputs larger than L2 (805 MB of primitive records), no flush",
                            parallelism=f"view-dp{world}"),
                clocks=clk,
                e2e=dict(value=n_views * 1000.0 / e2e_ms, unit="views/s",
                         h2d_bytes_per_step=sum(t.numel() * 4 for t in targets_host),
                         d2h_bytes_per_step=4 * len(cams)),
                roofline=dict(bound="hbm", kernel="pf_batch_render", achieved=achieved, peak=peak, unit="GB/s",
                              frac=achieved / peak, peak_source=peak_kind, traffic=None, algorithmic_bytes=alg,
                              ms=k_ms),
                gpu_launches=args.steps * per_step)
    if rank == 0:
        print(json.dumps(line), flush=True)
    step.graph = None
    if world > 1:
        torch.distributed.destroy_process_group()


def proposal_main(args, dev):
    """Proposal-seeded vs plain cell walk (one GPU): the 64-cluster scene of
    the tracer configuration (σ 0.1, r log-uniform in [0.001, 0.01], 10 %
    background) with its power-diagram adjacency, the network trained for 5000
    Adam steps of 65,536 rays on 2M rays labelled by the plain walk (2048
    random 32x32 views, first cell with transmittance < 0.999), its confidence
    gate calibrated on 256 held-out views, then one 2048x1536 frame from a
    held-out view.  Reported: plain and seeded frame times (the seeded time
    includes the network forward and the cell location), PSNR of the seeded
    frame against the plain one, and the same for seeding from the plain
    walk's own labels (the bound a perfect proposal reaches), for the
    occupancy-grid seeding (the conservative proposal without a network) and
    for the network with the occupancy seeding as its fallback."""
    from powerfoam_b200 import synthetic
    from powerfoam_b200.adjacency import power_adjacency, power_adjacency_diff, start_cell
    from powerfoam_b200.proposal import (OccupancySeeder, ProposalNet, SeededTracer, box_exit, camera_rays,
                                         make_training_rays, trace_labels)
    from powerfoam_b200.raytrace import RayTracer

    cfg = dict(synthetic.CONFIGS["trace6m"])
    if args.proposal_prims:
        s = (cfg["n"] / args.proposal_prims) ** (1 / 3)
        cfg["n"] = args.proposal_prims
        cfg["r_range"] = tuple(r * s for r in cfg["r_range"])
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    shells = (0.12, 0.02, 30.0) if args.proposal_scene == "shells" else None
    sc = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"],
                              r_range=cfg["r_range"], device=dev, shells=shells)
    t0 = time.perf_counter()
    adj, off = power_adjacency(sc["points"], sc["radii"])
    log(f"power adjacency {time.perf_counter() - t0:.1f} s, {adj.shape[0]} edges")
    pm = power_adjacency_diff(sc["points"], sc["radii"], adj, off)
    ev = synthetic.orbit_camera(4242, cfg["width"], cfg["height"], cfg["vfov"], device=dev)
    rgb = synthetic.texel_rgb(sc, ev)
    scene_args = (sc["points"], sc["radii"], sc["density"], sc["normals"], sc["texel_sites"], rgb,
                  sc["texel_height"], adj, off, pm)
    tr = RayTracer(Args(), dev)

    box = (sc["points"].min(0).values, sc["points"].max(0).values)

    def labelled(seed0, k):
        cams = [synthetic.orbit_camera(seed0 + i, 32, 32, cfg["vfov"], device=dev) for i in range(k)]
        return make_training_rays(tr, cams, scene_args, [start_cell(sc["points"], sc["radii"], c.eye) for c in cams],
                                  label_transmittance=0.999, box=box)

    t0 = time.perf_counter()
    rays8, val = labelled(10000, 2048), labelled(50000, 256)
    label_s = time.perf_counter() - t0
    net = ProposalNet(dev, seed=1)
    t0 = time.perf_counter()
    hist = net.train(rays8, steps=5000, batch=65536, lr=1e-3, overshoot_weight=100.0, margin=0.1, graph_steps=100)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    seeded = SeededTracer(tr, net, sc["points"], sc["radii"], conf_threshold=net.calibrate(val),
                          adjacency=adj, adjacency_offsets=off)
    torch.cuda.synchronize()
    vmap_s = time.perf_counter() - t0
    st = start_cell(sc["points"], sc["radii"], ev.eye)

    def timed(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            r = fn()
        b.record()
        torch.cuda.synchronize()
        return r, a.elapsed_time(b) / args.steps

    def psnr(a, b):
        mse = float(((a.double() - b.double()) ** 2).mean())
        return 10 * math.log10(1.0 / max(mse, 1e-20))

    plain, plain_ms = timed(lambda: tr.trace(ev, st, *scene_args, check_status=False))
    seeded.n_seeded.zero_()
    seed_r, seed_ms = timed(lambda: seeded.render(ev, st, scene_args))
    n_seeded = int(seeded.n_seeded.item()) // (args.steps + max(args.warmup, 3))
    lab = trace_labels(tr, ev, st, scene_args, label_transmittance=0.999)
    hit = lab["label_cell"] >= 0
    # where the plain walk's cells go: rays that never reach a significant cell, and the cells
    # hit rays walk before their first significant one (what a proposal can skip)
    vc = plain.visit_count
    stats = dict(nohit_rays=int((~hit).sum()), cells_nohit_rays=int(vc[~hit].sum()),
                 cells_before_label=int(lab["label_step"][hit].sum()))
    one = torch.ones_like(lab["label_t"])
    # the bound of a perfect proposal: hit rays seeded at their first significant cell, the others
    # where they leave the primitives' box
    t_exit = box_exit(camera_rays(ev), box[0], box[1]).view_as(lab["label_t"])
    t_lab = (torch.where(hit, lab["label_t"], t_exit) - net.margin).contiguous()
    conf_lab = one.contiguous()
    ideal_r, ideal_ms = timed(lambda: tr.trace(ev, seeded.locator.seed(ev, t_lab, conf_lab, 0.5, st), *scene_args,
                                                check_status=False))
    # the two parts of the label-seeded frame: locating the seeds, and the walk from them
    ideal_start, locate_ms = timed(lambda: seeded.locator.seed(ev, t_lab, conf_lab, 0.5, st))
    _, ideal_walk_ms = timed(lambda: tr.trace(ev, ideal_start, *scene_args, check_status=False))
    # the conservative proposal without a network (occupancy grid), alone and as the gate's fallback
    t0 = time.perf_counter()
    occ = OccupancySeeder(sc["points"], sc["radii"], sc["density"], seeded.locator, res=128)
    torch.cuda.synchronize()
    occ_build_s = time.perf_counter() - t0
    occ_r, occ_ms = timed(lambda: tr.trace(ev, occ.start_cells(ev, st), *scene_args, check_status=False))
    seeded.occupancy = occ
    comb_r, comb_ms = timed(lambda: seeded.render(ev, st, scene_args))
    seeded.occupancy = None
    H, W = cfg["height"], cfg["width"]
    line = dict(metric=METRIC, value=plain_ms / seed_ms, unit="x (plain / proposal-seeded frame time)", n_gpus=1,
                steps=args.steps, warmup=max(args.warmup, 3), ms_per_step=seed_ms, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f32 walk, bf16 network", data="synthetic",
                config=dict(workload="proposal", scene=args.proposal_scene, prims=cfg["n"], width=W, height=H,
                            plain_ms=plain_ms,
                            seeded_ms=seed_ms, psnr_db=psnr(seed_r.color, plain.color), seeded_rays=n_seeded,
                            rays=H * W, threshold=seeded.conf_threshold, cells_plain=int(plain.visit_count.sum()),
                            cells_seeded=int(seed_r.visit_count.sum()), label_seed_ms=ideal_ms, label_seed_locate_ms=locate_ms,
                            label_seed_walk_ms=ideal_walk_ms,
                            label_seed_psnr_db=psnr(ideal_r.color, plain.color),
                            label_seed_cells=int(ideal_r.visit_count.sum()), label_s=label_s, train_s=train_s,
                            train_rays=int(rays8.shape[0]), loss_first=hist[0], loss_last=hist[-1],
                            voxel_map_s=vmap_s, occupancy_ms=occ_ms, occupancy_psnr_db=psnr(occ_r.color, plain.color),
                            occupancy_cells=int(occ_r.visit_count.sum()), occupancy_build_s=occ_build_s,
                            network_occupancy_ms=comb_ms,
                            network_occupancy_psnr_db=psnr(comb_r.color, plain.color),
                            network_occupancy_cells=int(comb_r.visit_count.sum()), **stats))
    print(json.dumps(line), flush=True)


def trace_main(args, dev):
    """Tracer forward + adjoint (config 2): the 1,048,576-primitive scene of
    the rasterizer workload with its power-diagram adjacency (built on the
    GPU once, the neighbour sets of the reference's hull construction), one 1280x720 camera on the radius-3 orbit at a seeded
    azimuth / elevation, walks from the camera's cell; one step = the walk
    (colour, log transmittance, depth, normal), an L2 loss against a seeded
    uniform target and the hand-written adjoint to every primitive gradient."""
    from powerfoam_b200 import synthetic
    from powerfoam_b200.adjacency import power_adjacency, power_adjacency_diff, start_cell
    from powerfoam_b200.raytrace import RayTracer

    cfg = synthetic.CONFIGS["trace1m"]
    shells = (0.12, 0.02, 30.0) if args.proposal_scene == "shells" else None
    sc = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"],
                              r_range=cfg["r_range"], device=dev, shells=shells)
    t0 = time.perf_counter()
    adj, off = power_adjacency(sc["points"], sc["radii"])
    torch.cuda.synchronize()
    adj_s = time.perf_counter() - t0
    pm = power_adjacency_diff(sc["points"], sc["radii"], adj, off)
    cam = synthetic.orbit_camera(2, cfg["width"], cfg["height"], cfg["vfov"], device=dev)
    rgb = synthetic.texel_rgb(sc, cam)
    st = start_cell(sc["points"], sc["radii"], cam.eye)
    tr = RayTracer(Args(), dev)
    tr.host_sync = args.host_sync  # default: the forward never waits on the host; checked after the timing
    names = ["points", "radii", "density", "normals", "texel_sites", "texel_height"]
    params = {k: sc[k].clone().requires_grad_(True) for k in names}
    rgb_p = rgb.clone().requires_grad_(True)
    g = torch.Generator().manual_seed(202)
    target_host = torch.rand((cfg["height"], cfg["width"], 3), generator=g).pin_memory()
    target = target_host.to(dev)

    def step(t=None, ready=None):
        for p in list(params.values()) + [rgb_p]:
            p.grad = None
        color, log_t, depth, normal = tr.forward(cam, st, params["points"], params["radii"], params["density"],
                                                 params["normals"], params["texel_sites"], rgb_p,
                                                 params["texel_height"], adj, off, pm)
        if ready is not None:  # the target's upload on the copy stream
            torch.cuda.current_stream().wait_event(ready)
        loss = ((color - (target if t is None else t)) ** 2).sum()
        loss.backward()
        return loss

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        step()
    b.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    tr.check()  # a walk stopped early in any timed step raises here
    ms = a.elapsed_time(b) / args.steps
    # targets uploaded on a copy stream into two buffers, as in the rasterizer workload
    t_dev = [torch.empty_like(target) for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    ready = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]
    loss_host = torch.empty(args.steps, dtype=torch.float32).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for i in range(args.steps):
        b = i % 2
        copy_stream.wait_event(e0 if i < 2 else consumed[b])
        with torch.cuda.stream(copy_stream):
            t_dev[b].copy_(target_host, non_blocking=True)
            ready[b].record(copy_stream)
        loss = step(t_dev[b], ready[b])
        consumed[b].record()
        loss_host[i].copy_(loss.detach(), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    tr.check()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    r = tr.trace(cam, st, sc["points"], sc["radii"], sc["density"], sc["normals"], sc["texel_sites"], rgb,
                 sc["texel_height"], adj, off, pm)
    steps_total = int(r.visit_count.sum())
    deg = (off[1:] - off[:-1]).float().mean().item()
    line = dict(metric="tracer fwd+bwd ms/iter @1M prims 720p", value=1000.0 / ms, unit="frames/s (fwd+bwd)",
                n_gpus=1, steps=args.steps, warmup=max(args.warmup, 3), ms_per_step=ms, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                config=dict(workload="trace1m", prims=cfg["n"], width=cfg["width"], height=cfg["height"],
                            cells_walked=steps_total, mean_degree=deg, adjacency_s=adj_s,
                            l2="inputs larger than L2, no flush"),
                clocks=clk, e2e=dict(value=1000.0 / e2e_ms, unit="frames/s", h2d_bytes_per_step=target.numel() * 4,
                                     d2h_bytes_per_step=4),
                # per step: the recording walk (pf_trace_forward_record), then the adjoint's segment and
                # resume launches and seven gradient sanitising launches (pf_trace_backward_recorded)
                gpu_launches=args.steps * (1 + 2 + 7))
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = trace_cpu_baseline(sc, rgb, adj, off, pm, cam, st, cfg)
    print(json.dumps(line), flush=True)


def trace_cpu_baseline(sc, rgb, adj, off, pm, cam, start, cfg, w=None, h=None):
    """The oracle's tracer (CPU restatement, OpenMP over rays) forward + L2
    adjoint of the same view and frustum at w x h rays (default: the whole
    image, about 6 s on 16 host threads), scaled to the full image by ray
    count."""
    from oracle import oracle as orc

    w, h = w or cfg["width"], h or cfg["height"]
    orc.build()
    n = lambda t: t.detach().cpu().numpy()  # noqa: E731
    sph = np.concatenate([n(sc["points"]), n(sc["radii"])[:, None]], -1).astype(np.float32)
    nsig = np.concatenate([n(sc["normals"]), n(sc["density"])[:, None]], -1).astype(np.float32)
    oc = orc.camera(n(cam.eye), n(cam.right), n(cam.up), w, h)
    args = (oc, sph, nsig, n(sc["texel_sites"]), n(rgb), n(sc["texel_height"]), n(adj), n(off),
            n(pm).view(np.uint16))
    t0 = time.perf_counter()
    f = orc.trace_forward(*args, int(start), thr=1e-3)
    g_c = (2.0 * (f["color"] - np.random.default_rng(202).uniform(0, 1, f["color"].shape))).astype(np.float32)
    orc.trace_backward(*args, f, g_c, None, None, None, int(start), thr=1e-3)
    t_sample = time.perf_counter() - t0
    t = t_sample * (cfg["width"] * cfg["height"]) / (w * h)
    return dict(value=1.0 / t, unit="frames/s (fwd+bwd)", cores=orc.num_threads(), kind="port",
                sample=(f"oracle walk + adjoint of the same view at {w}x{h} rays ({t_sample:.2f}s), "
                        f"scaled to {cfg['width']}x{cfg['height']}"))


def interpen_main(args, dev):
    """Interpenetration loss forward + adjoint: the 3,145,728-primitive scene
    of the batched workload with its Čech adjacency (built on the GPU, once);
    one step = areas of every sphere, their sum (the trainer's loss term,
    train.py:277) and the adjoint to points and radii through the autograd
    mirror."""
    from oracle import oracle as orc
    from powerfoam_b200 import synthetic
    from powerfoam_b200.adjacency import CechBuilder
    from powerfoam_b200.geometry import InterpenetrationFunction

    cfg = synthetic.CONFIGS["batch3m"]
    sc = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"],
                              r_range=cfg["r_range"], device=dev)
    adj, off = CechBuilder(dev)(sc["points"], sc["radii"])
    n, e = cfg["n"], adj.numel()
    pts = sc["points"].clone().requires_grad_(True)
    radii = sc["radii"].clone().requires_grad_(True)
    events = {"fwd": [], "bwd": []}

    def step(record=False):
        pts.grad = None
        radii.grad = None
        if record:
            a0, a1, b1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a0.record()
        loss = InterpenetrationFunction.apply(pts, radii, adj, off).sum()
        if record:
            a1.record()
        loss.backward()
        if record:
            b1.record()
            events["fwd"].append((a0, a1))
            events["bwd"].append((a1, b1))
        return loss

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        step()
    b.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = a.elapsed_time(b) / args.steps
    for _ in range(args.steps):
        step(record=True)
    torch.cuda.synchronize()
    fwd_ms = statistics.mean(x.elapsed_time(y) for x, y in events["fwd"])
    bwd_ms = statistics.mean(x.elapsed_time(y) for x, y in events["bwd"])
    loss_host = torch.empty(args.steps, dtype=torch.float32).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for i in range(args.steps):
        loss_host[i].copy_(step().detach(), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    # unique bytes a launch must move: spheres, offsets, lists, areas (or
    # dL/dareas) and, for the adjoint, the (N,4) gradient written once
    fwd_bytes = 16 * n + 4 * (n + 1) + 4 * e + 4 * n
    bwd_bytes = fwd_bytes + 16 * n
    peak, peak_kind = load_peaks()
    dom = "bwd" if bwd_ms >= fwd_ms else "fwd"
    dom_ms, dom_bytes = (bwd_ms, bwd_bytes) if dom == "bwd" else (fwd_ms, fwd_bytes)
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    line = dict(metric="interpenetration loss fwd+bwd @3.1M prims", value=1000.0 / ms, unit="iterations/s",
                n_gpus=1, steps=args.steps, warmup=max(args.warmup, 3), ms_per_step=ms, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f32", data="synthetic (seeded scene, GPU Čech lists)",
                config=dict(workload="interpen3m", prims=n, pairs=e, mean_degree=e / n,
                            l2="inputs larger than L2 (50 MB spheres + lists), no flush"),
                clocks=clk,
                e2e=dict(value=1000.0 / e2e_ms, unit="iterations/s", h2d_bytes_per_step=0, d2h_bytes_per_step=4,
                         note="the scene is training state resident on the device; the loss is read back"),
                roofline=dict(bound="hbm", kernel="pf_interpenetration" + ("_backward" if dom == "bwd" else ""),
                              achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                              peak_source=peak_kind, traffic=None, algorithmic_bytes=dom_bytes, ms=dom_ms,
                              fwd_ms=fwd_ms, bwd_ms=bwd_ms),
                gpu_launches=args.steps * 2)
    if not args.no_cpu_baseline:
        sph = torch.cat([sc["points"], sc["radii"][:, None]], -1).cpu().numpy()
        a_np, o_np = adj.cpu().numpy(), off.cpu().numpy()
        m = min(n, 1 << 19)
        t0 = time.perf_counter()
        orc.interpenetration(sph, a_np, o_np, rows=m)
        orc.interpenetration_backward(sph, a_np, o_np, np.ones(n, np.float32), rows=m)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = dict(value=(m / n) / dt, unit="iterations/s", cores=1, kind="port",
                                    sample=f"the lists of the first {m} spheres, forward + adjoint (oracle, one "
                                           "thread), scaled by the sphere share")
    print(json.dumps(line), flush=True)


def power_main(args, dev):
    """Power-diagram adjacency of the 1,048,576-primitive rasterizer scene on
    the GPU (pf_power_adjacency; one step = one full build: grid, cells,
    symmetric CSR lists), against the reference's construction (lifted 4-D
    hull by scipy's Qhull on one host core, benchmark.py:25-83) on a bounded
    subset."""
    from powerfoam_b200 import synthetic
    from oracle.power_hull import build_power_adjacency
    from powerfoam_b200.adjacency import PowerBuilder

    cfg = synthetic.CONFIGS["raster1m"]
    sc = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"],
                              r_range=cfg["r_range"], device=dev)
    pts, radii = sc["points"], sc["radii"]
    b = PowerBuilder(dev)
    for _ in range(max(args.warmup, 3)):
        adj, off = b(pts, radii)
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        adj, off = b(pts, radii)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clk = clocks.stop()
    ms = statistics.mean(times)
    # end to end: host points and radii in, host lists out
    pts_h, radii_h = pts.cpu().pin_memory(), radii.cpu().pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        a_d, o_d = b(pts_h.to(dev, non_blocking=True), radii_h.to(dev, non_blocking=True))
        a_h, o_h = a_d.cpu(), o_d.cpu()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    n, e = cfg["n"], adj.numel()
    line = dict(metric="power-diagram adjacency build @1M prims", value=1000.0 / ms, unit="builds/s", n_gpus=1,
                steps=args.steps, warmup=max(args.warmup, 3), ms_per_step=ms, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic (seeded raster1m scene)",
                config=dict(workload="power1m", prims=n, directed_edges=e, mean_degree=e / n,
                            l2="compute-bound build; inputs 16 MB, no flush"),
                clocks=clk,
                e2e=dict(value=1000.0 / e2e_ms, unit="builds/s", h2d_bytes_per_step=16 * n,
                         d2h_bytes_per_step=4 * (e + n + 1)),
                # per build: grid (bounds init, bounds, grid, cell keys, 3 radix passes of 5 kernels, cell
                # ranges), cell weights 2, cells, symmetrize, count, scan 3, write, offsets
                gpu_launches=args.steps * (4 + 15 + 1 + 2 + 1 + 1 + 1 + 3 + 1 + 1))
    if not args.no_cpu_baseline:
        m = 1 << 17
        sub = torch.randperm(n, generator=torch.Generator().manual_seed(0))[:m]
        p_s, r_s = pts.cpu()[sub], radii.cpu()[sub]
        t0 = time.perf_counter()
        build_power_adjacency(p_s, r_s)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = dict(value=(m / n) / dt, unit="builds/s", cores=1, kind="reference",
                                    sample=f"the reference's hull construction (scipy Qhull) on {m} of the {n} "
                                           "primitives, scaled by the point share (Qhull is superlinear, so this "
                                           "overstates its full-size rate)")
    print(json.dumps(line), flush=True)


def color_main(args, dev):
    """Spherical-Voronoi texel colour forward + adjoint (color_fn.py) for the
    texel sites of the 1,048,576-primitive scene: 8 sites per primitive
    (8,388,608 points), sv_dof 8, float32 attributes, seeded; one step =
    colours of every texel, an L2 loss and the site gradients."""
    from powerfoam_b200 import synthetic
    from powerfoam_b200.color_fn import SphericalVoronoi

    cfg = synthetic.CONFIGS["raster1m"]
    sc = synthetic.make_scene(cfg["n"], seed=cfg["seed"], mixture=cfg["mixture"], sigma=cfg["sigma"],
                              r_range=cfg["r_range"], device=dev)
    cam = synthetic.orbit_camera(100, cfg["width"], cfg["height"], cfg["vfov"], device=dev)
    pts = sc["texel_sites"].reshape(-1, 3).contiguous()
    n, dof = pts.shape[0], 8
    g = torch.Generator(device=dev).manual_seed(7)
    ax = torch.randn(dof, n, 3, device=dev, generator=g)
    sites = (ax / ax.norm(dim=-1, keepdim=True)).requires_grad_(True)
    values = (0.3 * torch.randn(dof, n, 3, device=dev, generator=g)).requires_grad_(True)
    temps = (1.0 + 9.0 * torch.rand(dof, n, device=dev, generator=g)).requires_grad_(True)
    target = torch.rand(n, 3, device=dev, generator=g)

    class SvArgs:
        sv_dof = dof

    sv = SphericalVoronoi(SvArgs(), dev)
    events = {"fwd": [], "bwd": []}

    def step(record=False):
        for t in (sites, values, temps):
            t.grad = None
        if record:
            a0, a1, b1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a0.record()
        col = sv.forward(pts, cam, sites, values, temps)
        if record:
            a1.record()
        loss = ((col - target) ** 2).sum()
        loss.backward()
        if record:
            b1.record()
            events["fwd"].append((a0, a1))
            events["bwd"].append((a1, b1))
        return loss

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        step()
    b.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = a.elapsed_time(b) / args.steps
    for _ in range(args.steps):
        step(record=True)
    torch.cuda.synchronize()
    fwd_ms = statistics.mean(x.elapsed_time(y) for x, y in events["fwd"])
    bwd_ms = statistics.mean(x.elapsed_time(y) for x, y in events["bwd"])
    # unique bytes: points 12, per site axis 12 + value 12 + temperature 4; forward writes colour 12 + weight
    # sum 4; the adjoint also reads those and the colour gradient (12) and writes the 28 B of site gradients
    fwd_bytes = n * (12 + dof * 28 + 16)
    bwd_bytes = n * (12 + dof * 28 + 28) + n * dof * 28
    peak, peak_kind = load_peaks()
    dom_ms, dom_bytes, kern = ((bwd_ms, bwd_bytes, "pf_sv_backward") if bwd_ms >= fwd_ms
                               else (fwd_ms, fwd_bytes, "pf_sv_forward"))
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    loss_host = torch.empty(args.steps, dtype=torch.float32).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for i in range(args.steps):
        loss_host[i].copy_(step().detach(), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    line = dict(metric="spherical-Voronoi texel colour fwd+bwd @8.4M texels", value=1000.0 / ms,
                unit="iterations/s", n_gpus=1, steps=args.steps, warmup=max(args.warmup, 3), ms_per_step=ms,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                data="synthetic (texel sites of the seeded raster1m scene, seeded sites / values / temperatures)",
                config=dict(workload="color1m", points=n, sv_dof=dof,
                            l2="inputs larger than L2 (1.9 GB of site attributes), no flush"),
                clocks=clk,
                e2e=dict(value=1000.0 / e2e_ms, unit="iterations/s", h2d_bytes_per_step=0, d2h_bytes_per_step=4,
                         note="attributes are training state resident on the device; the loss is read back"),
                roofline=dict(bound="hbm", kernel=kern, achieved=achieved, peak=peak, unit="GB/s",
                              frac=achieved / peak, peak_source=peak_kind, traffic=None, algorithmic_bytes=dom_bytes,
                              ms=dom_ms, fwd_ms=fwd_ms, bwd_ms=bwd_ms),
                gpu_launches=args.steps * 2)
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    if args.workload == "proposal":
        proposal_main(args, dev)
        return
    if args.workload == "trace1m":
        trace_main(args, dev)
        return
    if args.workload == "interpen3m":
        interpen_main(args, dev)
        return
    if args.workload == "power1m":
        power_main(args, dev)
        return
    if args.workload == "color1m":
        color_main(args, dev)
        return
    if args.workload.startswith("batch"):
        batch_main(args, world, rank, local, dev)
        return
    from powerfoam_b200 import rasterize

    fisheye = args.workload == "fisheye1m"
    cfg, scene, cam, adj, adj_off, target = build_workload(dev, rank, args.tile,
                                                           "raster1m" if fisheye else args.workload)
    target_dev = target.to(dev)
    if fisheye:
        # the same scene and view through a 150-degree equidistant fisheye (generic camera)
        from powerfoam_b200 import synthetic

        cam.ray_maps = synthetic.fisheye_ray_maps(cam, 150.0)
        args.no_cpu_baseline = True
    R = rasterize.Rasterizer(ArgsGeneric() if fisheye else Args(), dev, tile_width=args.tile,
                             host_sync=args.host_sync)
    R.record_segments = not args.no_segment_records
    step, params = make_step(R, scene, cam, adj, adj_off, target_dev, world)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(max(args.warmup, 3)):
        step()
    barrier()
    # --graph: the whole step (colour pre-step, binning, forward, loss, adjoint) captured in
    # CUDA graphs, one per target buffer of the end-to-end loop; graph 0 reads the resident
    # target.  Possible because the step runs sync-free (nothing is read back per call).
    t_dev = [target_dev, torch.empty_like(target_dev)]
    graphs = None
    if args.graph:
        if world > 1 or args.host_sync:
            raise SystemExit("--graph: one GPU and the sync-free step only")
        t_dev[1].copy_(target_dev)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(2):
                step(t_dev[0])
                step(t_dev[1])
        torch.cuda.current_stream().wait_stream(side)
        graphs = []
        for b in range(2):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                lo = step(t_dev[b])
            graphs.append((g, lo))
        for _ in range(max(args.warmup, 3)):
            graphs[0][0].replay()
        barrier()

    # per-call device times of the compositing kernels, recorded live (eagerly after the
    # timed loop when it replays graphs)
    events = {"pf_raster_forward": [], "pf_raster_backward": []}
    pending = {}

    def hook(name, phase):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        if phase == "begin":
            pending[name] = e
        else:
            events[name].append((pending.pop(name), e))

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    rasterize.PROFILE_HOOK = None if graphs else hook
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        if graphs:
            graphs[0][0].replay()
        else:
            loss = step()
    end.record()
    barrier()
    rasterize.PROFILE_HOOK = None
    clk = clocks.stop()
    if graphs:
        rasterize.PROFILE_HOOK = hook
        for _ in range(3):
            step()
        barrier()
        rasterize.PROFILE_HOOK = None
    ms = start.elapsed_time(end) / args.steps
    if world > 1:
        ms = max_over_ranks(ms, dev)
    value = world * 1000.0 / ms
    fwd_ms = statistics.mean(a.elapsed_time(b) for a, b in events["pf_raster_forward"])
    bwd_ms = statistics.mean(a.elapsed_time(b) for a, b in events["pf_raster_backward"])

    # end to end through the public API: host target image in, loss out.  Each
    # step's target is uploaded from pinned memory on a copy stream into one of
    # two buffers (a training loop's prefetch), overlapping binning and the
    # forward; the loss waits for it, and a buffer is refilled only after the
    # loss that read it.
    target_host = target.pin_memory()
    loss_host = torch.empty(args.steps, dtype=torch.float32).pin_memory()
    copy_stream = torch.cuda.Stream()
    ready = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        b = i % 2
        copy_stream.wait_event(e0 if i < 2 else consumed[b])
        with torch.cuda.stream(copy_stream):
            t_dev[b].copy_(target_host, non_blocking=True)
            ready[b].record(copy_stream)
        if graphs:  # the upload ran during the previous step's replay
            torch.cuda.current_stream().wait_event(ready[b])
            graphs[b][0].replay()
            loss = graphs[b][1]
        else:
            loss = step(t_dev[b], ready[b])
        consumed[b].record()
        loss_host[i].copy_(loss.detach(), non_blocking=True)
    e1.record()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        e2e_ms = max_over_ranks(e2e_ms, dev)

    # statistics of one step for the roofline (outside the timed regions)
    R.collect_stats = True
    step()
    torch.cuda.synchronize()
    st = algorithmic_bytes(R.last_stats, cfg["height"], cfg["width"])
    R.collect_stats = False
    R.check()  # sync-free: a pair-buffer overflow or non-finite input in any step raises here
    peak, peak_kind = load_peaks()
    recs = st["records"] is not None
    dominant = "pf_raster_backward" if bwd_ms >= fwd_ms else "pf_raster_forward"
    dom_ms = max(bwd_ms, fwd_ms)
    dom_bytes = st["bwd"] if dominant == "pf_raster_backward" else st["fwd"]
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9

    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=max(args.warmup, 3),
                ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                data="synthetic (seeded scene, orbit camera, uniform target)",
                config=dict(workload=args.workload, prims=cfg["n"], width=cfg["width"], height=cfg["height"],
                            tile=args.tile, vfov=cfg["vfov"], pairs=st["pairs"], visited_pairs=st["V"],
                            l2="inputs larger than L2 (256 MB of primitive records), no flush",
                            step_mode="CUDA graph replays" if graphs else "eager calls, sync-free",
                            parallelism=f"view-dp{world}"),
                clocks=clk,
                e2e=dict(value=world * 1000.0 / e2e_ms, unit=UNIT, h2d_bytes_per_step=target.numel() * 4,
                         d2h_bytes_per_step=4),
                roofline=dict(bound="hbm", kernel=dominant, achieved=achieved, peak=peak, unit="GB/s",
                              frac=achieved / peak, peak_source=peak_kind,
                              traffic=(capture_traffic(dominant, args.workload, recs) or (None, None))[0],
                              traffic_source=(capture_traffic(dominant, args.workload, recs) or (None, None))[1],
                              algorithmic_bytes=dom_bytes, ms=dom_ms, fwd_ms=fwd_ms, bwd_ms=bwd_ms,
                              issue=issue_roofline(dominant, args.workload, recs, dom_ms, (clk or {}).get("sm_mhz")),
                              segment_records=st["records"]),
                gpu_launches=None)
    # kernels per step: pack 1, binning with tile order, prefetch 1, SH 1, forward 1, backward 1 + 1 sanitise;
    # with segment records the backward is two launches (the one that does not apply returns at once)
    line["gpu_launches"] = args.steps * (1 + bin_launches(st["T"]) + 1 + 1 + 1 + 1 + 1 + (1 if recs else 0))
    if fisheye:  # the cone hierarchy: one leaf launch and one per merged level
        dh, dw, levels = (cfg["height"] + 1) // 2, (cfg["width"] + 1) // 2, 1
        while dh > 1 or dw > 1:
            dh, dw, levels = (dh + 1) // 2, (dw + 1) // 2, levels + 1
        line["gpu_launches"] += args.steps * levels
        line["config"]["camera"] = "generic: 150-degree equidistant fisheye ray maps"
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not fisheye:
        line["cpu_baseline"] = cpu_baseline_line(OracleFrame(args.workload, args.tile), args.cpu_slices)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
