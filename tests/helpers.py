"""Shared test helpers: build scenes, run the oracle (CPU) and the library (GPU)
on the same inputs, compare."""

import numpy as np
import torch

from oracle import oracle as orc

F32 = np.float32


def np_scene(seed, n, lo=-0.6, hi=0.6, rmin=0.05, rmax=0.2, S=8, height_scale=0.1, toward=None):
    rng = np.random.default_rng(seed)
    pts = rng.uniform(lo, hi, size=(n, 3)).astype(F32)
    radii = np.exp(rng.uniform(np.log(rmin), np.log(rmax), n)).astype(F32)
    dens = (np.log1p(np.exp(rng.standard_normal(n))) * 10).astype(F32)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    w, x, y, z = q.T
    nrm = np.stack([1 - 2 * (y**2 + z**2), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1)
    tng = np.stack([2 * (x * y + z * w), 1 - 2 * (x**2 + z**2), 2 * (y * z - x * w)], -1)
    btg = np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x**2 + y**2)], -1)
    nrm, tng, btg = (v / np.linalg.norm(v, axis=-1, keepdims=True) for v in (nrm, tng, btg))
    if toward is not None:
        v = pts - np.asarray(toward, F32)
        s = np.sign(np.sum(nrm * v, -1, keepdims=True))
        nrm = -nrm * s
    s2 = rng.standard_normal((n, S, 2)) * 0.1
    off = s2 * radii[:, None, None]
    off = off[..., 0:1] * tng[:, None, :] + off[..., 1:2] * btg[:, None, :]
    return dict(points=pts, radii=radii, density=dens, normals=nrm.astype(F32),
                texel_sites=(pts[:, None, :] + off).astype(F32),
                texel_rgb=rng.uniform(0, 1, (n, S, 3)).astype(F32),
                texel_height=(rng.standard_normal((n, S)) * height_scale * radii[:, None]).astype(F32))


def np_camera(eye, target, W, H, vfov, up_w=(0.0, 1.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, up_w)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    th = np.tan(np.radians(vfov) / 2)
    return dict(eye=eye.astype(F32), right=(r * th * W / H).astype(F32), up=(u * th).astype(F32), width=W,
                height=H)


def cech_np(points, radii):
    """bvh.py:7-69 predicate, brute force, ascending lists."""
    lo = (points - radii[:, None]).astype(F32)
    hi = (points + radii[:, None]).astype(F32)
    c = (F32(0.5) * (lo + hi)).astype(F32)
    r = (F32(0.5) * (hi[:, 0] - lo[:, 0])).astype(F32)
    n = points.shape[0]
    adj, off = [], [0]
    for i in range(n):
        d = c[i][None, :] - c
        dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(F32)
        ov = np.all(lo[i] <= hi, axis=1) & np.all(hi[i] >= lo, axis=1)
        m = ov & (dist < (r[i] + r)) & (np.arange(n) != i)
        js = np.nonzero(m)[0]
        adj.extend(js.tolist())
        off.append(len(adj))
    return np.array(adj, np.int32), np.array(off, np.int32)


def orc_cam(cam):
    return orc.camera(cam["eye"], cam["right"], cam["up"], cam["width"], cam["height"])


def torch_cam(cam, device="cuda"):
    from powerfoam_b200.camera import TorchCamera

    return TorchCamera(eye=torch.from_numpy(cam["eye"]).to(device), right=torch.from_numpy(cam["right"]).to(device),
                       up=torch.from_numpy(cam["up"]).to(device), width=int(cam["width"]), height=int(cam["height"]))


def to_t(a, device="cuda"):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def packed(sc):
    sph = np.concatenate([sc["points"], sc["radii"][:, None]], -1).astype(F32)
    nsig = np.concatenate([sc["normals"], sc["density"][:, None]], -1).astype(F32)
    rgbh = np.concatenate([sc["texel_rgb"], sc["texel_height"][..., None]], -1).astype(F32)
    return sph, nsig, rgbh


def max_abs(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max()) if a.size else 0.0


def assert_close_rel(a, b, rel, what=""):
    """max |a - b| <= rel * max |b| (+ a denormal floor): normwise relative."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.abs(b).max()) if b.size else 0.0, 1e-30)
    err = float(np.abs(a - b).max()) if a.size else 0.0
    assert err <= rel * scale + 1e-12, f"{what}: max abs err {err:.3e} vs scale {scale:.3e} (rel {err / scale:.2e})"


# ---------------------------------------------------------------------------
# Restricted tile lists and finite differences on large frames.  The oracle
# composites only the tiles a check needs; every other tile gets an empty list.


def tile_pixels(t, H, W, tw):
    """Row-major pixel indices of tile t (tiles are column-major:
    tile_i = t % tiles_h, tile_j = t // tiles_h, rasterize.py:919-938)."""
    tiles_h = 1 + (H - 1) // tw
    ti, tj = t % tiles_h, t // tiles_h
    rows = np.arange(ti * tw, min((ti + 1) * tw, H))
    cols = np.arange(tj * tw, min((tj + 1) * tw, W))
    return (rows[:, None] * W + cols[None, :]).ravel()


def restrict_lists(offs, prims, tiles, T=None):
    """(tile_offsets (T+1) i64, tile_prims) holding only the lists of
    ``tiles``; the other tiles are empty."""
    T = offs.shape[0] - 1 if T is None else T
    tiles = np.unique(np.asarray(tiles, np.int64))
    lens = np.zeros(T, np.int64)
    lens[tiles] = offs[tiles + 1] - offs[tiles]
    new_offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    parts = [prims[offs[t]:offs[t + 1]] for t in tiles]
    new_prims = np.concatenate(parts).astype(np.int32) if parts else np.zeros(0, np.int32)
    return new_offs, new_prims


class PrimTiles:
    """For sorted binning output (keys, prims): the tiles each primitive is
    binned to, and the per-tile (key, prim) lists."""

    def __init__(self, keys, prims, offs):
        self.keys, self.prims, self.offs = keys, prims, offs
        self.tile = (keys >> 32).astype(np.int64)
        self.order = np.argsort(prims, kind="stable")
        sp = prims[self.order]
        self.first = np.searchsorted(sp, np.arange(int(prims.max()) + 2 if prims.size else 1))

    def tiles_of(self, p):
        if p + 1 >= self.first.shape[0]:
            return np.zeros(0, np.int64)
        return self.tile[self.order[self.first[p]:self.first[p + 1]]]

    def lists_with(self, tiles, p, new_keys):
        """Lists of ``tiles`` with primitive p's entries replaced by
        ``new_keys`` (its keys after a perturbation; tile in the high word),
        ordered by (key, prim) like pf_bin."""
        T = self.offs.shape[0] - 1
        tiles = np.unique(np.asarray(tiles, np.int64))
        new_tile = (new_keys >> 32).astype(np.int64)
        lens = np.zeros(T, np.int64)
        parts = []
        for t in tiles:
            a, b = self.offs[t], self.offs[t + 1]
            k, q = self.keys[a:b], self.prims[a:b]
            keep = q != p
            k, q = k[keep], q[keep]
            add = new_keys[new_tile == t]
            if add.size:
                k = np.concatenate([k, add])
                q = np.concatenate([q, np.full(add.shape[0], p, np.int32)])
                o = np.lexsort((q, k))
                k, q = k[o], q[o]
            lens[t] = q.shape[0]
            parts.append(q.astype(np.int32))
        new_offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        return new_offs, (np.concatenate(parts) if parts else np.zeros(0, np.int32))


FD_NAMES = ("points", "radii", "density", "normals", "texel_rgb")


def fd_gradient(oc, tw, sc, adj, adj_off, pt, target, name, idx, eps=1e-3):
    """Central difference of L = sum (color - target)^2 with respect to one
    scalar input, evaluated by the float64 oracle with exact neighbour
    spheres on the tiles the input can change (the primitive's own tiles
    before and after the step and, for centres and radii, the tiles of its
    neighbours, whose faces it moves).  Step h = eps * the input's scale:
    the primitive's radius for centres and radii (a centre has no magnitude
    of its own), max(|x|, 1e-2) otherwise.
    ``sc``: numpy scene (points, radii, density, normals, texel_sites,
    texel_rgb, texel_height); ``pt``: PrimTiles of the unperturbed binning.
    Returns (fd, tiles used)."""
    from oracle import oracle as orc

    H, W = oc.height, oc.width
    p = int(idx[0])
    x = float(sc[name][idx])
    h = (float(sc["radii"][p]) if name in ("points", "radii") else max(abs(x), 1e-2)) * eps
    tiles = [pt.tiles_of(p)]
    variants = []
    for sgn in (1.0, -1.0):
        arr = sc[name].copy()
        arr[idx] = np.float32(x + sgn * h)
        s2 = dict(sc, **{name: arr})
        sph, nsig, rgbh = packed(s2)
        if name in ("points", "radii"):
            k1, _, _, _ = orc.bin(oc, sph[p:p + 1], tw)
            tiles.append((k1 >> 32).astype(np.int64))
        else:
            k1 = None
        variants.append((float(arr[idx]) - x, sph, nsig, s2, rgbh, k1))
    if name in ("points", "radii"):
        for j in adj[adj_off[p]:adj_off[p + 1]]:
            tiles.append(pt.tiles_of(int(j)))
    tiles = np.unique(np.concatenate(tiles)) if tiles else np.zeros(0, np.int64)
    pix = np.concatenate([tile_pixels(int(t), H, W, tw) for t in tiles]) if tiles.size else np.zeros(0, np.int64)
    tgt = target.reshape(-1, 3)[pix].astype(np.float64)
    losses = []
    base_keys = None
    for dh, sph, nsig, s2, rgbh, k1 in variants:
        if k1 is None:
            if base_keys is None:
                a = pt.order[pt.first[p]:pt.first[p + 1]] if p + 1 < pt.first.shape[0] else np.zeros(0, np.int64)
                base_keys = pt.keys[a]
            k1 = base_keys
        offs, prims = pt.lists_with(tiles, p, k1)
        o = orc.raster_forward(oc, tw, sph, nsig, s2["texel_sites"], rgbh, adj, adj_off, None, offs, prims,
                               prec="f64")
        c = o["color"].reshape(-1, 3)[pix]
        losses.append((float(((c - tgt) ** 2).sum()), dh))
    (lp, hp), (lm, hm) = losses
    return (lp - lm) / (hp - hm), tiles


def vary_sites(sc, seed):
    """Per-site variation of a scene whose texel colours are equal on all of a
    primitive's sites and whose heights are zero (the SH pre-step's output):
    colours + N(0, 0.05^2) clamped at 0, heights N(0, (0.1 r)^2).  With equal
    colours and zero heights the texel-site gradient is zero in exact
    arithmetic -- a difference of equal blended colours times the weight
    derivative -- so the float32 values of the reference and of the kernels
    are rounding noise; the varied scene makes it well conditioned."""
    rng = np.random.default_rng(seed)
    rgb = np.maximum(sc["texel_rgb"] + rng.normal(0, 0.05, sc["texel_rgb"].shape), 0).astype(F32)
    h = (rng.standard_normal(sc["texel_height"].shape) * 0.1 * sc["radii"][:, None]).astype(F32)
    return dict(sc, texel_rgb=rgb, texel_height=h)


def assert_quantiles_close(a, b, tol=1e-5, max_flips=2):
    """Quantile depths (H,W,Q): a quantile is reached when the transmittance
    after a segment, expf(log_t), falls below q.  CUDA's expf and the C
    library's may differ by an ulp, so a q within an ulp of a transmittance
    is decided differently; at most ``max_flips`` pixels may differ (from the
    first quantile on which they disagree), every other one within tol."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    bad = (np.abs(a - b) > tol).any(-1)
    assert int(bad.sum()) <= max_flips, f"{int(bad.sum())} pixels' quantile depths differ"


def cycle_scene(cycle_density=0.0, S=8):
    """Three cells on the x axis whose float16 face records disagree: cell 0
    (a sphere the rays cross, density 5) exits into cell 1 at x = 1.5, cell 1
    into cell 2 at x = 2, and cell 2's face back to cell 1 (at x = 2.5) faces
    +x as well, so a ray along +x walks 0, 1, 2, 1, 2, ... forever -- the
    reference's walk never returns.  With cycle_density > 0 the spheres of
    cells 1 and 2 lie on the rays, so every lap absorbs and the walk ends on
    the transmittance.  Returns (scene dict, adjacency, offsets, float16
    face records (n_adj, 4)) and a camera at the origin looking along +x."""
    rng = np.random.default_rng(7)
    centers = np.array([[1.0, 0.0, 0.0], [1.75, 0.0, 0.0], [2.25, 0.0, 0.0]], F32)
    radii = np.array([0.2, 0.2, 0.2], F32)
    if cycle_density <= 0:  # off the rays: cells 1 and 2 are crossed without a hit
        centers[1:, 1] = 3.0
    density = np.array([5.0, cycle_density, cycle_density], F32)
    normals = np.tile(np.array([[1.0, 0.0, 0.0]], F32), (3, 1))
    sites = (centers[:, None, :] + rng.uniform(-0.1, 0.1, (3, S, 3))).astype(F32)
    sc = dict(points=centers, radii=radii, density=density, normals=normals, texel_sites=sites,
              texel_rgb=rng.uniform(0.1, 0.9, (3, S, 3)).astype(F32), texel_height=np.zeros((3, S), F32))
    adj = np.array([1, 2, 1], np.int32)
    off = np.array([0, 1, 2, 3], np.int32)
    faces = np.array([[1.0, 0.0, 0.0, 1.5], [1.0, 0.0, 0.0, 2.0], [1.0, 0.0, 0.0, 2.5]], np.float16)
    cam = np_camera((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 8, 6, 4.0)
    return sc, adj, off, faces, cam
