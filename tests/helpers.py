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
