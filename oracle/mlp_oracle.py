"""CPU restatement of the ray-proposal network (test infrastructure only: the
product path never imports it).  No counterpart in the reference; this
mirrors powerfoam_b200/csrc/pf_mlp.cu operation by operation:

* encoding: u = (origin / 3, unit direction); features = u, then for
  k = 0..5 and each of the 6 values sin(2^k pi u), cos(2^k pi u); feature 78
  is the constant 1 (bias input), 79 is 0;
* four layers Z = X W^T with BF16 operands (round to nearest even) and wide
  accumulation; hidden layers ReLU, their outputs padded to 80 columns with
  the constant 1 in column 64 and zeros after it;
* outputs: t = z0 * 6, confidence = sigmoid(z1);
* training step: loss = w (z0 - t/6)^2 (w = overshoot weight when z0 exceeds
  the label, else 1; hit rays only) + cross-entropy of sigmoid(z1) against
  "safe" = hit and 6 z0 - margin <= t; gradients of the batch mean, with the
  data gradients rounded to BF16 where the kernel stores them;
* minibatch sampling by the kernel's integer hash of (batch index, seed,
  step).

`exact=True` drops every BF16 rounding (float64 throughout): the reference
for finite differences of the restated loss.
"""

import numpy as np

K_IN = 80
OUTS = (64, 64, 64, 16)
ONES = (78, 64, 64, 64)
T_SCALE = 6.0
N_PARAMS = 3 * 64 * K_IN + 16 * K_IN


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out.reshape(a.shape)


def bf16_bits(x):
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def layers(params):
    p = np.asarray(params)
    p = p if p.dtype == np.float64 else p.astype(np.float32)
    ws, o = [], 0
    for out in OUTS:
        ws.append(p[o:o + out * K_IN].reshape(out, K_IN))
        o += out * K_IN
    return ws


def encode(rays6):
    r = np.asarray(rays6, np.float32)
    u = r.copy()
    u[:, :3] = (u[:, :3] * np.float32(1.0 / 3.0)).astype(np.float32)
    n = u.shape[0]
    f = np.zeros((n, K_IN), np.float32)
    f[:, :6] = u
    for k in range(6):
        a = np.pi * (np.float64(2.0 ** k) * u.astype(np.float64))
        f[:, 6 + 12 * k:6 + 12 * k + 12:2] = np.sin(a).astype(np.float32)
        f[:, 7 + 12 * k:7 + 12 * k + 12:2] = np.cos(a).astype(np.float32)
    f[:, 78] = 1.0
    return f


def _pad_hidden(h):
    out = np.zeros((h.shape[0], K_IN), h.dtype)
    out[:, :64] = h
    out[:, 64] = 1.0
    return out


def _round(x, exact):
    return np.asarray(x, np.float64) if exact else bf16(x)


def forward(params, rays6, cache=False, exact=False):
    W = [_round(w, exact).astype(np.float64) for w in layers(params)]
    X = _round(encode(rays6), exact)
    acts = [X]
    zs = []
    h = X
    for li in range(4):
        z = h.astype(np.float64) @ W[li].T
        z = z if exact else z.astype(np.float32)
        zs.append(z)
        if li < 3:
            h = _round(_pad_hidden(np.maximum(z, 0.0)), exact)
            acts.append(h)
    z4 = zs[3]
    t = z4[:, 0] * T_SCALE
    conf = 1.0 / (1.0 + np.exp(-z4[:, 1].astype(np.float64)))
    if not exact:
        t, conf = t.astype(np.float32), conf.astype(np.float32)
    if cache:
        return t, conf, acts, zs
    return t, conf


def mix32(x):
    x = np.asarray(x, np.uint64) & 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def batch_indices(batch, n_rays, step, seed):
    bi = np.arange(batch, dtype=np.uint64)
    h = mix32(((bi * 2654435761) + seed) & 0xFFFFFFFF) ^ ((np.uint64(step) * 0x9E3779B9) & 0xFFFFFFFF)
    h = mix32(h)
    return (h % np.uint64(n_rays)).astype(np.int64)


def loss_value(params, rays8, idx, w_over=10.0, margin=0.02, safe=None):
    """Mean loss of the rays idx in float64 without BF16 rounding; `safe`
    fixes the confidence targets (they are a step function of the output)."""
    rb = np.asarray(rays8, np.float32)[idx]
    t_lab = rb[:, 6].astype(np.float64)
    flagged = rb[:, 7] != 0
    _, _, _, zs = forward(params, rb[:, :6], cache=True, exact=True)
    z0, z1 = zs[3][:, 0], zs[3][:, 1]
    hit = t_lab >= 0
    e = z0 - t_lab / T_SCALE
    w = np.where((e > 0) & ~flagged, w_over, 1.0)
    if safe is None:
        safe = (hit & (flagged | (z0 * T_SCALE - margin <= t_lab))).astype(np.float64)
    p = 1.0 / (1.0 + np.exp(-z1))
    lt = np.where(hit, w * e * e, 0.0)
    lc = -(safe * np.log(p) + (1 - safe) * np.log(1 - p))
    return float(np.mean(lt + lc)), safe


def train_grad(params, rays8, batch, step, seed, w_over=10.0, margin=0.02, exact=False):
    """Mean-loss gradient (N_PARAMS,) and loss sums of one minibatch."""
    r = np.asarray(rays8, np.float32)
    idx = batch_indices(batch, r.shape[0], step, seed)
    rb = r[idx]
    t_lab = rb[:, 6].astype(np.float64)
    flagged = rb[:, 7] != 0  # never reaches a significant cell: any seed is safe, no overshoot weight
    W = [_round(w, exact).astype(np.float64) for w in layers(params)]
    _, _, acts, zs = forward(params, rb[:, :6], cache=True, exact=exact)
    z0 = zs[3][:, 0].astype(np.float64)
    z1 = zs[3][:, 1].astype(np.float64)
    hit = t_lab >= 0
    e = z0 - t_lab / T_SCALE
    w = np.where((e > 0) & ~flagged, w_over, 1.0)
    safe = (hit & (flagged | (z0 * T_SCALE - margin <= t_lab))).astype(np.float64)
    p = 1.0 / (1.0 + np.exp(-z1))
    if exact:
        g0 = np.where(hit, 2.0 * w * e / batch, 0.0)
        g1 = (p - safe) / batch
    else:
        inv_b = np.float32(1.0) / np.float32(batch)
        g0 = np.where(hit, (2.0 * w * e).astype(np.float32) * inv_b, 0.0).astype(np.float32)
        g1 = ((p - safe).astype(np.float32) * inv_b).astype(np.float32)
    loss_t = float(np.sum(np.where(hit, w * e * e, 0.0)))
    loss_c = float(np.sum(-(safe * np.log(np.maximum(p, 1e-12)) + (1 - safe) * np.log(np.maximum(1 - p, 1e-12)))))
    dz = np.zeros((batch, 16), np.float64 if exact else np.float32)
    dz[:, 0] = g0
    dz[:, 1] = g1
    dz = _round(dz, exact)
    grads = [None] * 4
    for li in (3, 2, 1, 0):
        grads[li] = (dz.astype(np.float64).T @ acts[li].astype(np.float64))[:OUTS[li]]
        if li == 0:
            break
        dh = (dz.astype(np.float64) @ W[li])[:, :64]
        mask = zs[li - 1] > 0
        dz = _round(np.where(mask, dh, 0.0) if exact else np.where(mask, dh, 0.0).astype(np.float32), exact)
    g = np.concatenate([gr.reshape(-1) for gr in grads]).astype(np.float64)
    return g, (loss_t, loss_c), idx, safe


def adam(w, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (float32, as the kernel); step = updates done before."""
    w, m, v, g = (np.asarray(a, np.float32) for a in (w, m, v, g))
    f = np.float32
    t = f(step + 1)
    b1, b2, lr, eps = f(b1), f(b2), f(lr), f(eps)
    m = (b1 * m + (f(1) - b1) * g).astype(np.float32)
    v = (b2 * v + (f(1) - b2) * g * g).astype(np.float32)
    mh = m / (f(1) - np.power(b1, t))
    vh = v / (f(1) - np.power(b2, t))
    w = (w - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
    return w, m, v


def init_params(seed=0):
    """Uniform fan-in initialisation of the data columns; bias and pad zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    o = 0
    for li, out in enumerate(OUTS):
        fan_in = 78 if li == 0 else 64
        bound = np.sqrt(6.0 / fan_in) if li < 3 else np.sqrt(1.0 / fan_in)
        w = np.zeros((out, K_IN), np.float32)
        rows = out if li < 3 else 2
        w[:rows, :fan_in] = rng.uniform(-bound, bound, (rows, fan_in)).astype(np.float32)
        p[o:o + out * K_IN] = w.reshape(-1)
        o += out * K_IN
    return p
