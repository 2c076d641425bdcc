"""Interpenetration penalty (powerfoam/geometry.py:88-189).

CPU: the oracle against the golden areas produced by the reference kernel
(tests/golden/interpen_small.npz) and its adjoint against central differences
of the float64 forward.  GPU: pf_interpenetration bit-identical to the oracle,
the adjoint within 1e-5 of the largest gradient (the float4 atomics sum in no
fixed order), the autograd mirror's returns, and the argument checks."""

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from tests.helpers import np_scene

F32 = np.float32


def _golden(golden):
    g = golden("interpen_small")
    return g["spheres"], g["adjacency"], g["adjacency_offsets"], g["areas"]


def test_oracle_matches_reference_kernel(golden):
    """Equal to the reference to one ulp: the reference's pow(x, 2.0) goes
    through the platform powf, which is not correctly rounded everywhere
    (one entry of this case differs by an ulp from the exact x * x)."""
    sph, adj, off, ref = _golden(golden)
    a = orc.interpenetration(sph, adj, off)
    ulps = np.abs(a.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1
    assert (ulps > 0).sum() <= 2
    assert (ref > 0).sum() > 50 and ref[199] == 0.0


def test_oracle_adjoint_matches_central_differences(golden):
    sph, adj, off, _ = _golden(golden)
    rng = np.random.default_rng(0)
    w = rng.standard_normal(sph.shape[0]).astype(F32)
    g = orc.interpenetration_backward(sph, adj, off, w, prec="f64")
    checked = 0
    for i in rng.choice(sph.shape[0] - 1, 40, replace=False):
        for k in range(4):
            x = float(sph[i, k])
            h = max(abs(x), 1e-2) * 1e-4
            p, m = sph.copy(), sph.copy()
            p[i, k] = F32(x + h)
            m[i, k] = F32(x - h)
            span = float(p[i, k]) - float(m[i, k])
            fd = (np.dot(orc.interpenetration(p, adj, off, prec="f64"), w)
                  - np.dot(orc.interpenetration(m, adj, off, prec="f64"), w)) / span
            assert abs(fd - g[i, k]) <= 1e-6 + 2e-3 * abs(g[i, k]), (i, k, fd, g[i, k])
            checked += g[i, k] != 0
    assert checked > 40


def test_oracle_adjoint_coincident_centres(golden):
    """Spheres 0 and 1 share a centre (d = 0): radii receive 2 (s - d) g,
    centres nothing from that pair; sphere 7 lists itself."""
    sph, adj, off, _ = _golden(golden)
    w = np.zeros(sph.shape[0], F32)
    w[0] = 1.0
    only = np.array([1], np.int32)
    off1 = np.zeros(sph.shape[0] + 1, np.int32)
    off1[1:] = 1
    g = orc.interpenetration_backward(sph, only, off1, w)
    s = F32(sph[0, 3] + sph[1, 3])
    assert g[0, 3] == F32(2.0) * s and g[1, 3] == F32(2.0) * s
    assert not g[:, :3].any()
    assert 7 in adj[off[7]:off[7 + 1]]


# ---------------------------------------------------------------------------
# GPU


def _gpu_args(sph, adj, off):
    d = torch.device("cuda")
    return (torch.from_numpy(sph).to(d), torch.from_numpy(adj).to(d), torch.from_numpy(off).to(d))


def _run_fwd(sph, adj, off, status=None):
    from powerfoam_b200 import _lib

    s, a, o = _gpu_args(sph, adj, off)
    out = torch.full((sph.shape[0],), -1.0, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda") if status is None else status
    _lib.call("pf_interpenetration", _lib.ptr(s), _lib.ptr(a) if adj.size else None, _lib.ptr(o), sph.shape[0],
              adj.size, _lib.ptr(out), _lib.ptr(st), _lib.stream_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy(), int(st.item())


def _run_bwd(sph, adj, off, ga):
    from powerfoam_b200 import _lib

    s, a, o = _gpu_args(sph, adj, off)
    g = torch.from_numpy(ga).cuda()
    out = torch.full((sph.shape[0], 4), 7.0, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("pf_interpenetration_backward", _lib.ptr(s), _lib.ptr(a), _lib.ptr(o), sph.shape[0], adj.size,
              _lib.ptr(g), _lib.ptr(out), _lib.ptr(st), _lib.stream_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy(), int(st.item())


def _cloud(seed, n, rmax):
    from powerfoam_b200.adjacency import cech_adjacency

    sc = np_scene(seed, n, -1.0, 1.0, rmax / 4, rmax)
    a, o = cech_adjacency(torch.from_numpy(sc["points"]).cuda(), torch.from_numpy(sc["radii"]).cuda())
    sph = np.concatenate([sc["points"], sc["radii"][:, None]], -1).astype(F32)
    return sph, a.cpu().numpy(), o.cpu().numpy()


def _assert_grad_close(got, ref):
    scale = float(np.abs(ref).max())
    assert np.abs(got - ref).max() <= 1e-5 * scale + 1e-30


@pytest.mark.gpu
def test_gpu_forward_bit_exact_golden(golden):
    sph, adj, off, ref = _golden(golden)
    got, st = _run_fwd(sph, adj, off)
    assert st == 0
    assert np.array_equal(got.view(np.uint32), orc.interpenetration(sph, adj, off).view(np.uint32))
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("seed,n,rmax", [(11, 2000, 0.12), (12, 20000, 0.08), (13, 33, 0.5)])
def test_gpu_forward_and_adjoint_cech_lists(seed, n, rmax):
    sph, adj, off = _cloud(seed, n, rmax)
    assert adj.size > n  # dense enough that rows span chunk boundaries
    got, st = _run_fwd(sph, adj, off)
    assert st == 0
    assert np.array_equal(got.view(np.uint32), orc.interpenetration(sph, adj, off).view(np.uint32))
    ga = np.random.default_rng(seed).standard_normal(n).astype(F32)
    g, st = _run_bwd(sph, adj, off, ga)
    assert st == 0
    _assert_grad_close(g, orc.interpenetration_backward(sph, adj, off, ga))


@pytest.mark.gpu
def test_gpu_adjoint_golden_with_edge_entries(golden):
    sph, adj, off, _ = _golden(golden)
    ga = np.random.default_rng(5).standard_normal(sph.shape[0]).astype(F32)
    g, st = _run_bwd(sph, adj, off, ga)
    assert st == 0
    _assert_grad_close(g, orc.interpenetration_backward(sph, adj, off, ga))


@pytest.mark.gpu
def test_gpu_long_and_empty_rows():
    """One row longer than a warp's staging chunk, empty rows around it,
    lists that are not sorted, repeated neighbours."""
    rng = np.random.default_rng(21)
    n = 97
    sph = np.concatenate([rng.uniform(-0.3, 0.3, (n, 3)), rng.uniform(0.05, 0.3, (n, 1))], -1).astype(F32)
    lists = [[] for _ in range(n)]
    lists[3] = rng.integers(0, n, 700).tolist()
    for i in range(40, n, 3):
        lists[i] = rng.integers(0, n, rng.integers(1, 60)).tolist()
    adj = np.array([j for l in lists for j in l], np.int32)
    off = np.concatenate([[0], np.cumsum([len(l) for l in lists])]).astype(np.int32)
    got, st = _run_fwd(sph, adj, off)
    assert st == 0
    assert np.array_equal(got.view(np.uint32), orc.interpenetration(sph, adj, off).view(np.uint32))
    ga = rng.standard_normal(n).astype(F32)
    g, _ = _run_bwd(sph, adj, off, ga)
    _assert_grad_close(g, orc.interpenetration_backward(sph, adj, off, ga))


@pytest.mark.gpu
def test_gpu_bad_indices_and_offsets_are_reported():
    sph = np.array([[0, 0, 0, 1], [0.5, 0, 0, 1], [9, 9, 9, 0.1]], F32)
    adj = np.array([1, 5, -1, 0], np.int32)
    off = np.array([0, 3, 4, 4], np.int32)
    got, st = _run_fwd(sph, adj, off)
    assert st == 3
    assert got[0] == F32(F32(2.0) - F32(0.5)) ** 2 and got[2] == 0.0
    # offsets past the end of the list are clamped to n_edges
    got, st = _run_fwd(sph, adj[:2], np.array([0, 1, 2, 9], np.int32))
    assert st == 3 and got[2] == 0.0
    from powerfoam_b200 import _lib

    with pytest.raises(_lib.PfError):
        _lib.call("pf_interpenetration", None, None, None, 3, 0, None, None, None)


@pytest.mark.gpu
def test_gpu_autograd_mirror(golden):
    from powerfoam_b200.geometry import InterpenetrationFunction, interpenetration

    sph, adj, off, _ = _golden(golden)
    pts = torch.from_numpy(sph[:, :3].copy()).cuda().requires_grad_(True)
    radii = torch.from_numpy(sph[:, 3].copy()).cuda().requires_grad_(True)
    a, o = torch.from_numpy(adj).cuda(), torch.from_numpy(off).cuda()
    areas = InterpenetrationFunction.apply(pts, radii, a, o)
    assert torch.equal(areas, interpenetration(pts, radii, a, o, validate=True))
    w = torch.from_numpy(np.random.default_rng(2).standard_normal(sph.shape[0]).astype(F32)).cuda()
    (areas * w).sum().backward()
    ref = orc.interpenetration_backward(sph, adj, off, w.cpu().numpy())
    _assert_grad_close(pts.grad.cpu().numpy(), ref[:, :3])
    _assert_grad_close(radii.grad.cpu().numpy(), ref[:, 3])
    # the loss the reference's trainer adds (train.py:277)
    assert float(areas.sum()) == pytest.approx(float(orc.interpenetration(sph, adj, off).sum()), rel=1e-6)


@pytest.mark.gpu
def test_gpu_empty_inputs():
    got, st = _run_fwd(np.zeros((0, 4), F32), np.zeros(0, np.int32), np.zeros(1, np.int32))
    assert got.shape == (0,) and st == 0
    sph = np.array([[0, 0, 0, 1], [5, 0, 0, 1]], F32)
    got, st = _run_fwd(sph, np.zeros(0, np.int32), np.zeros(3, np.int32))
    assert st == 0 and not got.any()


def test_check_adjacency_host():
    from powerfoam_b200.geometry import check_adjacency

    check_adjacency(torch.tensor([1, 0], dtype=torch.int32), torch.tensor([0, 1, 2], dtype=torch.int32), 2)
    with pytest.raises(ValueError):
        check_adjacency(torch.tensor([2], dtype=torch.int32), torch.tensor([0, 1, 1], dtype=torch.int32), 2)
    with pytest.raises(ValueError):
        check_adjacency(torch.tensor([1, 0], dtype=torch.int32), torch.tensor([0, 2, 1], dtype=torch.int32), 2)
    with pytest.raises(ValueError):
        check_adjacency(torch.tensor([1], dtype=torch.int32), torch.tensor([0, 1], dtype=torch.int32), 2)
