"""pf_bin_noalloc: the allocation-free binning entry point.

Callers that cannot allocate device memory while they render (a host
application's frame callback, code that must not synchronise the device
through cudaMalloc) bin through pf_bin_noalloc, whose scratch is a static
device array inside the library.  This test calls it through the C ABI twice in
a row (two different scenes and cameras, so the second call runs on scratch
that still holds the first call's data) and checks every output against
pf_bin with a caller-provided workspace, bit for bit.  It also checks that a
problem above the array's limits is refused with PF_ERR_ARGS.  This file is
collected last on purpose."""

import ctypes

import numpy as np
import pytest
import torch

from powerfoam_b200 import _lib
from tests.helpers import np_camera, np_scene, packed, to_t, torch_cam

pytestmark = pytest.mark.gpu


def _bin(fn, cam, tw, sph, cap, workspace=None):
    lib = _lib.load()
    c = torch_cam(cam).to_pf()
    T = (1 + (cam["height"] - 1) // tw) * (1 + (cam["width"] - 1) // tw)
    n = sph.shape[0]
    offs = torch.empty(T + 1, dtype=torch.int64, device="cuda")
    prims = torch.empty(cap, dtype=torch.int32, device="cuda")
    keys = torch.empty(cap, dtype=torch.int64, device="cuda")
    vis = torch.empty(n, dtype=torch.uint8, device="cuda")
    order = torch.empty(T, dtype=torch.int32, device="cuda")
    npairs = torch.zeros(1, dtype=torch.int64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    tail = (_lib.ptr(offs), _lib.ptr(prims), _lib.ptr(keys), _lib.ptr(vis), _lib.ptr(order), _lib.ptr(npairs),
            _lib.ptr(status), _lib.stream_ptr())
    if fn == "noalloc":
        rc = lib.pf_bin_noalloc(ctypes.byref(c), tw, _lib.ptr(sph), n, cap, *tail)
    else:
        rc = lib.pf_bin(ctypes.byref(c), tw, _lib.ptr(sph), n, _lib.ptr(workspace), workspace.numel(), cap, *tail)
    assert rc == _lib.PF_OK, lib.pf_last_error()
    torch.cuda.synchronize()
    k = int(npairs.item())
    assert int(status.item()) == 0 and k <= cap
    return dict(offs=offs.cpu().numpy(), prims=prims[:k].cpu().numpy(), keys=keys[:k].cpu().numpy(),
                vis=vis.cpu().numpy(), order=order.cpu().numpy(), n=k)


def _workspace(n, cap, T):
    nb = ctypes.c_size_t(0)
    _lib.call("pf_bin_workspace_size", n, cap, T, ctypes.byref(nb))
    return torch.empty(nb.value, dtype=torch.uint8, device="cuda")


@pytest.mark.parametrize("tw", [8, 16])
def test_noalloc_binning_matches_pf_bin_on_two_calls(tw):
    cases = [
        (np_scene(101, 5000, -1.0, 1.0, 0.005, 0.06), np_camera((0.4, 0.3, 2.5), (0, 0, 0), 320, 240, 55.0)),
        (np_scene(102, 20000, -1.0, 1.0, 0.003, 0.03), np_camera((-1.2, 0.8, 2.0), (0, 0, 0), 640, 360, 50.0)),
    ]
    for sc, cam in cases:
        sph = to_t(packed(sc)[0])
        cap = 1 << 17
        T = (1 + (cam["height"] - 1) // tw) * (1 + (cam["width"] - 1) // tw)
        a = _bin("noalloc", cam, tw, sph, cap)
        b = _bin("pf_bin", cam, tw, sph, cap, _workspace(sph.shape[0], cap, T))
        assert a["n"] == b["n"] and a["n"] > 0
        for k in ["offs", "prims", "keys", "vis", "order"]:
            assert np.array_equal(a[k], b[k]), k


def test_noalloc_rejects_problems_above_its_limits():
    lib = _lib.load()
    cam = np_camera((0.0, 0.0, 2.5), (0, 0, 0), 64, 48, 55.0)
    c = torch_cam(cam).to_pf()
    sph = torch.zeros((70000, 4), dtype=torch.float32, device="cuda")
    out = torch.zeros(8, dtype=torch.int64, device="cuda")
    rc = lib.pf_bin_noalloc(ctypes.byref(c), 8, _lib.ptr(sph), 70000, 1024, _lib.ptr(out), _lib.ptr(out), None, None,
                            None, _lib.ptr(out), _lib.ptr(out), _lib.stream_ptr())
    assert rc == _lib.PF_ERR_ARGS
    assert b"65536" in lib.pf_last_error()
    rc = lib.pf_bin_noalloc(ctypes.byref(c), 8, _lib.ptr(sph), 1000, 1 << 20, _lib.ptr(out), _lib.ptr(out), None,
                            None, None, _lib.ptr(out), _lib.ptr(out), _lib.stream_ptr())
    assert rc == _lib.PF_ERR_ARGS


def test_noalloc_at_its_limits():
    """The largest problem the static array is sized for -- 65,536
    primitives, a pair capacity of 262,144 and 16,384 tiles (1024 x 1024 at
    tile 8) -- bins exactly as pf_bin does; one tile more (1160 x 904: 145 x
    113 = 16,385 tiles) is refused with PF_ERR_ARGS before anything runs."""
    tw, cap = 8, 1 << 18
    sc = np_scene(103, 1 << 16, -1.0, 1.0, 0.002, 0.01)
    cam = np_camera((0.3, 0.2, 2.5), (0, 0, 0), 1024, 1024, 55.0)
    sph = to_t(packed(sc)[0])
    T = (1024 // tw) * (1024 // tw)
    assert T == 1 << 14
    a = _bin("noalloc", cam, tw, sph, cap)
    b = _bin("pf_bin", cam, tw, sph, cap, _workspace(sph.shape[0], cap, T))
    assert a["n"] == b["n"] and a["n"] > 0
    for k in ["offs", "prims", "keys", "vis", "order"]:
        assert np.array_equal(a[k], b[k]), k
    lib = _lib.load()
    c = torch_cam(np_camera((0.0, 0.0, 2.5), (0, 0, 0), 1160, 904, 55.0)).to_pf()
    out = torch.zeros(8, dtype=torch.int64, device="cuda")
    rc = lib.pf_bin_noalloc(ctypes.byref(c), tw, _lib.ptr(sph), 1000, 1024, _lib.ptr(out), _lib.ptr(out), None, None,
                            None, _lib.ptr(out), _lib.ptr(out), _lib.stream_ptr())
    assert rc == _lib.PF_ERR_ARGS
    assert b"16384" in lib.pf_last_error()
