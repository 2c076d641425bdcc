"""A numpy restatement of the slice of the Warp 1.10 runtime that the Power Foam
rendering kernels use, so that the reference's own kernel source
(powerfoam/rasterize.py, raytrace.py, texture.py, rendering_math.py,
camera.py) can be executed on the CPU to produce golden vectors.

warp-lang==1.10.0 (reference requirements.txt:22) is not installable here, so
its semantics are restated from its public documentation:

* ``float`` inside a kernel is float32; literals are rounded to float32 when
  they meet a float32 operand (numpy's NEP 50 weak-scalar rule gives the same).
* vec3f/vec4f/vec4h are fixed-size float32/float16 vectors with per-component
  arithmetic; ``dot`` sums in index order; ``normalize(a) = a / length(a)``.
* integer ``//`` and ``%`` follow C (truncation toward zero), as Warp's
  generated CUDA does.
* ``int32(float)`` truncates toward zero and saturates, NaN -> 0, as the GPU's
  cvt.rzi does.
* ``wp.cast(x, wp.uint32)`` reinterprets the bits.
* ``wp.float16`` rounds to nearest even.
* ``min``/``max`` are ``a < b ? a : b`` / ``a > b ? a : b``.
* ``a[i] += v`` on an array is an atomic add.
* ``wp.tile(x)``, ``wp.tile_max``, ``wp.tile_sum`` are block collectives: the
  threads of a block run as Python threads that meet at a barrier.  The GIL
  switch interval is raised so a thread only yields at a barrier; every
  read-modify-write between barriers is therefore atomic.

This module is test infrastructure; the product never imports it.
"""

import math
import sys
import threading
import types

import numpy as np

F32 = np.float32
F16 = np.float16

_tls = threading.local()


# ----------------------------------------------------------------------------
# C-semantics integers
class CInt(int):
    """int whose // and % truncate toward zero (C / Warp integer semantics)."""

    def __new__(cls, v):
        return int.__new__(cls, int(v))

    def _w(self, v):
        return CInt(v) if isinstance(v, int) and not isinstance(v, bool) else v

    def __add__(self, o):
        return self._w(int(self) + o) if isinstance(o, int) else int(self) + o

    __radd__ = __add__

    def __sub__(self, o):
        return self._w(int(self) - o) if isinstance(o, int) else int(self) - o

    def __rsub__(self, o):
        return self._w(o - int(self)) if isinstance(o, int) else o - int(self)

    def __mul__(self, o):
        return self._w(int(self) * o) if isinstance(o, int) else int(self) * o

    __rmul__ = __mul__

    def __floordiv__(self, o):
        if isinstance(o, int):
            q = abs(int(self)) // abs(int(o))
            return CInt(q if (int(self) >= 0) == (int(o) >= 0) else -q)
        return int(self) // o

    def __rfloordiv__(self, o):
        return CInt(o).__floordiv__(int(self))

    def __mod__(self, o):
        if isinstance(o, int):
            return CInt(int(self) - int(o) * int(self.__floordiv__(o)))
        return int(self) % o

    def __neg__(self):
        return CInt(-int(self))

    def __lshift__(self, o):
        return CInt(int(self) << int(o))

    def __or__(self, o):
        return CInt(int(self) | int(o))


def _int32(x):
    if isinstance(x, (np.floating, float)):
        xf = float(x)
        if math.isnan(xf):
            return CInt(0)
        if xf >= 2147483647.0:
            return CInt(2147483647)
        if xf <= -2147483648.0:
            return CInt(-2147483648)
        return CInt(int(xf))
    return CInt(int(x))


def _int64(x):
    return CInt(int(x))


# ----------------------------------------------------------------------------
# vectors
def _vec(dtype, n):
    def ctor(*args):
        if len(args) == 0:
            return np.zeros(n, dtype=dtype)
        if len(args) == 1:
            a = args[0]
            if np.ndim(a) == 0:
                return np.full(n, a, dtype=dtype)
            return np.asarray(a, dtype=dtype).copy()
        return np.array([dtype(a) for a in args], dtype=dtype)

    return ctor


def dot(a, b):
    r = a[0] * b[0]
    for i in range(1, len(a)):
        r = r + a[i] * b[i]
    return r


def length(a):
    return np.sqrt(dot(a, a))


def length_sq(a):
    return dot(a, a)


def normalize(a):
    l = length(a)
    if l > 0.0:
        return a / l
    return np.zeros_like(a)


def cross(a, b):
    return np.array(
        [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]],
        dtype=a.dtype,
    )


def _min(a, b):
    return a if a < b else b


def _max(a, b):
    return a if a > b else b


def _cast(x, dtype):
    assert dtype is _uint32
    return CInt(int(np.asarray(x, dtype=np.float32).view(np.uint32)))


def _uint32(x):
    return CInt(int(x) & 0xFFFFFFFF)


def _atomic_add(arr, idx, v):
    old = arr[idx]
    arr[idx] = arr[idx] + v
    return CInt(int(old))


def norm_l1(v):
    r = abs(v[0])
    for i in range(1, len(v)):
        r = r + abs(v[i])
    return r


# ----------------------------------------------------------------------------
# block collectives
class _Block:
    def __init__(self, n):
        self.n = n
        self.barrier = threading.Barrier(n)
        self.slots = [None] * n


def _gather(x):
    blk = _tls.block
    lane = _tls.lane
    blk.slots[lane] = x
    blk.barrier.wait()
    vals = list(blk.slots)
    blk.barrier.wait()
    return vals


def tile(x):
    vals = _gather(x)
    if np.ndim(vals[0]) == 0:
        return np.array(vals)
    return np.stack(vals, axis=1)


def tile_max(t):
    return np.array([np.max(t)])


def tile_sum(t):
    return np.array([np.sum(t)])


def tile_load(arr, shape=None):
    return arr[: shape[0]]


def tid():
    return CInt(_tls.tid)


# ----------------------------------------------------------------------------
# decorators and launch
def _func(f):
    return f


def _kernel(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


def _struct(cls):
    return cls


def launch(kernel, dim, inputs, block_dim=256, cooperative=False):
    """Run kernel(*inputs) for every thread id in [0, dim).

    Kernels that use block collectives run one block at a time with
    block_dim Python threads; the others run sequentially."""
    if not cooperative:
        for t in range(dim):
            _tls.tid = t
            kernel(*inputs)
        return
    old = sys.getswitchinterval()
    sys.setswitchinterval(1000.0)
    try:
        assert dim % block_dim == 0
        for b in range(dim // block_dim):
            blk = _Block(block_dim)
            errs = []

            def run(lane, blk=blk):
                _tls.tid = b * block_dim + lane
                _tls.lane = lane
                _tls.block = blk
                try:
                    kernel(*inputs)
                except BaseException as e:  # noqa: BLE001
                    errs.append(e)
                    blk.barrier.abort()

            ths = [threading.Thread(target=run, args=(l,)) for l in range(block_dim)]
            for t in ths:
                t.start()
            for t in ths:
                t.join()
            if errs:
                raise errs[0]
    finally:
        sys.setswitchinterval(old)


def _array(*a, **k):
    return None


def install():
    """Register the shim as the ``warp`` module (and a stub ``open3d``)."""
    wp = types.ModuleType("warp")
    wp.func = _func
    wp.kernel = _kernel
    wp.struct = _struct
    wp.constant = lambda v: F32(v) if isinstance(v, float) else v
    wp.float32 = F32
    wp.float16 = F16
    wp.int32 = _int32
    wp.int64 = _int64
    wp.uint32 = _uint32
    wp.uint64 = _int64
    wp.bool = bool
    wp.vec3f = _vec(F32, 3)
    wp.vec4f = _vec(F32, 4)
    wp.vec3h = _vec(F16, 3)
    wp.vec4h = _vec(F16, 4)
    wp.vec3 = wp.vec3f
    wp.array = _array
    wp.array2d = _array
    wp.array3d = _array
    wp.dot = dot
    wp.length = length
    wp.length_sq = length_sq
    wp.normalize = normalize
    wp.cross = cross
    wp.min = _min
    wp.max = _max
    wp.abs = abs
    wp.sqrt = np.sqrt
    wp.exp = np.exp
    wp.log = np.log
    wp.floor = np.floor
    wp.ceil = np.ceil
    wp.cast = _cast
    wp.atomic_add = _atomic_add
    wp.tid = tid
    wp.tile = tile
    wp.tile_max = tile_max
    wp.tile_sum = tile_sum
    wp.tile_load = tile_load
    wp.math = types.SimpleNamespace(norm_l1=norm_l1)
    # fixed-size local matrices (the generic binning's traversal stacks, the
    # cone builders' scratch): zero-initialised numpy arrays of that type
    wp.mat = lambda shape, dtype: np.zeros(shape, dtype=np.int32 if dtype in (_int32, _uint32, _int64) else F32)
    wp.identity = lambda n, dtype: np.eye(n, dtype=F32)
    wp.outer = lambda a, b: np.outer(np.asarray(a, F32), np.asarray(b, F32)).astype(F32)
    wp.array2d = _array
    wp.launch = launch
    wp.cw_div = lambda a, b: a / b
    wp.Bvh = None
    wp.uint64 = _int64
    sys.modules["warp"] = wp
    o3d = types.ModuleType("open3d")
    o3d.camera = types.SimpleNamespace(PinholeCameraParameters=object, PinholeCameraIntrinsic=object)
    sys.modules["open3d"] = o3d
    return wp


def patch_module_builtins(mod):
    """Inside Warp kernels ``float``/``int`` are float32/int32 conversions."""
    mod.float = F32
    mod.int = CInt


class _Sq(np.float32):
    """float32 whose ``** 2.0`` is the correctly rounded square x*x (the
    meaning taken for pow(x, 2.0) in proj_sphere_to_obb; glibc's powf is not
    correctly rounded for every x)."""

    def __pow__(self, e):
        if e == 2.0:
            v = np.float32(self)
            return v * v
        return np.float32(self) ** e


def patch_camera_module(cam_mod, wp):
    proxy = types.ModuleType("warp_camera_proxy")
    proxy.__dict__.update(wp.__dict__)
    proxy.dot = lambda a, b: _Sq(dot(a, b))
    cam_mod.wp = proxy
