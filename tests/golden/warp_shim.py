"""A minimal, sequential stand-in for the NVIDIA Warp runtime.

Test infrastructure only: it lets the golden-vector script import and run the
reference's own ``@wp.kernel`` source (``src/gpufluid/solvers/solver3d.py``,
``src/gpufluid/primitives/gridmath.py``) on the host, because Warp
(``warp-lang>=1.13`` per the reference's ``pyproject.toml:7``, no lock file)
is not installed here.

Execution model restated from Warp's documented semantics:

* ``wp.launch(kernel, dim, inputs)`` runs the kernel body once per thread id,
  sequentially, in row-major order of ``dim`` (last index fastest).  Every
  valid Warp schedule is allowed to run threads in any order; sequential order
  is one of them, so atomics are applied in thread order.
* Scalars annotated ``float`` are IEEE float32 (``np.float32``); Python
  literals combine with them as float32 (NumPy 2 / NEP 50 weak scalars), the
  same as Warp's float32 constants.  ``int`` is a Python int (truncating
  ``int()``).
* ``wp.vec3`` / ``wp.mat33`` values are float32 NumPy arrays with value (copy)
  semantics on read.

Only the subset of the Warp API that the hot path touches is provided.
"""
from __future__ import annotations

import inspect
import sys
import types

import numpy as np

_F32 = np.float32


class vec3:  # noqa: N801 - mirrors the Warp type name
    """Constructor and dtype tag for a float32 3-vector."""

    def __new__(cls, *a):
        if len(a) == 1:
            return np.asarray(a[0], dtype=_F32).reshape(3).copy()
        return np.array(a, dtype=_F32)


class vec3i:  # noqa: N801
    def __new__(cls, *a):
        if len(a) == 1:
            return np.asarray(a[0], dtype=np.int32).reshape(3).copy()
        return np.array(a, dtype=np.int32)


class mat33:  # noqa: N801
    def __new__(cls, *a):
        if len(a) == 1:
            return np.asarray(a[0], dtype=_F32).reshape(3, 3).copy()
        return np.array(a, dtype=_F32).reshape(3, 3)


def _np_dtype(dtype):
    if dtype is float or dtype is None:
        return _F32, ()
    if dtype is int:
        return np.int32, ()
    if dtype is vec3:
        return _F32, (3,)
    if dtype is vec3i:
        return np.int32, (3,)
    if dtype is mat33:
        return _F32, (3, 3)
    raise TypeError(f"warp_shim: unsupported dtype {dtype!r}")


class Array(np.ndarray):
    """ndarray with the few ``wp.array`` methods the solver calls.

    Element reads of vector/matrix arrays return copies (Warp value semantics).
    """

    _vec_ndim = 0

    def __getitem__(self, idx):
        r = np.ndarray.__getitem__(self, idx)
        if self._vec_ndim and isinstance(r, np.ndarray) and r.ndim == self._vec_ndim:
            return np.array(r)  # plain copy
        return r

    def __setitem__(self, idx, value):
        # assign through a base-class view so the copying __getitem__ above is
        # never used to locate the destination
        np.ndarray.__setitem__(self.view(np.ndarray), idx, value)

    def numpy(self):
        return np.array(self.view(np.ndarray))

    def zero_(self):
        self.fill(0)

    def fill_(self, v):
        self.fill(v)

    @property
    def device(self):
        return "cpu"


def _wrap(data, vec_ndim):
    a = np.ascontiguousarray(data).view(Array)
    a._vec_ndim = vec_ndim
    return a


def zeros(shape, dtype=float, device=None, **_kw):
    dt, tail = _np_dtype(dtype)
    if isinstance(shape, int):
        shape = (shape,)
    return _wrap(np.zeros(tuple(shape) + tail, dtype=dt), len(tail))


def array(data, dtype=float, device=None, **_kw):
    dt, tail = _np_dtype(dtype)
    a = np.array(data, dtype=dt)
    if tail and a.shape[-len(tail):] != tail:
        a = a.reshape((-1,) + tail)
    return _wrap(a, len(tail))


def copy(dst, src, *a, **k):
    np.copyto(dst.view(np.ndarray), np.asarray(src).reshape(dst.shape))


# ----------------------------------------------------------------- kernel exec
_TID = [0]


def tid():
    return _TID[0]


class Kernel:
    def __init__(self, fn):
        self.fn = fn
        self.__name__ = fn.__name__
        self.key = fn.__name__
        sig = inspect.signature(fn)
        self.ann = [_ann_name(p.annotation) for p in sig.parameters.values()]

    def __call__(self, *a, **k):
        return self.fn(*a, **k)


def kernel(fn=None, **_kw):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


def func(fn=None, **_kw):
    if fn is None:
        return lambda f: f
    return fn


def _ann_name(a):
    if a is float:
        return "float"
    if a is int:
        return "int"
    if a is vec3:
        return "wp.vec3"
    return str(a)


def _convert(ann, v):
    if ann == "float":
        return _F32(v)
    if ann == "int":
        return int(v)
    if ann == "wp.vec3":
        return vec3(v)
    return v


# Optional observer called after each launch: hook(kernel_name, args).
LAUNCH_HOOK = [None]


def launch(kernel, dim, inputs=(), outputs=(), device=None, **_kw):
    args = [_convert(a, v) for a, v in zip(kernel.ann, list(inputs) + list(outputs))]
    fn = kernel.fn
    if isinstance(dim, int):
        for t in range(dim):
            _TID[0] = t
            fn(*args)
    else:
        dims = tuple(int(d) for d in dim)
        if len(dims) == 1:
            for t in range(dims[0]):
                _TID[0] = t
                fn(*args)
        elif len(dims) == 3:
            for i in range(dims[0]):
                for j in range(dims[1]):
                    for k in range(dims[2]):
                        _TID[0] = (i, j, k)
                        fn(*args)
        else:
            raise NotImplementedError(dims)
    if LAUNCH_HOOK[0] is not None:
        LAUNCH_HOOK[0](kernel.key, args)


# ------------------------------------------------------------------ builtins
def floor(x):
    return np.floor(_F32(x))


def _is_int(x):
    return isinstance(x, (int, np.integer)) and not isinstance(x, bool)


def clamp(x, lo, hi):
    if _is_int(x) and _is_int(lo) and _is_int(hi):
        return min(max(int(x), int(lo)), int(hi))
    x, lo, hi = _F32(x), _F32(lo), _F32(hi)
    if x < lo:
        return lo
    if x > hi:
        return hi
    return x


def abs(x):  # noqa: A001
    return np.abs(x)


def max(a, b):  # noqa: A001
    if _is_int(a) and _is_int(b):
        return a if a > b else b
    a, b = _F32(a), _F32(b)
    return a if a > b else b


def min(a, b):  # noqa: A001
    import builtins
    if _is_int(a) and _is_int(b):
        return builtins.min(a, b)
    a, b = _F32(a), _F32(b)
    return a if a < b else b


def sqrt(x):
    return np.sqrt(_F32(x))


def dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


_GRIDS = {}


class HashGrid:
    """Point grid for neighbour queries (only what a query returns matters)."""

    def __init__(self, dim_x=1, dim_y=1, dim_z=1, device=None):
        self.id = len(_GRIDS) + 1
        self.points = np.zeros((0, 3), _F32)
        _GRIDS[self.id] = self

    def build(self, points, radius):
        self.points = np.asarray(points, dtype=_F32).reshape(-1, 3)


def hash_grid_query(grid_id, point, radius):
    """Every point of the grid: a superset of the points within ``radius``,
    which is all a Warp hash-grid query promises (callers test distances)."""
    return range(len(_GRIDS[int(grid_id)].points))


def atomic_add(arr, *idx_val):
    """Adds and returns the value before the add (Warp's atomic_add)."""
    *idx, val = idx_val
    base = arr.view(np.ndarray)
    idx = tuple(int(i) for i in idx)
    old = base[idx].copy()
    base[idx] = base[idx] + val
    return old


def atomic_max(arr, *idx_val):
    *idx, val = idx_val
    base = arr.view(np.ndarray)
    idx = tuple(int(i) for i in idx)
    if val > base[idx]:
        base[idx] = val
    return base[idx]



class _Device:
    is_capturing = False

    def __init__(self, name="cpu"):
        self.name = name

    def __str__(self):
        return self.name


def init():
    return None


def get_devices():
    return ["cpu"]


def get_device(name=None):
    return _Device(str(name or "cpu"))


def synchronize():
    return None


class ScopedTimer:
    def __init__(self, name, dict=None, **_kw):  # noqa: A002
        self.name, self.dict = name, dict

    def __enter__(self):
        import time
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *a):
        import time
        if self.dict is not None:
            self.dict.setdefault(self.name, []).append((time.perf_counter() - self.t0) * 1e3)
        return False


class _Types(types.ModuleType):
    pass


def __getattr__(name):
    if name.startswith("array"):
        return lambda *a, **k: None
    raise AttributeError(name)


def install():
    """Register this module as ``warp`` in ``sys.modules``."""
    mod = sys.modules[__name__]
    mod.array3d = lambda *a, **k: None
    mod.float32 = float
    mod.int32 = int
    mod.uint64 = int
    sys.modules["warp"] = mod
    return mod
