"""Minimal stand-in for the ``taichi`` package, used ONLY to execute the
reference's own Python source (dasfadwqd/LBDEM-Taichi, ``src/``) on the CPU so
that its outputs can be frozen as golden fixtures.

Taichi is not installable in this environment.  The reference's kernels are
ordinary Python functions decorated with ``@ti.kernel``/``@ti.func``; executing
their bodies serially with NumPy float64 storage reproduces what
``ti.init(arch=ti.cpu, default_fp=ti.f64)`` computes, up to the ordering of
floating-point sums that Taichi would run in parallel (atomic adds).

Semantics implemented (only what the reference's hot path uses):
  * ``ti.field`` / ``ti.Vector.field`` -> NumPy-backed fields; scalar element
    reads return float/int subclasses that remember where they came from (so
    ``ti.atomic_add(field[i], v)`` can write back), vector element reads return
    writable NumPy views (so ``f[i, j, k][q] = v`` works).
  * ``@ti.dataclass`` -> struct type with ``.field(shape=...)`` (struct of
    arrays); element proxies support attribute get/set; assigning a struct
    value zero-fills the members it does not name, as Taichi does.
  * vector/matrix types, ``ti.math`` helpers, ``ti.ndrange``/``ti.grouped``,
    the quantised bit-array placement used for the DEM collision bit table.

This module is test infrastructure; nothing in the product imports it.
"""
from __future__ import annotations

import itertools
import math
import sys
import types

import numpy as np

# --------------------------------------------------------------------------
# dtypes
# --------------------------------------------------------------------------
f64 = np.float64
f32 = np.float32
i32 = np.int32
i64 = np.int64
u8 = np.uint8
u32 = np.uint32


def _np_dtype(dt):
    if dt is float or dt is f64 or dt is f32:
        return np.float64
    if dt is int or dt is i32 or dt is i64 or dt is u32 or dt is u8:
        return np.int64
    if dt is bool:
        return np.int64
    if isinstance(dt, _QuantInt):
        return np.int64
    raise TypeError(f"unsupported dtype {dt!r}")


class _QuantInt:
    def __init__(self, bits, signed):
        self.bits, self.signed = bits, signed


# --------------------------------------------------------------------------
# vectors / matrices
# --------------------------------------------------------------------------
class TiArr(np.ndarray):
    """ndarray with the few Taichi vector/matrix methods the reference calls."""

    @property
    def x(self):
        return self[0]

    @x.setter
    def x(self, v):
        self[0] = v

    @property
    def y(self):
        return self[1]

    @y.setter
    def y(self, v):
        self[1] = v

    @property
    def z(self):
        return self[2]

    @z.setter
    def z(self, v):
        self[2] = v

    @property
    def w(self):
        return self[3]

    def cross(self, other):
        return _arr(np.cross(np.asarray(self), np.asarray(other)))

    def dot(self, other):
        return _dot(self, other)

    def norm(self):
        return math.sqrt(_dot(self, self))

    def normalized(self):
        return _arr(np.asarray(self) / math.sqrt(_dot(self, self)))

    def transpose(self):
        return _arr(np.asarray(self).T)


def _arr(a, dtype=np.float64):
    return np.array(a, dtype=dtype).view(TiArr)


def _dot(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = 0.0
    for k in range(a.shape[0]):
        s += float(a[k]) * float(b[k])
    return np.float64(s)


class VectorType:
    def __init__(self, n, dtype):
        self.n = n
        self.dtype = _np_dtype(dtype)
        self.elem_shape = (n,)

    def __call__(self, *args):
        if len(args) == 1 and np.ndim(args[0]) == 1:
            vals = list(args[0])
        else:
            vals = list(args)
        assert len(vals) == self.n
        return _arr(vals, self.dtype)


class MatrixType:
    def __init__(self, n, m, dtype):
        self.n, self.m = n, m
        self.dtype = _np_dtype(dtype)
        self.elem_shape = (n, m)

    def __call__(self, rows):
        return _arr(rows, self.dtype)


class _Types:
    def vector(self, n, dtype):
        return VectorType(n, dtype)

    def matrix(self, n, m, dtype):
        return MatrixType(n, m, dtype)

    class quant:
        @staticmethod
        def int(bits, signed=True):
            return _QuantInt(bits, signed)


types_ns = _Types()


class Matrix:
    """``ti.Matrix`` static helpers."""

    def __new__(cls, rows):
        return _arr(rows)

    @staticmethod
    def diag(n, val):
        return _arr(np.eye(n) * val)

    @staticmethod
    def inverse(m):
        a = np.asarray(m, dtype=np.float64)
        if a.shape == (3, 3):
            det = (a[0, 0] * (a[1, 1] * a[2, 2] - a[2, 1] * a[1, 2])
                   - a[1, 0] * (a[0, 1] * a[2, 2] - a[2, 1] * a[0, 2])
                   + a[2, 0] * (a[0, 1] * a[1, 2] - a[1, 1] * a[0, 2]))
            inv_det = 1.0 / det
            out = np.zeros((3, 3))
            for i in range(3):
                for j in range(3):
                    out[j, i] = inv_det * (a[(i + 1) % 3, (j + 1) % 3] * a[(i + 2) % 3, (j + 2) % 3]
                                           - a[(i + 2) % 3, (j + 1) % 3] * a[(i + 1) % 3, (j + 2) % 3])
            return _arr(out)
        return _arr(np.linalg.inv(a))


class Vector:
    def __new__(cls, vals, dt=None):
        return _arr(vals)

    @staticmethod
    def field(n=None, dtype=float, shape=None, **kw):
        return Field(dtype, shape, (n,))


# --------------------------------------------------------------------------
# scalar element references
# --------------------------------------------------------------------------
class FloatRef(float):
    pass


class IntRef(int):
    pass


def _ref(arr, idx):
    v = arr[idx]
    if np.issubdtype(arr.dtype, np.floating):
        r = FloatRef(float(v))
    else:
        r = IntRef(int(v))
    r._arr = arr
    r._idx = idx
    return r


def _norm_idx(idx):
    if isinstance(idx, tuple):
        return tuple(int(i) for i in idx)
    if isinstance(idx, np.ndarray):
        return tuple(int(i) for i in idx)
    return int(idx)


# --------------------------------------------------------------------------
# fields
# --------------------------------------------------------------------------
class Field:
    def __init__(self, dtype, shape, elem_shape=()):
        self.dtype = _np_dtype(dtype)
        self.elem_shape = tuple(elem_shape)
        self.arr = None
        if shape is not None:
            self._alloc(shape)

    def _alloc(self, shape):
        if isinstance(shape, (int, np.integer)):
            shape = (int(shape),)
        self._shape = tuple(int(s) for s in shape)
        self.arr = np.zeros(self._shape + self.elem_shape, dtype=self.dtype)

    @property
    def shape(self):
        return self._shape

    def __getitem__(self, idx):
        idx = _norm_idx(idx)
        if self.elem_shape:
            return self.arr[idx].view(TiArr)
        return _ref(self.arr, idx)

    def __setitem__(self, idx, val):
        self.arr[_norm_idx(idx)] = np.asarray(val)

    def __iter__(self):
        if len(self._shape) == 1:
            return iter(range(self._shape[0]))
        return itertools.product(*[range(s) for s in self._shape])

    def fill(self, v):
        self.arr[...] = np.asarray(v)

    def to_numpy(self):
        return self.arr.copy()

    def from_numpy(self, a):
        self.arr[...] = np.asarray(a).reshape(self.arr.shape)


class StructType:
    def __init__(self, cls):
        self.cls = cls
        self.name = cls.__name__
        self.members = {}
        for name, ann in cls.__annotations__.items():
            if isinstance(ann, (VectorType, MatrixType)):
                self.members[name] = (ann.dtype, ann.elem_shape)
            else:
                self.members[name] = (_np_dtype(ann), ())

    def field(self, shape):
        return StructField(self, shape)

    def __call__(self, **kw):
        for k in kw:
            if k not in self.members:
                raise AttributeError(f"{self.name} has no member {k}")
        return StructValue(self, kw)


class StructValue:
    def __init__(self, stype, vals):
        self.stype = stype
        self.vals = vals


class StructField:
    def __init__(self, stype, shape):
        object.__setattr__(self, "stype", stype)
        m = {name: Field(dt, shape, es) for name, (dt, es) in stype.members.items()}
        object.__setattr__(self, "_members", m)
        if isinstance(shape, (int, np.integer)):
            shape = (int(shape),)
        object.__setattr__(self, "_shape", tuple(int(s) for s in shape))

    @property
    def shape(self):
        return self._shape

    def __getattr__(self, name):
        m = object.__getattribute__(self, "_members")
        if name in m:
            return m[name]
        raise AttributeError(name)

    def __getitem__(self, idx):
        return StructElem(self, _norm_idx(idx))

    def __setitem__(self, idx, val):
        idx = _norm_idx(idx)
        if isinstance(val, StructElem):
            for name, f in self._members.items():
                f.arr[idx] = val.sf._members[name].arr[val.idx]
        elif isinstance(val, StructValue):
            for name, f in self._members.items():
                f.arr[idx] = np.asarray(val.vals[name]) if name in val.vals else 0
        else:
            raise TypeError(val)

    def __iter__(self):
        if len(self._shape) == 1:
            return iter(range(self._shape[0]))
        return itertools.product(*[range(s) for s in self._shape])


class StructElem:
    __slots__ = ("sf", "idx", "__dict__")

    def __init__(self, sf, idx):
        object.__setattr__(self, "sf", sf)
        object.__setattr__(self, "idx", idx)

    def __getattr__(self, name):
        m = self.sf._members
        if name in m:
            return m[name][self.idx]
        raise AttributeError(name)

    def __setattr__(self, name, val):
        m = self.sf._members
        if name in m:
            m[name].arr[self.idx] = np.asarray(val)
        else:
            # Taichi python-scope write to a member the struct does not have:
            # it lands on this temporary proxy and is lost.
            object.__setattr__(self, name, val)


def dataclass(cls):
    return StructType(cls)


# --------------------------------------------------------------------------
# SNode tree (only the quantised bit array used for the collision bit table)
# --------------------------------------------------------------------------
i_axis = "i"


class _Node:
    def __init__(self, n):
        self.n = n

    def dense(self, axis, n):
        return _Node(self.n * n)

    def quant_array(self, axis, dimensions, max_num_bits):
        return _Node(self.n * dimensions)

    def place(self, f):
        f._alloc(self.n)
        return self


root = _Node(1)


# --------------------------------------------------------------------------
# functions
# --------------------------------------------------------------------------
def field(dtype=float, shape=None, **kw):
    return Field(dtype, shape)


def kernel(fn):
    return fn


def func(fn):
    return fn


def data_oriented(cls):
    return cls


def init(*a, **k):
    return None


def template():
    return None


def static(x, *a):
    return x


def static_assert(cond, msg=""):
    assert cond, msg


def loop_config(**kw):
    return None


def ndrange(*dims):
    return itertools.product(*[range(int(d)) for d in dims])


def grouped(f):
    return iter(f)


def atomic_add(target, val):
    if isinstance(target, (FloatRef, IntRef)):
        old = target._arr[target._idx]
        target._arr[target._idx] = old + val
        return type(old)(old) if not isinstance(old, np.ndarray) else old.copy()
    if isinstance(target, np.ndarray):
        old = np.array(target)
        target += np.asarray(val)
        return old
    raise TypeError(f"atomic_add on {type(target)}")


def sqrt(x):
    return np.sqrt(x)


def log(x):
    return np.log(x)


def exp(x):
    return np.exp(x)


def pow(x, y):
    return np.power(x, y)


def abs(x):
    return np.abs(x)


def cast(x, dt):
    if _np_dtype(dt) is np.int64:
        return int(x)
    return float(x)


def floor(x, dtype=float):
    r = np.floor(np.asarray(x, dtype=np.float64))
    if dtype is int or dtype is i32 or dtype is i64:
        return r.astype(np.int64).view(TiArr)
    return r.view(TiArr)


# ti.math
math_ns = types.ModuleType("taichi.math")
math_ns.pi = math.pi
math_ns.dot = _dot
math_ns.cross = lambda a, b: _arr(np.cross(np.asarray(a), np.asarray(b)))
math_ns.length = lambda v: np.float64(math.sqrt(_dot(v, v)))
math_ns.normalize = lambda v: _arr(np.asarray(v, dtype=np.float64) / math.sqrt(_dot(v, v)))
math_ns.sqrt = np.sqrt
math_ns.pow = np.power
math_ns.log = np.log
math_ns.exp = np.exp
math_ns.vec3 = VectorType(3, float)


def install():
    """Register this module as ``taichi`` / ``taichi.math`` in sys.modules."""
    mod = types.ModuleType("taichi")
    for name in ("f64", "f32", "i32", "i64", "u8", "u32", "Matrix", "Vector", "field",
                 "kernel", "func", "data_oriented", "init", "template", "static",
                 "static_assert", "loop_config", "ndrange", "grouped", "atomic_add",
                 "sqrt", "log", "exp", "pow", "abs", "cast", "floor", "dataclass", "root"):
        setattr(mod, name, globals()[name])
    import builtins
    mod.max = builtins.max
    mod.min = builtins.min
    mod.types = types_ns
    mod.i = i_axis
    mod.cpu = "cpu"
    mod.gpu = "gpu"
    mod.cuda = "cuda"
    mod.StructField = StructField
    mod.SNode = _Node
    mod.math = math_ns
    sys.modules["taichi"] = mod
    sys.modules["taichi.math"] = math_ns
    return mod
