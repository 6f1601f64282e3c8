"""A serial CPU stand-in for the part of NVIDIA Warp that the reference's hot-path kernels use, so that those
kernels -- their source, unchanged -- run in this container on small seeded inputs and produce the fixtures that
pin the oracle (tests/golden/make_golden.py). Test infrastructure only: nothing in the product imports it.

Execution model. A launch runs the kernel body once per thread index, in ascending order, each to completion.
Atomics therefore act in thread order: a compare-and-swap claim is won by the lowest index, an atomic counter
hands out ascending positions, float atomic sums add in index order. That is one of the orders the reference's
GPU run may produce (Warp gives no order), and it is the order the oracle and the B200 library fix.

Arithmetic keeps Warp's kernel types:
  * `float` and float literals are float32 (numpy float32 scalars, every operation rounded as written, no fused
    multiply-add); `float(x)` inside a kernel converts to float32;
  * `int` is a C int: `/` of two ints truncates toward zero and `%` takes the sign of the dividend;
  * wp.int64 arithmetic wraps modulo 2^64 and `>>` shifts arithmetically (numpy int64);
  * vectors and matrices are float32; a matrix-vector product sums its terms in index order.

Restated here (Warp is not installed; warp-lang >= 1.12 is the reference's dependency, pyproject.toml:25, with no
version pinned): every built-in below. Those whose low bits may differ from Warp's own are eig3 (numpy's float64
eigh of the float32 matrix, rounded to float32), quat_rotate (the expansion x (2w^2 - 1) + 2 v (v.x) + 2 w (v x x))
and sin / cos (numpy's float32 routines); HashGrid queries return every point within the radius (a superset is
what Warp returns; the kernels filter by distance). array_scan is an exclusive prefix sum in numpy.

One source transform: Warp's `while wp.hash_grid_query_next(q, j):` assigns j by reference, which Python cannot
express; the loader rewrites exactly that statement into `for j in <the query's candidates>:`.
"""

from __future__ import annotations

import ast
import builtins
import importlib.abc
import importlib.machinery
import importlib.util
import math
import sys
import types as _types
from pathlib import Path

import numpy as np

f32 = np.float32

# ---- scalars --------------------------------------------------------------------------------------------------


class WInt(int):
    """A C int inside a kernel: truncating division and remainder, int results stay WInt."""

    __slots__ = ()

    def _ok(b):
        return type(b) is WInt or type(b) is int or type(b) is bool

    def __add__(a, b):
        return WInt(int(a) + int(b)) if WInt._ok(b) else NotImplemented

    __radd__ = __add__

    def __sub__(a, b):
        return WInt(int(a) - int(b)) if WInt._ok(b) else NotImplemented

    def __rsub__(a, b):
        return WInt(int(b) - int(a)) if WInt._ok(b) else NotImplemented

    def __mul__(a, b):
        return WInt(int(a) * int(b)) if WInt._ok(b) else NotImplemented

    __rmul__ = __mul__

    @staticmethod
    def _cdiv(x: int, y: int) -> int:
        q = builtins.abs(x) // builtins.abs(y)
        return q if (x >= 0) == (y >= 0) else -q

    def __truediv__(a, b):
        if WInt._ok(b):
            return WInt(WInt._cdiv(int(a), int(b)))
        return NotImplemented

    def __rtruediv__(a, b):
        if WInt._ok(b):
            return WInt(WInt._cdiv(int(b), int(a)))
        return NotImplemented

    def __floordiv__(a, b):
        return a.__truediv__(b)

    def __mod__(a, b):
        if WInt._ok(b):
            x, y = int(a), int(b)
            return WInt(x - y * WInt._cdiv(x, y))
        return NotImplemented

    def __rmod__(a, b):
        if WInt._ok(b):
            x, y = int(b), int(a)
            return WInt(x - y * WInt._cdiv(x, y))
        return NotImplemented

    def __and__(a, b):
        return WInt(int(a) & int(b)) if WInt._ok(b) else NotImplemented

    __rand__ = __and__

    def __or__(a, b):
        return WInt(int(a) | int(b)) if WInt._ok(b) else NotImplemented

    __ror__ = __or__

    def __xor__(a, b):
        return WInt(int(a) ^ int(b)) if WInt._ok(b) else NotImplemented

    __rxor__ = __xor__

    def __lshift__(a, b):
        return WInt(int(a) << int(b)) if WInt._ok(b) else NotImplemented

    def __rlshift__(a, b):
        return WInt(int(b) << int(a)) if WInt._ok(b) else NotImplemented

    def __rshift__(a, b):
        return WInt(int(a) >> int(b)) if WInt._ok(b) else NotImplemented

    def __rrshift__(a, b):
        return WInt(int(b) >> int(a)) if WInt._ok(b) else NotImplemented

    def __neg__(a):
        return WInt(-int(a))


def _k_int(x=0):
    """int(x) in a kernel: a C int (float conversions truncate toward zero)."""
    if isinstance(x, (np.floating, float)):
        return WInt(math.trunc(float(x)))
    return WInt(int(x))


def _k_float(x=0.0):
    """float(x) in a kernel: float32."""
    return f32(x)


def _num(x):
    """A kernel scalar from whatever a built-in returned: int -> WInt, float -> float32, numpy kept."""
    if type(x) is float:
        return f32(x)
    if type(x) is int or type(x) is bool:
        return WInt(x)
    return x


def _is_float(x) -> bool:
    return isinstance(x, (float, np.floating))


# ---- vectors and matrices ----------------------------------------------------------------------------------------


class Vec:
    """A Warp vector: float32 (or the declared dtype) components."""

    __slots__ = ("v",)
    __array_ufunc__ = None  # numpy scalars defer to these operators
    N = 3
    DT = np.float32

    def __init__(self, *args):
        n, dt = type(self).N, type(self).DT
        if len(args) == 0:
            self.v = np.zeros(n, dt)
        elif len(args) == 1:
            a = args[0]
            if isinstance(a, Vec):
                self.v = a.v.astype(dt, copy=True)
            elif isinstance(a, np.ndarray):
                self.v = a.astype(dt, copy=True).reshape(n)
            else:
                self.v = np.full(n, a, dt)
        else:
            if len(args) != n:
                raise TypeError(f"vector of length {n} built from {len(args)} values")
            self.v = np.array([float(x) if not isinstance(x, np.generic) else x for x in args], dt)

    @classmethod
    def _of(cls, arr):
        o = cls.__new__(cls)
        o.v = arr
        return o

    def __getitem__(self, i):
        return _num(self.v[int(i)])

    def __setitem__(self, i, x):
        self.v[int(i)] = x

    def __len__(self):
        return type(self).N

    def __add__(self, o):
        return type(self)._of(self.v + o.v)

    def __sub__(self, o):
        return type(self)._of(self.v - o.v)

    def __neg__(self):
        return type(self)._of(-self.v)

    def __mul__(self, s):
        if isinstance(s, (Vec, Mat)):
            return NotImplemented
        return type(self)._of(self.v * _scalar(s, self.v.dtype))

    __rmul__ = __mul__

    def __truediv__(self, s):
        return type(self)._of(self.v / _scalar(s, self.v.dtype))

    def __repr__(self):
        return f"vec{type(self).N}({', '.join(str(x) for x in self.v)})"


def _scalar(s, dt):
    if isinstance(s, np.generic):
        return s
    return dt.type(s) if hasattr(dt, "type") else np.dtype(dt).type(s)


def vector(length: int, dtype=np.float32):
    dt = np.dtype(_np_dtype(dtype))
    return type(f"vec{length}", (Vec,), {"N": length, "DT": dt, "__slots__": ()})


class Mat:
    """A Warp matrix: float32, row major."""

    __slots__ = ("m",)
    __array_ufunc__ = None
    R = 3
    C = 3

    def __init__(self, *args):
        r, c = type(self).R, type(self).C
        if len(args) == 0:
            self.m = np.zeros((r, c), np.float32)
        elif len(args) == 1 and not isinstance(args[0], (np.ndarray, Mat)):
            self.m = np.full((r, c), args[0], np.float32)
        elif len(args) == 1:
            a = args[0]
            self.m = (a.m if isinstance(a, Mat) else a).astype(np.float32, copy=True).reshape(r, c)
        else:
            if len(args) != r * c:
                raise TypeError(f"{r}x{c} matrix built from {len(args)} values")
            self.m = np.array([float(x) if not isinstance(x, np.generic) else x for x in args],
                              np.float32).reshape(r, c)

    @classmethod
    def _of(cls, arr):
        o = cls.__new__(cls)
        o.m = arr
        return o

    def __getitem__(self, ij):
        if isinstance(ij, tuple):
            return _num(self.m[int(ij[0]), int(ij[1])])
        return vec_types[type(self).C]._of(self.m[int(ij)].copy())

    def __add__(self, o):
        return type(self)._of(self.m + o.m)

    def __sub__(self, o):
        return type(self)._of(self.m - o.m)

    def __mul__(self, o):
        if isinstance(o, Vec):
            # row i: ((m[i,0] v0 + m[i,1] v1) + m[i,2] v2) ..., each product and sum rounded to float32
            r = self.m[:, 0] * o.v[0]
            for j in range(1, type(self).C):
                r = r + self.m[:, j] * o.v[j]
            return vec_types[type(self).R]._of(r)
        if isinstance(o, Mat):
            out = np.zeros((type(self).R, type(o).C), np.float32)
            for i in range(type(self).R):
                for j in range(type(o).C):
                    s = self.m[i, 0] * o.m[0, j]
                    for k in range(1, type(self).C):
                        s = s + self.m[i, k] * o.m[k, j]
                    out[i, j] = s
            return mat_types[(type(self).R, type(o).C)]._of(out)
        return type(self)._of(self.m * _scalar(o, self.m.dtype))

    def __rmul__(self, s):
        return type(self)._of(self.m * _scalar(s, self.m.dtype))

    def __truediv__(self, s):
        return type(self)._of(self.m / _scalar(s, self.m.dtype))


# ---- scalar types -------------------------------------------------------------------------------------------------


def float32(x=0.0):
    return f32(x)


def float64(x=0.0):
    return np.float64(x)


def int32(x=0):
    return _k_int(x)


def int64(x=0):
    return np.int64(int(x))


def uint32(x=0):
    return np.uint32(int(x) & 0xFFFFFFFF)


def uint8(x=0):
    return WInt(int(x) & 0xFF)


def uint64(x=0):
    return np.uint64(int(x) & 0xFFFFFFFFFFFFFFFF)


def _np_dtype(t):
    table = {float32: np.float32, float64: np.float64, int32: np.int32, int64: np.int64, uint32: np.uint32,
             uint8: np.uint8, uint64: np.uint64, float: np.float32, int: np.int32, np.float32: np.float32}
    return table.get(t, t)


vec2 = vector(2)
vec3 = vector(3)
vec4 = vector(4)
vec_types = {2: vec2, 3: vec3, 4: vec4}
mat33 = type("mat33", (Mat,), {"R": 3, "C": 3, "__slots__": ()})
mat44 = type("mat44", (Mat,), {"R": 4, "C": 4, "__slots__": ()})
mat_types = {(3, 3): mat33, (4, 4): mat44}


class quat(Vec):
    __slots__ = ()
    N = 4
    DT = np.dtype(np.float32)


# ---- arrays ----------------------------------------------------------------------------------------------------


class ArrayType:
    def __init__(self, dtype=float32, ndim: int = 1):
        self.dtype = dtype


def array(dtype=float32, ndim: int = 1, **_):
    return ArrayType(dtype, ndim)


class Array:
    """A launch argument: a numpy array seen with the kernel's element type."""

    __slots__ = ("a", "vt", "mt", "wint")

    def __init__(self, a: np.ndarray, dtype):
        self.a = a
        self.vt = dtype if isinstance(dtype, type) and issubclass(dtype, Vec) else None
        self.mt = dtype if isinstance(dtype, type) and issubclass(dtype, Mat) else None
        self.wint = a.dtype in (np.int32, np.uint8, np.int16)

    def __getitem__(self, i):
        x = self.a[int(i)]
        if self.vt is not None:
            return self.vt._of(x.copy())
        if self.mt is not None:
            return self.mt._of(x.copy())
        if self.wint:
            return WInt(int(x))
        return x

    def __setitem__(self, i, x):
        if isinstance(x, Vec):
            self.a[int(i)] = x.v
        elif isinstance(x, Mat):
            self.a[int(i)] = x.m
        else:
            self.a[int(i)] = x

    def __len__(self):
        return len(self.a)

    @property
    def shape(self):
        return self.a.shape


def _raw(x):
    if isinstance(x, Vec):
        return x.v
    if isinstance(x, Mat):
        return x.m
    return x


def atomic_add(arr: Array, i, x):
    i = int(i)
    old = arr[i]
    arr.a[i] = arr.a[i] + _raw(x)
    return old


def atomic_sub(arr: Array, i, x):
    i = int(i)
    old = arr[i]
    arr.a[i] = arr.a[i] - _raw(x)
    return old


def atomic_min(arr: Array, i, x):
    i = int(i)
    old = arr[i]
    arr.a[i] = np.minimum(arr.a[i], _raw(x))
    return old


def atomic_max(arr: Array, i, x):
    i = int(i)
    old = arr[i]
    arr.a[i] = np.maximum(arr.a[i], _raw(x))
    return old


def atomic_cas(arr: Array, i, compare, value):
    i = int(i)
    old = arr[i]
    if old == compare:
        arr.a[i] = value
    return old


# ---- built-ins ---------------------------------------------------------------------------------------------------

_TID = [WInt(0)]


def tid():
    return _TID[0]


def _promote(*xs):
    if any(_is_float(x) for x in xs):
        if any(isinstance(x, np.float64) for x in xs):
            return [np.float64(x) for x in xs]
        return [f32(x) for x in xs]
    if any(isinstance(x, np.int64) for x in xs):
        return [np.int64(x) for x in xs]
    return list(xs)


def min(a, b):  # noqa: A001 - Warp's name
    if isinstance(a, Vec):
        return type(a)._of(np.minimum(a.v, b.v))
    a, b = _promote(a, b)
    return _num(b if b < a else a)


def max(a, b):  # noqa: A001 - Warp's name
    if isinstance(a, Vec):
        return type(a)._of(np.maximum(a.v, b.v))
    a, b = _promote(a, b)
    return _num(b if b > a else a)


def clamp(x, lo, hi):
    x, lo, hi = _promote(x, lo, hi)
    return _num(lo if x < lo else (hi if x > hi else x))


def abs(x):  # noqa: A001 - Warp's name
    if isinstance(x, Vec):
        return type(x)._of(np.abs(x.v))
    return _num(-x if x < 0 else x)


def floor(x):
    return np.floor(f32(x)) if not isinstance(x, np.float64) else np.floor(x)


def ceil(x):
    return np.ceil(f32(x)) if not isinstance(x, np.float64) else np.ceil(x)


def sqrt(x):
    return np.sqrt(f32(x)) if not isinstance(x, np.float64) else np.sqrt(x)


def sin(x):
    return np.sin(f32(x)) if not isinstance(x, np.float64) else np.sin(x)


def cos(x):
    return np.cos(f32(x)) if not isinstance(x, np.float64) else np.cos(x)


def exp(x):
    return np.exp(f32(x)) if not isinstance(x, np.float64) else np.exp(x)


def atan2(y, x):
    return np.arctan2(f32(y), f32(x))


def where(c, a, b):
    return a if c else b


def select(c, a, b):
    return b if c else a


def dot(a: Vec, b: Vec):
    p = a.v * b.v
    s = p[0]
    for k in range(1, len(p)):
        s = s + p[k]
    return s


def length(a: Vec):
    return np.sqrt(dot(a, a))


def length_sq(a: Vec):
    return dot(a, a)


def normalize(a: Vec):
    n = length(a)
    if n > 0.0:
        return a / n
    return type(a)()


def cross(a: Vec, b: Vec):
    x, y = a.v, b.v
    return vec3(x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0])


def outer(a: Vec, b: Vec):
    return mat_types[(a.N, b.N)]._of(a.v[:, None] * b.v[None, :])


def transpose(m: Mat):
    return type(m)._of(m.m.T.copy())


def transform_point(T: Mat, p: Vec):
    m = T.m
    r = m[:3, 0] * p.v[0]
    r = r + m[:3, 1] * p.v[1]
    r = r + m[:3, 2] * p.v[2]
    r = r + m[:3, 3]
    return vec3._of(r)


def transform_vector(T: Mat, p: Vec):
    m = T.m
    r = m[:3, 0] * p.v[0]
    r = r + m[:3, 1] * p.v[1]
    r = r + m[:3, 2] * p.v[2]
    return vec3._of(r)


def quat_from_axis_angle(axis: Vec, angle):
    h = f32(angle) * f32(0.5)
    s, c = np.sin(h), np.cos(h)
    return quat._of(np.array([axis.v[0] * s, axis.v[1] * s, axis.v[2] * s, c], np.float32))


def quat_rotate(q: quat, x: Vec):
    qx, qy, qz, qw = q.v
    a, b, cc = x.v
    two = f32(2.0)
    c = two * qw * qw - f32(1.0)
    d = two * (qx * a + qy * b + qz * cc)
    return vec3(a * c + qx * d + (qy * cc - qz * b) * qw * two,
                b * c + qy * d + (qz * a - qx * cc) * qw * two,
                cc * c + qz * d + (qx * b - qy * a) * qw * two)


def eig3(A: Mat):
    w, V = np.linalg.eigh(A.m.astype(np.float64))
    return mat33._of(V.astype(np.float32)), vec3._of(w.astype(np.float32))


# ---- hash grid --------------------------------------------------------------------------------------------------


class HashGrid:
    """The points a query may visit: every point within the radius (scipy's KD-tree), in index order."""

    def __init__(self, points: np.ndarray):
        from scipy.spatial import cKDTree

        self.points = np.asarray(points, np.float64)
        self.tree = cKDTree(self.points) if len(self.points) else None


def hash_grid_query(grid: HashGrid, p: Vec, radius):
    if grid.tree is None:
        return []
    # a slightly wider ball: the kernel applies its own float32 distance test to every candidate
    return sorted(grid.tree.query_ball_point(p.v.astype(np.float64), float(radius) * 1.001 + 1e-6))


def hash_grid_query_next(q, j):  # pragma: no cover - rewritten away by the loader
    raise RuntimeError("hash_grid_query_next runs only through the loader's rewrite")


# ---- kernels, functions, structs -------------------------------------------------------------------------------

_OVERRIDES = {"int": _k_int, "float": _k_float}


def _rebind(fn):
    g = dict(fn.__globals__)
    g.update(_OVERRIDES)
    return _types.FunctionType(fn.__code__, g, fn.__name__, fn.__defaults__, fn.__closure__)


class Func:
    def __init__(self, fn):
        self.py = fn
        self.fn = None
        self.__name__ = fn.__name__

    def __call__(self, *args):
        if self.fn is None:
            self.fn = _rebind(self.py)
        return self.fn(*args)


def func(fn):
    return Func(fn)


class Kernel:
    def __init__(self, fn):
        self.py = fn
        self.fn = None
        self.__name__ = fn.__name__
        self.params = None

    def _prepare(self):
        import inspect

        self.fn = _rebind(self.py)
        g = self.py.__globals__
        sig = inspect.signature(self.py)
        self.params = []
        for name, p in sig.parameters.items():
            ann = p.annotation
            if isinstance(ann, str):
                ann = eval(ann, g)  # noqa: S307 - the reference's own annotation expression
            self.params.append((name, ann))

    def launch(self, dim: int, *args):
        if self.fn is None:
            self._prepare()
        if len(args) != len(self.params):
            raise TypeError(f"{self.__name__}: {len(args)} arguments for {len(self.params)} parameters")
        conv = [_convert(a, t) for a, (_, t) in zip(args, self.params)]
        fn = self.fn
        with np.errstate(all="ignore"):
            for i in range(int(dim)):
                _TID[0] = WInt(i)
                fn(*conv)


def kernel(fn=None, **_):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


class StructBase:
    _fields: dict = {}


def struct(cls):
    ann = dict(getattr(cls, "__annotations__", {}))
    mod = sys.modules.get(cls.__module__)
    out = type(cls.__name__, (StructBase,), {"_ann": ann, "_mod": mod, "__doc__": cls.__doc__})
    return out


def _convert(a, t):
    if isinstance(t, ArrayType):
        if isinstance(a, Array):
            return a
        dt = t.dtype
        return Array(a, dt)
    if t is float or t is float32:
        return f32(a)
    if t is float64:
        return np.float64(a)
    if t is int or t is int32:
        return WInt(int(a))
    if t is int64:
        return np.int64(a)
    if t is uint32:
        return np.uint32(a)
    if t is uint64:
        return a
    if isinstance(t, type) and issubclass(t, Vec):
        return a if isinstance(a, t) else t(np.asarray(a, np.float64))
    if isinstance(t, type) and issubclass(t, Mat):
        return a if isinstance(a, t) else t(np.asarray(a))
    if isinstance(t, type) and issubclass(t, StructBase):
        out = t()
        g = t._mod.__dict__ if t._mod is not None else {}
        for name, ft in t._ann.items():
            if isinstance(ft, str):
                ft = eval(ft, g)  # noqa: S307 - the reference's own annotation expression
            setattr(out, name, _convert(getattr(a, name), ft))
        return out
    return a


def launch(k: Kernel, dim: int, inputs=(), outputs=(), **_):
    k.launch(dim, *inputs, *outputs)


def constant(x):
    return x


# ---- the rest of the `warp` namespace the reference's modules touch at import ---------------------------------

types = _types.SimpleNamespace(vector=vector, matrix=None)
utils = _types.SimpleNamespace(array_scan=None)
config = _types.SimpleNamespace(quiet=True)


def init():
    return None


def array_scan_exclusive(x: np.ndarray) -> np.ndarray:
    out = np.zeros_like(x)
    out[1:] = np.cumsum(x[:-1])
    return out


# ---- loading the reference's modules ----------------------------------------------------------------------------


class _HashGridLoop(ast.NodeTransformer):
    """`while wp.hash_grid_query_next(q, j): body` -> `for j in q: body` (Warp writes j by reference)."""

    def visit_While(self, node):
        self.generic_visit(node)
        t = node.test
        if (isinstance(t, ast.Call) and isinstance(t.func, ast.Attribute) and t.func.attr == "hash_grid_query_next"
                and len(t.args) == 2 and isinstance(t.args[1], ast.Name)):
            return ast.copy_location(ast.For(target=ast.Name(id=t.args[1].id, ctx=ast.Store()), iter=t.args[0],
                                             body=node.body, orelse=node.orelse), node)
        return node


class _Loader(importlib.abc.Loader):
    def __init__(self, path: Path):
        self.path = path

    def create_module(self, spec):
        return None

    def exec_module(self, module):
        tree = _HashGridLoop().visit(ast.parse(self.path.read_text(), str(self.path)))
        ast.fix_missing_locations(tree)
        exec(compile(tree, str(self.path), "exec"), module.__dict__)  # noqa: S102 - the reference's module


class _Finder(importlib.abc.MetaPathFinder):
    def __init__(self, pkg: str, root: Path):
        self.pkg, self.root = pkg, root

    def find_spec(self, fullname, path=None, target=None):
        if not fullname.startswith(self.pkg + "."):
            return None
        f = self.root / (fullname.split(".", 1)[1] + ".py")
        if not f.exists():
            return None
        return importlib.util.spec_from_file_location(fullname, f, loader=_Loader(f))


def load_reference(package_dir: Path, modules=("gpu", "odom", "perception", "mapgrid", "localize"),
                   pkg: str = "lw_reference"):
    """Import the reference's modules (package_dir = <reference>/python/livox_warp) against this shim. Returns a
    namespace of the loaded modules. The package's own __init__ is not run."""
    package_dir = Path(package_dir)
    this = sys.modules[__name__]
    saved = sys.modules.get("warp")
    sys.modules["warp"] = this
    finder = _Finder(pkg, package_dir)
    sys.meta_path.insert(0, finder)
    try:
        if pkg not in sys.modules:
            p = _types.ModuleType(pkg)
            p.__path__ = [str(package_dir)]
            p.__package__ = pkg
            sys.modules[pkg] = p
        out = {}
        for m in modules:
            out[m] = importlib.import_module(f"{pkg}.{m}")
        return _types.SimpleNamespace(**out)
    finally:
        sys.meta_path.remove(finder)
        if saved is None:
            sys.modules.pop("warp", None)
        else:
            sys.modules["warp"] = saved
