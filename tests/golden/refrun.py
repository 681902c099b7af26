# TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
"""Run the reference's own Warp kernels (alloy/solvers/sph/*.py) on the CPU, one Python call per thread, in float32.

warp-lang (pinned 1.18.0 by the reference) is not installed in this container and cannot be, so ``warp`` is replaced
by a stand-in and the reference's modules are loaded from their source with three rewrites of every ``@wp.kernel`` /
``@wp.func`` body (host code is left alone):

- float literals become float32 constants and ``float(x)`` becomes ``float32(x)``: Warp types both as float32 in a
  kernel, and numpy scalars then keep every operation in float32 (numpy 2 treats Python scalars as weak);
- ``while wp.hash_grid_query_next(query, j):`` becomes ``for j in query:``;
- the decorators become the stand-in's (a kernel is launched as a loop over ``wp.tid()``).

Vectors are value types of float32 (vec*) or float64 (vec*d) components with Warp's operators; ``dot`` sums the
products left to right, ``length`` is the float32 square root of it. Scalar arrays are numpy arrays, vector arrays a
wrapper that hands out copies. The hash grid is a uniform grid of cell h that returns the candidates of the 27 cells
around a point in ascending particle id: the reference's queries only ever keep points within h (its own distance
tests), so the set is Warp's; the ORDER is Warp's hash-cell order in the reference and ascending id here, which
fixes the order of the particle-wall colour sums (particle_walls.py:65-84) that Warp leaves unpinned.

Not reproduced: whether Warp's CPU code generation contracts a * b + c into a fused multiply-add. The comparisons
made with these outputs are therefore within stated tolerances, never bit for bit, except for neighbour rows (integer
ids, id-sorted).

Used by tests/golden/make_step_golden.py only, in a container that holds the reference checkout.
"""

from __future__ import annotations

import ast
import enum
import itertools
import math
import sys
import types
from pathlib import Path

import numpy as np

F32 = np.float32
F64 = np.float64
np.seterr(all="ignore")


def f32(x=0.0):
    return F32(x)


# ------------------------------------------------------------------------------------------------------------ vectors
class Vec:
    """A Warp vector value (copy on every read from an array)."""

    __slots__ = ("c",)
    __array_ufunc__ = None  # numpy scalar * Vec defers to Vec.__rmul__

    def __init__(self, c):
        self.c = list(c)

    def __getitem__(self, k):
        return self.c[k]

    def __setitem__(self, k, v):
        self.c[k] = type(self.c[k])(v)

    def __len__(self):
        return len(self.c)

    def __add__(self, o):
        return Vec([a + b for a, b in zip(self.c, o.c)])

    def __sub__(self, o):
        return Vec([a - b for a, b in zip(self.c, o.c)])

    def __neg__(self):
        return Vec([-a for a in self.c])

    def __mul__(self, s):
        if isinstance(s, Vec):
            raise TypeError("vec * vec is not a Warp operator")
        return Vec([a * s for a in self.c])

    def __rmul__(self, s):
        return Vec([s * a for a in self.c])

    def __truediv__(self, s):
        return Vec([a / s for a in self.c])

    def __repr__(self):
        return f"Vec({[float(a) for a in self.c]})"


class VecType:
    """vec2/vec3/vec4 (float32), vec2d/vec3d (float64), vec3i/vec4i/vec3l (integer): constructor and dtype token."""

    def __init__(self, width: int, scalar, name: str):
        self.width, self.scalar, self.__name__ = width, scalar, name

    def __call__(self, *a):
        if len(a) == 0:
            a = (0,) * self.width
        elif len(a) == 1 and self.width > 1:
            if isinstance(a[0], Vec):
                a = tuple(a[0].c)
            else:
                a = (a[0],) * self.width
        if len(a) != self.width:
            raise TypeError(f"{self.__name__} takes {self.width} components, got {len(a)}")
        return Vec([self.scalar(x) for x in a])

    def __getitem__(self, _):  # annotations such as wp.array[wp.vec3] when evaluated
        return self


def _i32(x):
    return int(x)


def _i64(x):
    return int(x)


def _i8(x):
    return int(x)


def _u64(x):
    return int(x)


def _u16(x):
    return int(x) & 0xFFFF


def _u8(x):
    return int(x) & 0xFF


# ------------------------------------------------------------------------------------------------------------- arrays
class WArr(np.ndarray):
    """A numpy array with the wp.array host methods the reference calls."""

    def zero_(self):
        self[...] = 0

    def fill_(self, v):
        self[...] = v

    def numpy(self):
        return np.asarray(self)

    def assign(self, src):
        self[...] = np.asarray(src).reshape(self.shape)


class VecArray:
    """Array of vectors: ``a[i]`` (or ``a[i, k]``) returns a Vec copy, ``a[i] = v`` stores one."""

    def __init__(self, data: np.ndarray, vt: VecType):
        self.data, self.vt = data.view(WArr), vt

    @property
    def shape(self):
        return self.data.shape[:-1]

    def __getitem__(self, idx):
        return Vec(self.data[idx])

    def __setitem__(self, idx, v):
        self.data[idx] = v.c if isinstance(v, Vec) else v

    def zero_(self):
        self.data[...] = 0

    def numpy(self):
        return np.asarray(self.data)

    def assign(self, src):
        self.data[...] = np.asarray(src).reshape(self.data.shape)


_SCALARS = {}


def _alloc(shape, dtype, fill=0):
    shape = (shape,) if isinstance(shape, (int, np.integer)) else tuple(shape)
    if isinstance(dtype, VecType):
        return VecArray(np.full(shape + (dtype.width,), fill, dtype=np.dtype(dtype.scalar)), dtype)
    dt = _SCALARS.get(dtype, dtype)
    if isinstance(dt, Stub):  # transforms, spatial vectors, matrices: never read on this path
        return VecArray(np.full(shape + (16,), fill, np.float32), VecType(16, F32, "opaque"))
    return np.full(shape, fill, dtype=np.dtype(dt)).view(WArr)


def _array(data, dtype=None, device=None, **_):
    if isinstance(dtype, VecType):
        d = np.asarray(data, dtype=np.dtype(dtype.scalar)).reshape(-1, dtype.width)
        return VecArray(d.copy(), dtype)
    dt = _SCALARS.get(dtype, dtype)
    return np.array(data, dtype=None if dt is None else np.dtype(dt)).view(WArr)


def _copy(dst, src, dest_offset=0, src_offset=0, count=None):
    d = dst.data if isinstance(dst, VecArray) else dst
    s = src.data if isinstance(src, VecArray) else src
    n = len(s) - src_offset if count is None else count
    d[dest_offset:dest_offset + n] = s[src_offset:src_offset + n]


def _clone(a):
    if isinstance(a, VecArray):
        return VecArray(a.data.copy(), a.vt)
    return a.copy()


# ---------------------------------------------------------------------------------------------------------- hash grid
class Grid:
    """Uniform grid of cell ``h`` over the grouped points (group -1 is left out, as Warp's grouped hash grid does):
    queries return the ids of one group in the 27 cells around a point, ascending (module doc)."""

    def __init__(self, q: VecArray, h: float, group: np.ndarray):
        self.h = float(h)
        self.cells: dict[tuple, dict[int, list[int]]] = {}
        x = np.asarray(q.data, np.float64)
        key = np.floor(x / self.h).astype(np.int64)
        for i in range(len(x)):
            g = int(group[i])
            if g == -1:
                continue
            self.cells.setdefault(tuple(key[i]), {}).setdefault(g, []).append(i)

    def query(self, x: Vec, radius, group: int):
        k = np.floor(np.asarray([float(c) for c in x.c]) / self.h).astype(np.int64)
        out: list[int] = []
        for d in itertools.product((-1, 0, 1), repeat=3):
            out.extend(self.cells.get((k[0] + d[0], k[1] + d[1], k[2] + d[2]), {}).get(int(group), ()))
        out.sort()
        return out


# ------------------------------------------------------------------------------------------------------ the stand-in
class Stub:
    """Any name of a module that is not on the liquid step's path; calling it is an error."""

    def __init__(self, name="stub"):
        self._name = name

    def __getattr__(self, k):
        if k.startswith("__"):
            raise AttributeError(k)
        return Stub(f"{self._name}.{k}")

    def __call__(self, *a, **k):
        raise RuntimeError(f"{self._name} is not on the liquid step's path (called by a stand-in run)")

    def __getitem__(self, k):
        return self

    def __mro_entries__(self, bases):
        return (object,)


def _stub_getattr(prefix: str):
    def get(k):
        if k.startswith("__"):
            raise AttributeError(k)
        return Stub(f"{prefix}.{k}")

    return get


_TID = [0]


class Kernel:
    def __init__(self, fn):
        self.fn = fn
        self.__name__ = fn.__name__


def _kernel(fn=None, **_):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


def _func(fn=None, **_):
    if fn is None:
        return lambda f: f
    return fn


def _launch(kernel, dim, inputs=(), device=None, **_):
    args = [F32(a) if isinstance(a, float) else a for a in inputs]
    fn = kernel.fn
    if isinstance(dim, (tuple, list)) and len(dim) > 1:
        for t in itertools.product(*(range(int(d)) for d in dim)):
            _TID[0] = t
            fn(*args)
        return
    n = int(dim[0]) if isinstance(dim, (tuple, list)) else int(dim)
    for t in range(n):
        _TID[0] = t
        fn(*args)


def _atomic_add(arr, *idx_val):
    *idx, v = idx_val
    idx = tuple(int(i) for i in idx)
    old = arr[idx if len(idx) > 1 else idx[0]]
    arr[idx if len(idx) > 1 else idx[0]] = old + v
    return old


def _atomic_max(arr, i, v):
    old = arr[int(i)]
    if v > old:
        arr[int(i)] = v
    return old


def _dot(a, b):
    s = a.c[0] * b.c[0]
    for x, y in zip(a.c[1:], b.c[1:]):
        s = s + x * y
    return s


def _length(a):
    return np.sqrt(_dot(a, a))


def _normalize(a):
    n = _length(a)
    if n > 0:
        return a / n
    return Vec([type(c)(0) for c in a.c])


def _cross(a, b):
    return Vec([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def _max(a, b):
    return a if a > b else b


def _min(a, b):
    return a if a < b else b


def _clamp(x, lo, hi):
    return _min(_max(x, lo), hi)


class Tf:
    """A Warp transform value: translation p (vec3) and rotation q = (x, y, z, w)."""

    __slots__ = ("p", "q")
    __array_ufunc__ = None

    def __init__(self, p, q):
        self.p, self.q = p, tuple(F32(c) for c in q)


class TfArray:
    """Array of transforms, stored [n][7] (p, q)."""

    def __init__(self, data):
        self.data = np.asarray(data, np.float32).reshape(-1, 7).view(WArr)
        self.shape = (len(self.data),)

    def __getitem__(self, i):
        r = self.data[int(i)]
        return Tf(Vec([r[0], r[1], r[2]]), r[3:7])


def _quat_rotate(q, v):
    """v rotated by q: v (2 w^2 - 1) + 2 w (u x v) + 2 u (u . v), u = q.xyz (float32)."""
    u = Vec([q[0], q[1], q[2]])
    w = q[3]
    two = F32(2.0)
    return v * (two * w * w - F32(1.0)) + _cross(u, v) * (two * w) + u * (two * _dot(u, v))


def _tf_inverse(X):
    qc = (-X.q[0], -X.q[1], -X.q[2], X.q[3])
    return Tf(-_quat_rotate(qc, X.p), qc)


def _sign(x):
    return F32(-1.0) if x < 0 else F32(1.0)


class _Device:
    is_cuda = False
    is_cpu = True
    alias = "cpu"


def _capture_while(cond, body, **_):
    while int(cond[0]) != 0:
        body()


def warp_stand_in() -> types.ModuleType:
    wp = types.ModuleType("warp")
    wp.__getattr__ = _stub_getattr("wp")  # everything not defined below
    wp.float32, wp.float64, wp.float16 = F32, F64, np.float16
    wp.int32, wp.int64, wp.int8, wp.uint64, wp.uint16, wp.uint8 = _i32, _i64, _i8, _u64, _u16, _u8
    _SCALARS.update({F32: np.float32, F64: np.float64, float: np.float32, int: np.int32, _i32: np.int32,
                     _i64: np.int64, _i8: np.int8, _u64: np.uint64, _u16: np.uint16, _u8: np.uint8})
    wp.vec2, wp.vec3, wp.vec4 = VecType(2, F32, "vec2"), VecType(3, F32, "vec3"), VecType(4, F32, "vec4")
    wp.vec2d, wp.vec3d = VecType(2, F64, "vec2d"), VecType(3, F64, "vec3d")
    wp.vec3i, wp.vec4i = VecType(3, np.int32, "vec3i"), VecType(4, np.int32, "vec4i")
    wp.vec3l = VecType(3, np.int64, "vec3l")
    wp.transform, wp.spatial_vector, wp.mat33, wp.quat = (Stub("wp.transform"), Stub("wp.spatial_vector"),
                                                         Stub("wp.mat33"), Stub("wp.quat"))

    class _ArrayType:
        def __class_getitem__(cls, item):
            return cls

    wp.array = wp.array2d = wp.array3d = _ArrayType
    wp.kernel, wp.func = _kernel, _func
    wp.struct = lambda cls=None, **_: cls if cls is not None else (lambda c: c)  # noqa: E731
    wp.constant = lambda x: F32(x) if isinstance(x, float) else x  # noqa: E731
    wp.overload = lambda *a, **k: None  # noqa: E731
    wp.pi = F32(math.pi)
    wp.tid = lambda: _TID[0]  # noqa: E731
    wp.launch = _launch
    wp.capture_while = _capture_while
    wp.zeros = lambda shape, dtype=float, device=None, **_: _alloc(shape, dtype, 0)  # noqa: E731
    wp.ones = lambda shape, dtype=float, device=None, **_: _alloc(shape, dtype, 1)  # noqa: E731
    wp.full = lambda shape, value, dtype=float, device=None, **_: _alloc(shape, dtype, value)  # noqa: E731
    wp.array_from = _array
    wp.copy, wp.clone = _copy, _clone
    wp.get_device = lambda d=None: _Device()  # noqa: E731
    wp.atomic_add, wp.atomic_max = _atomic_add, _atomic_max
    wp.dot, wp.length, wp.normalize, wp.cross = _dot, _length, _normalize, _cross
    wp.max, wp.min, wp.clamp, wp.abs = _max, _min, _clamp, abs
    wp.sqrt = np.sqrt
    wp.ceil = np.ceil
    wp.floor = np.floor
    wp.round = np.round
    wp.isfinite = np.isfinite
    wp.hash_grid_point_id = lambda grid, t: t  # noqa: E731 (every thread runs; the order of threads is free)
    wp.hash_grid_query = lambda grid, x, r, group=0: grid.query(x, r, group)  # noqa: E731
    wp.context = types.SimpleNamespace(Device=_Device)
    wp.transform_point = lambda X, p: _quat_rotate(X.q, p) + X.p  # noqa: E731
    wp.transform_vector = lambda X, v: _quat_rotate(X.q, v)  # noqa: E731
    wp.transform_inverse = _tf_inverse
    wp.transform_get_translation = lambda X: X.p  # noqa: E731
    wp.sign = _sign
    return wp


def _with_array(wp):
    """``wp.array(data, dtype=...)`` also serves as the type token in annotations."""

    class _A:
        def __class_getitem__(cls, item):
            return cls

        def __new__(cls, data=None, dtype=None, device=None, **kw):
            return _array(data, dtype, device, **kw)

    wp.array = wp.array2d = _A
    return wp


# ---------------------------------------------------------------------------------------------------- source loading
class _KernelBody(ast.NodeTransformer):
    def __init__(self, consts: dict):
        self.consts = consts

    def visit_Constant(self, node):
        if type(node.value) is float:
            name = self.consts.setdefault(node.value, f"_f32c{len(self.consts)}")
            return ast.copy_location(ast.Name(id=name, ctx=ast.Load()), node)
        return node

    def visit_Call(self, node):
        self.generic_visit(node)
        if isinstance(node.func, ast.Name) and node.func.id == "float":
            node.func = ast.copy_location(ast.Name(id="_f32", ctx=ast.Load()), node.func)
        return node

    def visit_While(self, node):
        self.generic_visit(node)
        t = node.test
        if (isinstance(t, ast.Call) and isinstance(t.func, ast.Attribute) and t.func.attr == "hash_grid_query_next"):
            q, var = t.args
            loop = ast.For(target=ast.Name(id=var.id, ctx=ast.Store()), iter=q, body=node.body, orelse=[])
            return ast.copy_location(loop, node)
        return node


def _is_device_code(fn: ast.FunctionDef) -> bool:
    for d in fn.decorator_list:
        f = d.func if isinstance(d, ast.Call) else d
        if isinstance(f, ast.Attribute) and f.attr in ("kernel", "func"):
            return True
    return False


def _rewrite(tree: ast.Module, consts: dict) -> ast.Module:
    body = []
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and _is_device_code(node):
            for i, stmt in enumerate(node.body):
                node.body[i] = _KernelBody(consts).visit(stmt)
        body.append(node)
    tree.body = body
    return ast.fix_missing_locations(tree)


class ParticleFlags(enum.IntEnum):
    """newton ParticleFlags (newton/_src/geometry/flags.py)."""

    ACTIVE = 1
    PROXY = 2


def _newton_stand_in() -> types.ModuleType:
    nt = types.ModuleType("alloy._vendor.newton")
    nt.__getattr__ = _stub_getattr("newton")
    nt.ParticleFlags = ParticleFlags
    nt.GeoType = types.SimpleNamespace(NONE=0, PLANE=1, HFIELD=2, SPHERE=3, CAPSULE=4, ELLIPSOID=5, CYLINDER=6, BOX=7,
                                       MESH=8, CONE=9, CONVEX_MESH=10, GAUSSIAN=11)
    nt.ShapeFlags = types.SimpleNamespace(COLLIDE_PARTICLES=4)
    nt.BodyFlags = types.SimpleNamespace(DYNAMIC=1, KINEMATIC=2)
    nt.ModelFlags = types.SimpleNamespace(BODY_INERTIAL_PROPERTIES=1, BODY_PROPERTIES=2, SHAPE_PROPERTIES=4)
    return nt


class _StubModule(types.ModuleType):
    def __getattr__(self, k):
        if k.startswith("__"):
            raise AttributeError(k)
        return Stub(f"{self.__name__}.{k}")


def _shape_sdf_module(root: Path) -> types.ModuleType:
    """``eval_shape_sdf`` for box shapes: (phi, phi, grad) from the vendored Newton's own ``sdf_box`` and
    ``sdf_box_grad`` (alloy/_vendor/newton/_src/geometry/kernels.py), rewritten like every device function here.
    Other shape types are not on this stand-in's path."""
    path = root / "alloy" / "_vendor" / "newton" / "_src" / "geometry" / "kernels.py"
    tree = ast.parse(path.read_text(), str(path))
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in ("sdf_box", "sdf_box_grad")]
    consts: dict = {}
    mod = ast.Module(body=keep, type_ignores=[])
    mod = _rewrite(mod, consts)
    ns = {"wp": sys.modules["warp"], "_f32": f32, "abs": abs}
    for v, name in consts.items():
        ns[name] = F32(v)
    exec(compile(mod, str(path), "exec"), ns)
    m = _StubModule("alloy._vendor.newton._src.geometry.soft_contacts_sdf")

    def eval_shape_sdf(geo, scale, x_local, sdf_index, tex):
        if int(geo) != int(GEO_BOX):
            raise RuntimeError(f"shape type {int(geo)} is not on this stand-in's path (boxes only)")
        p = ns["sdf_box"](x_local, scale[0], scale[1], scale[2])
        return p, p, ns["sdf_box_grad"](x_local, scale[0], scale[1], scale[2])

    m.eval_shape_sdf = eval_shape_sdf
    return m


GEO_BOX = 7  # newton GeoType.BOX (newton/_src/geometry/types.py)
PKG = "alloy.solvers.sph"
# The liquid step's modules, in load order; every other sibling module is a stub (its names raise when called).
PATH_MODULES = ("kernels", "bodies", "pressure", "reduce", "boundary_slots", "particle_walls", "soft_walls",
                "boundary", "integrate", "krylov", "solve_driver", "neighbors", "config")


def load_reference(root: Path) -> types.SimpleNamespace:
    """Load the reference's liquid-step modules from ``root`` (an alloy checkout) under the stand-in."""
    sph = Path(root) / "alloy" / "solvers" / "sph"
    if not (sph / "pressure.py").exists():
        raise FileNotFoundError(f"{sph} is not the reference's alloy/solvers/sph")
    wp = _with_array(warp_stand_in())
    sys.modules["warp"] = wp
    for name in ("alloy", "alloy._vendor", "alloy.solvers", PKG, "alloy.core"):
        m = types.ModuleType(name)
        m.__path__ = []
        sys.modules[name] = m
    nt = _newton_stand_in()
    sys.modules["alloy._vendor.newton"] = nt
    sys.modules["alloy._vendor"].newton = nt
    for name in ("alloy._vendor.newton._src", "alloy._vendor.newton._src.geometry",
                 "alloy._vendor.newton._src.geometry.kernels", "alloy._vendor.newton._src.geometry.sdf_texture",
                 "alloy._vendor.newton.solvers",
                 "alloy.core.newton_compat", "alloy.core.protocols", "alloy.core.errors", "alloy.solvers.sph.types"):
        sys.modules[name] = _StubModule(name)
    sys.modules["alloy._vendor.newton._src.geometry.soft_contacts_sdf"] = _shape_sdf_module(Path(root))
    for f in sph.glob("*.py"):
        full = f"{PKG}.{f.stem}"
        if f.stem not in PATH_MODULES and full not in sys.modules:
            sys.modules[full] = _StubModule(full)
    mods = {}
    for stem in PATH_MODULES:
        path = sph / f"{stem}.py"
        consts: dict = {}
        tree = _rewrite(ast.parse(path.read_text(), str(path)), consts)
        mod = types.ModuleType(f"{PKG}.{stem}")
        mod.__file__, mod.__package__ = str(path), PKG
        mod.__dict__["_f32"] = f32
        for v, name in consts.items():
            mod.__dict__[name] = F32(v)
        sys.modules[mod.__name__] = mod
        exec(compile(tree, str(path), "exec"), mod.__dict__)
        setattr(sys.modules[PKG], stem, mod)
        mods[stem] = mod
    return types.SimpleNamespace(wp=wp, **mods)
