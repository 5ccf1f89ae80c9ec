"""CPU stand-in for the ``warp`` module, used only to generate golden fixtures.

The reference solver is written against NVIDIA Warp, which is not installed
in the build container.  Its kernels are plain Python functions decorated with
``@wp.kernel``/``@wp.func``; with the decorators made transparent and
``wp.launch`` emulated by a serial loop over thread ids, CPython evaluates the
reference's own kernel bodies in IEEE float64 (no fused multiply-add, libm
transcendentals).  That is the reference algorithm executed literally, which
is what the fixtures under ``tests/golden`` record.

Only ``tests/golden/make_golden.py`` installs this module; nothing in the
package or the benchmarks imports it.
"""

from __future__ import annotations

import ast
import inspect
import itertools
import math
import sys
import textwrap
import types

import numpy as np

_TID: list = [0]


class _Array(np.ndarray):
    """numpy array with the few Warp array methods the reference calls."""

    device = "cpu"

    def numpy(self):
        return np.asarray(self)

    def zero_(self):
        self[...] = 0
        return self


def _wrap(a) -> _Array:
    return np.ascontiguousarray(a).view(_Array)


def _dtype(dtype):
    if dtype in (int, "int32") or getattr(dtype, "__name__", "") == "int32":
        return np.int32
    return np.float64


class _TypeStub:
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        return _TypeStub()

    def __getattr__(self, name):
        return _TypeStub()

    def __getitem__(self, k):
        return _TypeStub()


class _Mat33(np.ndarray):
    """3x3 float64 matrix; ``*`` with a 3-vector is a matrix-vector product."""

    def __mul__(self, other):
        other = np.asarray(other)
        if other.ndim == 1 and other.shape[0] == 3:
            out = np.zeros(3)
            for i in range(3):
                acc = 0.0
                for j in range(3):
                    acc = acc + float(self[i, j]) * float(other[j])
                out[i] = acc
            return out
        return np.asarray(self) * other

    __rmul__ = np.ndarray.__rmul__


def _mat33(*a):
    if len(a) == 1:
        m = np.full((3, 3), float(a[0]))
    else:
        m = np.array([float(x) for x in a], dtype=np.float64).reshape(3, 3)
    return m.view(_Mat33)


def _vec(n):
    def make(*a):
        if not a:
            return np.zeros(n)
        if len(a) == 1:
            return np.full(n, float(a[0]))
        return np.array([float(x) for x in a], dtype=np.float64)

    return make


def _wp_value(v):
    """Warp vectors and matrices are values: binding one to a new name copies it."""
    if isinstance(v, np.ndarray) and not isinstance(v, _Array):
        return v.copy()
    return v


class _CopyOnBind(ast.NodeTransformer):
    """`x = y` with y a bare name becomes `x = _wp_value(y)`."""

    def visit_Assign(self, node):
        if len(node.targets) == 1 and isinstance(node.value, ast.Name):
            node.value = ast.Call(func=ast.Name(id="_wp_value", ctx=ast.Load()),
                                  args=[node.value], keywords=[])
        return node


def _value_semantics(fn):
    """The decorated kernel or function with Warp's value semantics for
    vectors and matrices (NumPy arrays alias on assignment; Warp values do
    not: `fixed = h_old; fixed[0] = 0.0` must leave h_old unchanged)."""
    try:
        src = textwrap.dedent(inspect.getsource(fn))
    except (OSError, TypeError):
        return fn
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    tree = ast.fix_missing_locations(_CopyOnBind().visit(tree))
    glb = fn.__globals__
    glb.setdefault("_wp_value", _wp_value)
    ns: dict = {}
    exec(compile(tree, inspect.getsourcefile(fn) or "<warp>", "exec"), glb, ns)
    return ns[fdef.name]


def _launch(kernel, dim, inputs, device=None, **_kw):
    dims = (dim,) if isinstance(dim, int) else tuple(int(d) for d in dim)
    if len(dims) == 1:
        for t in range(dims[0]):
            _TID[0] = t
            kernel(*inputs)
    else:
        for t in itertools.product(*[range(d) for d in dims]):
            _TID[0] = t
            kernel(*inputs)


def _atomic_add(arr, *args):
    *idx, val = args
    idx = tuple(int(i) for i in idx)
    arr[idx] = arr[idx] + val


def _copy(dst, src, *a, **k):
    dst[...] = np.asarray(src)


def install() -> types.ModuleType:
    wp = types.ModuleType("warp")
    wp.init = lambda: None
    wp.set_module_options = lambda *a, **k: None
    wp.func = _value_semantics
    wp.kernel = _value_semantics
    wp.constant = lambda x: x
    wp.float64 = float
    wp.int32 = int
    wp.vec4i = lambda *a: tuple(int(x) for x in a)
    wp.vec2d = _vec(2)
    wp.vec3d = _vec(3)
    wp.vec4d = _vec(4)
    wp.mat33d = _mat33
    wp.types = types.SimpleNamespace(vector=lambda length, dtype: _vec(length))
    for name in ("array", "array2d", "array3d", "array4d"):
        setattr(wp, name, _TypeStub())
    wp.sqrt = math.sqrt
    wp.log = math.log
    wp.exp = math.exp
    wp.sin = math.sin
    wp.cos = math.cos
    wp.abs = abs
    wp.max = max
    wp.min = min
    wp.dot = lambda a, b: sum(float(x) * float(y) for x, y in zip(a, b))
    wp.outer = lambda a, b: np.outer(a, b).view(_Mat33)
    wp.determinant = lambda m: float(np.linalg.det(np.asarray(m)))
    wp.tid = lambda: _TID[0]
    wp.launch = _launch
    wp.atomic_add = _atomic_add
    wp.copy = _copy
    wp.synchronize_device = lambda *a, **k: None
    wp.is_cuda_available = lambda: False
    wp.get_cuda_device_count = lambda: 0
    wp.get_device = lambda d=None: "cpu"
    wp.array = lambda a, dtype=None, device=None, **k: _wrap(np.array(a, dtype=_dtype(dtype)))
    wp.zeros = lambda shape, dtype=None, device=None, **k: _wrap(np.zeros(shape, _dtype(dtype)))
    wp.zeros_like = lambda a, **k: _wrap(np.zeros_like(np.asarray(a)))
    wp.full = lambda shape, value, dtype=None, device=None, **k: _wrap(
        np.full(shape, value, _dtype(dtype))
    )
    sys.modules["warp"] = wp
    return wp
