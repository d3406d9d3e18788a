"""A numpy stand-in for the few Taichi names that SeisWave_Taichi's solver
modules use, so that the reference's own source files run unmodified on small
grids in this image (which has no Taichi).  Test infrastructure only: the
fixtures it helps write (tests/golden/reference_small.npz, by
tests/golden/make_reference_golden.py) pin the oracle and the CUDA kernels to
the reference's own code.

Names provided: field, ndrange, kernel, func, data_oriented, exp, log, sqrt,
f32, f64, i32 -- the whole Taichi surface of src/Elastic2D_CPML.py,
src/Elastic3D_SSG_CPML.py, src/Elastic3D_SSG_Tensor.py,
src/Elastic3D_SSG_SPML.py, src/Differential2D.py, src/Differential3D.py and
src/BaseFun.py (a grep of `ti.` over those files).

What is emulated, and why it matters for bit-level parity:

* Python scope runs as plain Python, as under Taichi: a field element read
  there is a Python float (the float32 value widened), a write rounds to the
  field's type.  This is how the reference's SetADEPML2D/3D compute the PML
  profiles in float64 from float32-rounded values.
* Kernel scope (@ti.kernel and the @ti.func's it calls) is typed the way
  Taichi's frontend types it, with default_fp = f32 and default_ip = i32:
  - a field element read is a numpy scalar of the field's type, and numpy 2's
    promotion rules (NEP 50: Python scalars are "weak") make every operation
    with a float32 operand a float32 operation, as Taichi's f32 IR is;
  - an expression of Python values only (`pi**2`, `1.5/self.f0`) is folded in
    Python (float64), as Taichi's AST builder folds it, and becomes f32 when
    it meets a typed value or is assigned;
  - assigning to a local name (`dx=self.dx`) and passing a Python float to a
    @ti.func make an f32 variable (Taichi's expr_init);
  - kernel arguments are cast to their annotation (`nt:int`, `source:ti.f32`);
  - `x**n` with a non-negative integer constant n on a typed value is
    evaluated by repeated multiplication, as Taichi demotes integer powers
    (numpy's float32 scalar power calls powf, which is not always the
    correctly rounded x*x).
  These rules are applied by rewriting each kernel's and func's syntax tree
  once (the same source Taichi parses), not by editing the reference files.
* Top-level loops of a kernel run one after another in source order with the
  serial statements between them, i.e. Taichi's sequence of offloaded tasks;
  every reference loop is a pure map over its range, so running a parallel
  loop serially gives the parallel result.
* Indices are bounds-checked (Taichi's debug mode): an out-of-range access
  raises IndexError instead of silently touching another cell.

exp/log/sqrt on float32 values use numpy's float32 routines (Taichi uses the
backend's libm or device intrinsics; they may differ in the last bit, which
the parity tests' tolerance covers and their bit-exactness report shows).
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

f32 = np.float32
f64 = np.float64
i32 = np.int32
i64 = np.int64
u8 = np.uint8

_DEFAULT_FP = np.float32
_DEFAULT_IP = np.int32
_state = {"depth": 0}


def _np_type(dtype):
    if dtype is None or dtype is float:
        return _DEFAULT_FP
    if dtype is int:
        return _DEFAULT_IP
    return np.dtype(dtype).type


class Field:
    """Dense zero-initialised array with Taichi's indexing rules."""

    def __init__(self, dtype=None, shape=()):
        if isinstance(shape, (int, np.integer)):
            shape = (int(shape),)
        self.dtype = _np_type(dtype)
        self.a = np.zeros(tuple(int(s) for s in shape), dtype=self.dtype)
        self.shape = self.a.shape

    def _idx(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        if len(idx) != self.a.ndim:
            raise IndexError(f"field of rank {self.a.ndim} indexed with {len(idx)} indices")
        out = []
        for v, n in zip(idx, self.shape):
            v = int(v)
            if v < 0 or v >= n:
                raise IndexError(f"index {idx} out of range for shape {self.shape}")
            out.append(v)
        return tuple(out)

    def __getitem__(self, idx):
        v = self.a[self._idx(idx)]
        return v if _state["depth"] > 0 else v.item()

    def __setitem__(self, idx, value):
        self.a[self._idx(idx)] = value

    def to_numpy(self):
        return self.a.copy()

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        if arr.shape != self.shape:
            raise ValueError(f"from_numpy: shape {arr.shape} != {self.shape}")
        self.a[...] = arr.astype(self.dtype)

    def fill(self, value):
        self.a.fill(value)


def field(dtype=None, shape=(), **kw):
    if "dtype" in kw:
        dtype = kw.pop("dtype")
    return Field(dtype, shape)


def ndrange(*args):
    ranges = []
    for a in args:
        if isinstance(a, (tuple, list)):
            ranges.append(range(int(a[0]), int(a[1])))
        else:
            ranges.append(range(int(a)))
    if len(ranges) == 1:
        return ranges[0]
    return itertools.product(*ranges)


def _unary(npf, mf):
    def op(x):
        if isinstance(x, np.generic):
            return npf(x)
        return mf(x)
    return op


exp = _unary(np.exp, math.exp)
log = _unary(np.log, math.log)
sqrt = _unary(np.sqrt, math.sqrt)


def _ti_var(v):
    """Taichi's expr_init: a Python float becomes an f32 variable."""
    if isinstance(v, bool):
        return v
    if isinstance(v, float):
        return _DEFAULT_FP(v)
    return v


def _ti_pow(x, n):
    """x ** n as Taichi lowers it: Python values fold in Python; a typed value
    raised to a non-negative integer constant is repeated multiplication."""
    if not isinstance(x, np.generic) and not isinstance(n, np.generic):
        return x ** n
    if isinstance(n, (int, np.integer)) and not isinstance(n, bool) and int(n) >= 0:
        n = int(n)
        result = None
        base = x
        while n > 0:
            if n & 1:
                result = base if result is None else result * base
            n >>= 1
            if n:
                base = base * base
        return result if result is not None else type(x)(1)
    return np.power(x, n)


class _Rewrite(ast.NodeTransformer):
    def visit_Assign(self, node):
        self.generic_visit(node)
        if all(isinstance(t, ast.Name) for t in node.targets):
            node.value = ast.Call(func=ast.Name("__ti_var", ast.Load()), args=[node.value], keywords=[])
        return node

    def visit_BinOp(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Pow):
            return ast.Call(func=ast.Name("__ti_pow", ast.Load()), args=[node.left, node.right], keywords=[])
        return node


def _rewrite(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    tree = ast.fix_missing_locations(_Rewrite().visit(tree))
    g = fn.__globals__
    g.setdefault("__ti_var", _ti_var)
    g.setdefault("__ti_pow", _ti_pow)
    ns = {}
    exec(compile(tree, inspect.getsourcefile(fn) or "<ti>", "exec"), g, ns)
    out = ns[fdef.name]
    out.__wrapped_source__ = fn
    return out


def _cast_arg(v, ann):
    if ann is inspect.Parameter.empty:
        return v
    if ann is int or ann is i32 or ann is i64:
        return int(v)
    if ann is float:
        return _DEFAULT_FP(v)
    if ann is f32 or ann is f64:
        return ann(v)
    return v


def kernel(fn):
    body = _rewrite(fn)
    sig = inspect.signature(fn)

    def call(*args, **kw):
        bound = sig.bind(*args, **kw)
        for name, v in list(bound.arguments.items()):
            if name != "self":
                bound.arguments[name] = _cast_arg(v, sig.parameters[name].annotation)
        _state["depth"] += 1
        try:
            return body(*bound.args, **bound.kwargs)
        finally:
            _state["depth"] -= 1

    call.__name__ = fn.__name__
    call.__doc__ = fn.__doc__
    return call


def func(fn):
    body = _rewrite(fn)

    def call(*args, **kw):
        args = [_ti_var(a) for a in args]
        kw = {k: _ti_var(v) for k, v in kw.items()}
        return body(*args, **kw)

    call.__name__ = fn.__name__
    return call


def data_oriented(cls):
    return cls


def static(x):
    return x


def init(*args, **kw):
    return None


def sync():
    return None


def install():
    """Register this module as `taichi` (and an inert matplotlib, which the
    reference's 2D module imports for plotting only) in sys.modules."""
    me = sys.modules[__name__]
    sys.modules["taichi"] = me
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        plt = types.ModuleType("matplotlib.pyplot")
        mpl.pyplot = plt
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = plt
    return me
