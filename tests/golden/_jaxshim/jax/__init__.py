"""A float64 NumPy stand-in for the small part of the JAX API that BMC-JAX's hot path uses.

Test infrastructure only. JAX is not installed in the build container, so the reference package
cannot be imported as it ships. This module lets `tests/golden/make_golden.py` execute the
reference's OWN Python source (its matrix build, time step, event scan, spread average, event
builders and LM loop) eagerly on NumPy arrays in float64, to produce golden vectors that pin the
oracle and the CUDA path to the reference's behaviour rather than to a restatement of it.

What is provided, and with which semantics:
  jax.numpy      NumPy, with arrays carrying JAX's functional `.at[idx].set/add/get`.
  jax.lax        scan / cond / switch executed eagerly (a Python loop / a Python `if`).
  jax.vmap       a Python loop over the mapped axis, outputs stacked (pytrees of NamedTuples).
  jax.jit, jax.checkpoint   identity decorators.
  jax.scipy.linalg.expm     scipy.linalg.expm (float64 scaling and squaring, as JAX's x64 path).
  jax.jacfwd / jax.jacrev   central finite differences (step 1e-6 relative). Used only for loose
                            cross-checks of fitted results; exact Jacobians come from the oracle.
  jax.config     update/read of jax_enable_x64 (always float64 here).
Anything else raises AttributeError, so an unsupported call cannot pass silently.
"""
import sys
import types
import contextlib

import numpy as _np
import scipy.linalg as _sla

__version__ = "0.0-numpy-standin"


# --------------------------------------------------------------------------------------------
# arrays with the functional update syntax
# --------------------------------------------------------------------------------------------
class _AtIndex:
    def __init__(self, arr, idx):
        self._arr, self._idx = arr, idx

    def set(self, v):
        out = _np.array(self._arr, copy=True).view(Array)
        out[self._idx] = _np.asarray(v)
        return out

    def add(self, v):
        out = _np.array(self._arr, copy=True).view(Array)
        out[self._idx] += _np.asarray(v)
        return out

    def multiply(self, v):
        out = _np.array(self._arr, copy=True).view(Array)
        out[self._idx] *= _np.asarray(v)
        return out

    def get(self):
        return _wrap(_np.asarray(self._arr)[self._idx])


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIndex(self._arr, idx)


class Array(_np.ndarray):
    @property
    def at(self):
        return _At(self)


def _wrap(x):
    if isinstance(x, Array):
        return x
    if isinstance(x, _np.ndarray):
        return x.view(Array)
    if isinstance(x, (_np.generic,)):
        return _np.asarray(x).view(Array)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


# --------------------------------------------------------------------------------------------
# jax.numpy
# --------------------------------------------------------------------------------------------
numpy = types.ModuleType("jax.numpy")
_PASSTHROUGH = {"pi", "e", "inf", "nan", "newaxis", "float32", "float64", "int32", "int64",
                "bool_", "floating", "integer", "dtype", "ndarray", "issubdtype", "complex64",
                "complex128", "uint8"}


def _np_getattr(name):
    if name in _PASSTHROUGH:
        return getattr(_np, name)
    f = getattr(_np, name)
    if not callable(f):
        return f

    def g(*a, **k):
        return _wrap(f(*a, **k))
    g.__name__ = name
    return g


numpy.__getattr__ = _np_getattr
numpy.linalg = types.SimpleNamespace(
    solve=lambda a, b: _wrap(_np.linalg.solve(a, b)),
    norm=lambda *a, **k: _wrap(_np.linalg.norm(*a, **k)),
    inv=lambda a: _wrap(_np.linalg.inv(a)),
    pinv=lambda a: _wrap(_np.linalg.pinv(a)))


# --------------------------------------------------------------------------------------------
# pytrees
# --------------------------------------------------------------------------------------------
def _is_namedtuple(x):
    return isinstance(x, tuple) and hasattr(x, "_fields")


def _tree_map(f, tree, *rest):
    if _is_namedtuple(tree):
        return type(tree)(*[_tree_map(f, a, *[r[i] for r in rest]) for i, a in enumerate(tree)])
    if isinstance(tree, (tuple, list)):
        return type(tree)(_tree_map(f, a, *[r[i] for r in rest]) for i, a in enumerate(tree))
    if isinstance(tree, dict):
        return {k: _tree_map(f, tree[k], *[r[k] for r in rest]) for k in tree}
    if tree is None:
        return None
    return f(tree, *rest)


def _leaves(tree):
    out = []
    _tree_map(lambda a: out.append(a), tree)
    return out


tree = types.ModuleType("jax.tree")
tree.map = _tree_map
tree.leaves = _leaves
tree_util = types.ModuleType("jax.tree_util")
tree_util.tree_map = _tree_map
tree_util.tree_leaves = _leaves


def _stack(results):
    first = results[0]
    if first is None:
        return None
    return _tree_map(lambda *xs: _wrap(_np.stack([_np.asarray(x) for x in xs])), first, *results[1:])


# --------------------------------------------------------------------------------------------
# transformations
# --------------------------------------------------------------------------------------------
def jit(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


def checkpoint(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


def vmap(fun, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        sizes = set()
        for a, ax in zip(args, axes):
            if ax is not None:
                for leaf in _leaves(a):
                    sizes.add(_np.shape(leaf)[ax])
        if len(sizes) != 1:
            raise ValueError(f"vmap: inconsistent mapped sizes {sizes}")
        n = sizes.pop()
        outs = []
        for i in range(n):
            sl = [a if ax is None else _tree_map(lambda x, i=i, ax=ax: _wrap(_np.take(_np.asarray(x), i, axis=ax)), a)
                  for a, ax in zip(args, axes)]
            outs.append(fun(*sl))
        return _stack(outs)
    return mapped


def eval_shape(fun, *args):
    return fun(*args)


def _jac(fun, argnums=0):
    def jac(*args):
        x = _np.asarray(args[argnums], dtype=_np.float64)
        f0 = _np.asarray(fun(*args))
        J = _np.empty(f0.shape + x.shape)
        for j in _np.ndindex(x.shape):
            h = 1e-6 * max(1.0, abs(float(x[j])))
            xp = x.copy(); xp[j] += h
            xm = x.copy(); xm[j] -= h
            ap = list(args); ap[argnums] = _wrap(xp)
            am = list(args); am[argnums] = _wrap(xm)
            J[(...,) + j] = (_np.asarray(fun(*ap)) - _np.asarray(fun(*am))) / (2 * h)
        return _wrap(J)
    return jac


jacfwd = _jac
jacrev = _jac


def clear_caches():
    pass


@contextlib.contextmanager
def default_matmul_precision(p):
    yield


# --------------------------------------------------------------------------------------------
# jax.lax
# --------------------------------------------------------------------------------------------
lax = types.ModuleType("jax.lax")


def _cond(pred, true_fun, false_fun, *operands, **kw):
    if "operand" in kw:
        operands = (kw["operand"],)
    return true_fun(*operands) if bool(_np.asarray(pred)) else false_fun(*operands)


def _switch(index, branches, *operands):
    i = int(_np.clip(int(_np.asarray(index)), 0, len(branches) - 1))
    return branches[i](*operands)


def _scan(f, init, xs, length=None, **kw):
    if xs is None:
        n = int(length)
        items = [None] * n
    else:
        n = _np.shape(_leaves(xs)[0])[0]
        items = [_tree_map(lambda a, i=i: _wrap(_np.asarray(a)[i]), xs) for i in range(n)]
    carry, ys = init, []
    for it in items:
        carry, y = f(carry, it)
        ys.append(y)
    return carry, (_stack(ys) if n else None)


lax.cond = _cond
lax.switch = _switch
lax.scan = _scan


# --------------------------------------------------------------------------------------------
# jax.scipy.linalg, jax.config
# --------------------------------------------------------------------------------------------
scipy = types.ModuleType("jax.scipy")
scipy.linalg = types.ModuleType("jax.scipy.linalg")
scipy.linalg.expm = lambda A: _wrap(_sla.expm(_np.asarray(A, dtype=_np.float64)))


class _Config:
    def __init__(self):
        self._v = {"jax_enable_x64": True}

    def update(self, k, v):
        self._v[k] = v

    def read(self, k):
        return self._v.get(k, True)


config = _Config()

for _name, _mod in {"jax.numpy": numpy, "jax.lax": lax, "jax.scipy": scipy,
                    "jax.scipy.linalg": scipy.linalg, "jax.tree": tree,
                    "jax.tree_util": tree_util}.items():
    sys.modules[_name] = _mod
