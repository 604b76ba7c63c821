"""A minimal numpy stand-in for the parts of JAX that dftax's DF path uses.

Test infrastructure only. ``make_golden.py`` uses it to run dftax's OWN
integral, metric and energy code (the reference's Python source, unmodified)
in a container where JAX is not installed, so that the golden fixtures under
``tests/golden/`` are outputs of the reference itself rather than of a
restatement.

What is covered is exactly what the reference's DF path touches:
``jax.numpy`` array functions and the ``.at[...]`` update syntax,
``jax.vmap`` (a Python loop over the mapped axis), ``jax.jit`` (identity),
``jax.custom_jvp`` (forward only), ``lax.fori_loop``, the block forms of
``lax.gather`` / ``lax.scatter`` used by ``eri3c_bucketed``, the incomplete
gamma functions (scipy), ``equinox.Module`` (a dataclass) and the
``jaxtyping`` annotation names. Arithmetic is numpy float64, i.e. the same
IEEE operations XLA performs on CPU up to reduction order.
"""

from __future__ import annotations

import dataclasses
import sys
import types

import numpy as np
import scipy.special as _sps


# ---------------------------------------------------------------------------
# Array type with the functional ``.at[...]`` update syntax
# ---------------------------------------------------------------------------

class JArr(np.ndarray):
    """ndarray with JAX's ``x.at[idx].set(v)`` / ``.add(v)`` copy-on-update."""

    @property
    def at(self):
        return _At(self)


class _At:
    def __init__(self, a):
        self._a = a

    def __getitem__(self, idx):
        return _AtIdx(self._a, idx)


class _AtIdx:
    def __init__(self, a, idx):
        self._a, self._idx = a, idx

    def set(self, v, **_):
        out = np.array(self._a, copy=True)
        out[self._idx] = np.asarray(v)
        return out.view(JArr)

    def add(self, v, **_):
        out = np.array(self._a, copy=True)
        np.add.at(out, self._idx, np.asarray(v))
        return out.view(JArr)

    def get(self, **_):
        return _wrap(np.asarray(self._a)[self._idx])


def _wrap(r):
    if isinstance(r, np.ndarray) and not isinstance(r, JArr):
        return r.view(JArr)
    if isinstance(r, tuple):
        return tuple(_wrap(x) for x in r)
    if isinstance(r, list):
        return [_wrap(x) for x in r]
    if isinstance(r, (np.floating, np.integer, np.bool_, float, int)):
        return np.asarray(r).view(JArr)
    return r


def _w(f):
    def g(*a, **k):
        return _wrap(f(*a, **k))
    g.__name__ = getattr(f, "__name__", "f")
    return g


# ---------------------------------------------------------------------------
# jax.numpy
# ---------------------------------------------------------------------------

jnp = types.ModuleType("jax.numpy")
for _name in (
    "zeros", "zeros_like", "ones", "ones_like", "arange", "concatenate", "stack",
    "where", "sum", "einsum", "exp", "sqrt", "maximum", "minimum", "clip",
    "round", "log", "dot", "meshgrid", "abs", "max", "min", "full", "eye",
    "tril_indices", "triu_indices", "outer", "matmul", "transpose", "swapaxes",
    "prod", "cumsum", "empty", "diag", "trace", "isfinite", "allclose",
    "linspace", "floor", "ceil", "sign", "square", "power", "take", "tile",
    "repeat", "broadcast_to", "expand_dims", "moveaxis", "mean", "all", "any",
    "argmax", "argsort", "sort", "nonzero", "reshape", "ravel", "cos", "sin",
    "arccos", "arctan2", "cbrt", "convolve", "flip", "triu", "tril", "erf" if hasattr(np, "erf") else "exp",
):
    setattr(jnp, _name, _w(getattr(np, _name)))
jnp.einsum = _w(lambda *a, **k: np.einsum(*a, optimize=True, **k))
jnp.asarray = _w(lambda a, dtype=None: np.asarray(a, dtype=dtype))
jnp.array = _w(lambda a, dtype=None, copy=True: np.array(a, dtype=dtype))
jnp.issubdtype = np.issubdtype
jnp.floating = np.floating
jnp.integer = np.integer
jnp.finfo = np.finfo
jnp.float64 = np.float64
jnp.float32 = np.float32
jnp.int32 = np.int32
jnp.int64 = np.int64
jnp.bool_ = np.bool_
jnp.pi = np.pi
jnp.inf = np.inf
jnp.nan = np.nan
jnp.ndarray = np.ndarray
jnp.linalg = types.SimpleNamespace(
    eigh=_w(np.linalg.eigh), inv=_w(np.linalg.inv), solve=_w(np.linalg.solve),
    cholesky=_w(np.linalg.cholesky), norm=_w(np.linalg.norm),
)


# ---------------------------------------------------------------------------
# jax.vmap / jit / custom_jvp / lax
# ---------------------------------------------------------------------------

def _stack_tree(outs):
    first = outs[0]
    if isinstance(first, tuple):
        return tuple(_stack_tree([o[i] for o in outs]) for i in range(len(first)))
    return np.stack([np.asarray(o) for o in outs]).view(JArr)


def vmap(fun, in_axes=0, out_axes=0, *args, **kwargs):
    """Python-loop ``vmap``: maps ``fun`` over the given axis of each argument."""

    def mapped(*a):
        axes = (tuple(in_axes) if isinstance(in_axes, (tuple, list))
                else (in_axes,) * len(a))
        n = None
        for x, ax in zip(a, axes):
            if ax is not None:
                n = np.shape(x)[ax]
                break
        outs = []
        for i in range(n):
            sub = [x if ax is None else _wrap(np.take(np.asarray(x), i, axis=ax))
                   for x, ax in zip(a, axes)]
            outs.append(fun(*sub))
        if n == 0:
            raise ValueError("vmap over an empty axis is not supported by the shim")
        return _stack_tree(outs)

    return mapped


def jit(fun=None, **_):
    if fun is None:
        return lambda f: f
    return fun


class custom_jvp:
    """Forward-only ``jax.custom_jvp``: calls the primal; ``defjvp`` records."""

    def __init__(self, fun, **_):
        self.fun = fun
        self.jvp = None

    def __call__(self, *a, **k):
        return self.fun(*a, **k)

    def defjvp(self, jvp):
        self.jvp = jvp
        return jvp


class custom_vjp(custom_jvp):
    def defvjp(self, fwd, bwd):
        self.fwdbwd = (fwd, bwd)


def fori_loop(lo, hi, body, init):
    val = init
    for i in range(lo, hi):
        val = body(i, val)
    return val


def scan(f, init, xs, length=None):
    carry, ys = init, []
    n = length if xs is None else np.shape(xs)[0]
    for i in range(n):
        carry, y = f(carry, None if xs is None else xs[i])
        ys.append(y)
    return carry, (None if ys[0] is None else _stack_tree(ys))


def _scatter(out, starts, vals, dnums, **_):
    """Block scatter as used by ``eri3c_bucketed._scatter_blocks``."""
    res = np.array(out, copy=True)
    vals = np.asarray(vals)
    win = vals.shape[1:]
    for s, v in zip(np.asarray(starts), vals):
        res[tuple(slice(int(a), int(a) + w) for a, w in zip(s, win))] = v
    return res.view(JArr)


def _gather(x, starts, dnums, slice_sizes, **_):
    """Block row gather as used by ``eri3c_bucketed._gather_rows``."""
    x = np.asarray(x)
    n = slice_sizes[0]
    return np.stack([x[int(s[0]):int(s[0]) + n] for s in np.asarray(starts)]).view(JArr)


lax = types.ModuleType("jax.lax")
lax.fori_loop = fori_loop
lax.scan = scan
lax.scatter = _scatter
lax.gather = _gather
lax.ScatterDimensionNumbers = lambda **k: k
lax.GatherDimensionNumbers = lambda **k: k
lax.GatherScatterMode = types.SimpleNamespace(PROMISE_IN_BOUNDS="promise")
lax.stop_gradient = lambda x: x

special = types.ModuleType("jax.scipy.special")
special.gammainc = _w(_sps.gammainc)
special.gammaln = _w(_sps.gammaln)
special.erf = _w(_sps.erf)
jscipy = types.ModuleType("jax.scipy")
jscipy.special = special

jax = types.ModuleType("jax")
jax.numpy = jnp
jax.lax = lax
jax.scipy = jscipy
jax.vmap = vmap
jax.jit = jit
jax.custom_jvp = custom_jvp
jax.custom_vjp = custom_vjp
jax.checkpoint = lambda f, **_: f
jax.config = types.SimpleNamespace(read=lambda *_: True, update=lambda *_: None)
jax.Array = np.ndarray


# ---------------------------------------------------------------------------
# equinox / jaxtyping
# ---------------------------------------------------------------------------

class Module:
    """``eqx.Module`` stand-in: subclasses become keyword-constructible dataclasses."""

    def __init_subclass__(cls, **kw):
        super().__init_subclass__(**kw)
        dataclasses.dataclass(cls)


def field(*, static=False, default=dataclasses.MISSING, **_):
    if default is dataclasses.MISSING:
        return dataclasses.field()
    return dataclasses.field(default=default)


eqx = types.ModuleType("equinox")
eqx.Module = Module
eqx.field = field
eqx.filter_jit = jit
eqx.is_inexact_array = lambda x: isinstance(x, np.ndarray)


class _Subscriptable:
    def __getitem__(self, item):
        return self

    def __or__(self, other):
        return self

    def __ror__(self, other):
        return self


jaxtyping = types.ModuleType("jaxtyping")
for _n in ("Array", "Float", "Int", "Scalar", "Bool", "PyTree", "Shaped"):
    setattr(jaxtyping, _n, _Subscriptable())


def install():
    """Register the stand-ins in ``sys.modules`` (idempotent)."""
    sys.modules.setdefault("jax", jax)
    sys.modules.setdefault("jax.numpy", jnp)
    sys.modules.setdefault("jax.lax", lax)
    sys.modules.setdefault("jax.scipy", jscipy)
    sys.modules.setdefault("jax.scipy.special", special)
    sys.modules.setdefault("equinox", eqx)
    sys.modules.setdefault("jaxtyping", jaxtyping)
