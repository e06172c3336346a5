"""A numpy stand-in for the subset of JAX that microcosmos's physics hot path uses.

Test infrastructure only. JAX is not installed in this environment, so this module
is installed as ``jax`` in ``sys.modules`` by ``make_golden.py`` before the reference
package (``src/microcosmos``) is imported from its source tree. The reference code then
runs unmodified on numpy float32 arrays and its outputs become the golden fixtures in
this directory.

Semantics reproduced (JAX with x64 disabled):
  * float64 inputs become float32 and int64 becomes int32; an int array combined with
    a float operand is promoted to float32 (JAX's lattice) rather than float64;
  * ``x.at[idx].add(v)`` / ``.set(v)`` return updated copies (sequential ``np.add.at``,
    i.e. updates applied in index order);
  * ``jit`` is the identity, ``vmap`` loops over the leading axis, ``lax.scan`` and
    ``lax.fori_loop`` are Python loops, ``stop_gradient`` is the identity;
  * ``jax.scipy.ndimage.map_coordinates(order=1, mode="wrap")`` follows JAX's
    formulation: per-axis (floor, floor+1) nodes with weights (1-t, t), indices
    wrapped by floored modulo, terms taken in ``itertools.product`` order, weights
    multiplied in axis order and terms added left to right.
Arithmetic differs from XLA's only by summation order inside reductions and by the
transcendental implementations (numpy's float32 cos/sin/exp vs XLA's).
"""
from __future__ import annotations

import dataclasses
import functools
import itertools
import sys
import types

import numpy as np


# ----------------------------------------------------------------------------- dtype rules
def _canon_dtype(dt):
    dt = np.dtype(dt)
    if dt == np.float64:
        return np.dtype(np.float32)
    if dt == np.int64:
        return np.dtype(np.int32)
    if dt == np.complex128:
        return np.dtype(np.complex64)
    if dt == np.uint64:
        return np.dtype(np.uint32)
    return dt


def _canon(x):
    """Convert any array-like to a float32/int32 `Arr` (JAX x64-off canonicalisation)."""
    if isinstance(x, Arr):
        return x
    a = np.asarray(x)
    a = a.astype(_canon_dtype(a.dtype), copy=False)
    return a.view(Arr)


def _is_py_scalar(x):
    return isinstance(x, (bool, int, float, complex)) and not isinstance(x, np.generic)


def _coerce_inputs(inputs):
    """JAX-like promotion for a ufunc call: if any operand is floating, cast int operands
    to float32; 64-bit arrays become 32-bit.  Python scalars stay weak."""
    arrs = []
    any_float = False
    any_complex = False
    for x in inputs:
        if _is_py_scalar(x):
            arrs.append(x)
            continue
        a = np.asarray(x)
        if isinstance(x, Arr):
            a = x.view(np.ndarray)
        a = a.astype(_canon_dtype(a.dtype), copy=False)
        if np.issubdtype(a.dtype, np.complexfloating):
            any_complex = True
        elif np.issubdtype(a.dtype, np.floating):
            any_float = True
        arrs.append(a)
    if any_float or any_complex:
        target = np.complex64 if any_complex else np.float32
        out = []
        for a in arrs:
            if isinstance(a, np.ndarray) and (np.issubdtype(a.dtype, np.integer) or a.dtype == np.bool_):
                out.append(a.astype(target))
            elif isinstance(a, np.ndarray) and any_complex and np.issubdtype(a.dtype, np.floating):
                out.append(a)
            else:
                out.append(a)
        arrs = out
    return arrs


class _AtIndexer:
    def __init__(self, arr, idx):
        self.arr = arr
        self.idx = idx

    def add(self, v):
        out = np.array(self.arr.view(np.ndarray), copy=True)
        v = np.asarray(v)
        if not _is_py_scalar(v):
            v = v.astype(out.dtype, copy=False)
        np.add.at(out, _plain_idx(self.idx), v)
        return out.view(Arr)

    def set(self, v):
        out = np.array(self.arr.view(np.ndarray), copy=True)
        out[_plain_idx(self.idx)] = np.asarray(v).astype(out.dtype, copy=False)
        return out.view(Arr)

    def get(self):
        return self.arr[self.idx]


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIndexer(self.arr, idx)


def _plain_idx(idx):
    if isinstance(idx, tuple):
        return tuple(_plain_idx(i) for i in idx)
    if isinstance(idx, Arr):
        return idx.view(np.ndarray)
    return idx


class Arr(np.ndarray):
    """ndarray with JAX-style `.at` updates and x64-off dtype promotion."""

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        ins = _coerce_inputs(inputs)
        if "out" in kwargs:
            kwargs["out"] = tuple(o.view(np.ndarray) if isinstance(o, Arr) else o for o in kwargs["out"])
        res = getattr(ufunc, method)(*ins, **kwargs)
        return _wrap(res)

    def __array_function__(self, func, types_, args, kwargs):
        def unwrap(x):
            if isinstance(x, Arr):
                return x.view(np.ndarray)
            if isinstance(x, (list, tuple)):
                return type(x)(unwrap(i) for i in x)
            return x
        res = func(*unwrap(args), **{k: unwrap(v) for k, v in kwargs.items()})
        return _wrap(res)

    def __getitem__(self, idx):
        res = np.ndarray.__getitem__(self.view(np.ndarray), _plain_idx(idx))
        return _wrap(res)

    @property
    def at(self):
        return _At(self)

    def astype(self, dtype, *a, **k):
        if dtype is int:
            dtype = np.int32
        if dtype is float:
            dtype = np.float32
        return _wrap(np.ndarray.astype(self.view(np.ndarray), _canon_dtype(dtype)))

    def __float__(self):
        return float(self.view(np.ndarray))

    def __int__(self):
        return int(self.view(np.ndarray))

    def __bool__(self):
        return bool(self.view(np.ndarray))

    def __index__(self):
        return int(self.view(np.ndarray))

    def block_until_ready(self):
        return self


def _wrap(res):
    if isinstance(res, tuple):
        return tuple(_wrap(r) for r in res)
    if isinstance(res, list):
        return [_wrap(r) for r in res]
    if isinstance(res, (np.ndarray, np.generic)):
        a = np.asarray(res)
        a = a.astype(_canon_dtype(a.dtype), copy=False)
        return a.view(Arr)
    return res


# ----------------------------------------------------------------------------- jax.numpy
def _make_jnp():
    jnp = types.ModuleType("jax.numpy")

    def passthrough(name):
        f = getattr(np, name)

        @functools.wraps(f)
        def g(*args, **kw):
            args = [(_canon(a) if isinstance(a, (np.ndarray, list)) and not isinstance(a, Arr) and name not in ("stack", "concatenate") else a) for a in args]
            if "dtype" in kw and kw["dtype"] is not None:
                kw["dtype"] = _canon_dtype(kw["dtype"] if kw["dtype"] not in (int, float) else (np.int32 if kw["dtype"] is int else np.float32))
            return _wrap(f(*args, **kw))
        return g

    for name in ["floor", "abs", "cos", "sin", "exp", "sqrt", "where", "maximum", "minimum",
                 "sum", "mean", "roll", "flip", "mod", "arctan2", "arctan", "tan", "isfinite",
                 "all", "any", "allclose", "moveaxis", "argmax", "clip", "repeat", "tile",
                 "meshgrid", "square", "log", "isnan", "prod", "max", "min", "sign", "round",
                 "transpose", "reshape", "full_like", "ones_like", "linspace", "cumsum",
                 "expand_dims", "squeeze", "diff", "dot", "outer", "cross", "atleast_1d", "broadcast_to"]:
        setattr(jnp, name, passthrough(name))

    def zeros(shape, dtype=None):
        return np.zeros(shape, _canon_dtype(dtype or np.float32)).view(Arr)

    def ones(shape, dtype=None):
        return np.ones(shape, _canon_dtype(dtype or np.float32)).view(Arr)

    def full(shape, fill_value, dtype=None):
        if dtype is None:
            fv = np.asarray(fill_value)
            dtype = np.float32 if np.issubdtype(fv.dtype, np.floating) else _canon_dtype(fv.dtype)
        return np.full(shape, fill_value, _canon_dtype(dtype)).view(Arr)

    def zeros_like(a, dtype=None):
        return np.zeros_like(np.asarray(a), dtype=_canon_dtype(dtype or np.asarray(a).dtype)).view(Arr)

    def array(a, dtype=None):
        if isinstance(a, (list, tuple)) and any(isinstance(i, Arr) for i in a):
            a = np.stack([np.asarray(i) for i in a])
        out = np.array(a, dtype=None if dtype is None else _canon_dtype(dtype))
        return _canon(out)

    def asarray(a, dtype=None):
        return array(a, dtype)

    def arange(*args, dtype=None):
        out = np.arange(*args)
        if dtype is not None:
            out = out.astype(_canon_dtype(dtype))
        return _canon(out)

    def stack(arrs, axis=0):
        return _wrap(np.stack([np.asarray(a) for a in _coerce_inputs(arrs)], axis=axis))

    def concatenate(arrs, axis=0):
        return _wrap(np.concatenate([np.asarray(a) for a in _coerce_inputs(arrs)], axis=axis))

    def einsum(spec, *ops):
        ops = _coerce_inputs(ops)
        return _wrap(np.einsum(spec, *[np.asarray(o) for o in ops]))

    def tensordot(a, b, axes=2):
        a, b = _coerce_inputs((a, b))
        return _wrap(np.tensordot(np.asarray(a), np.asarray(b), axes=axes))

    jnp.zeros, jnp.ones, jnp.full, jnp.zeros_like = zeros, ones, full, zeros_like
    jnp.array, jnp.asarray, jnp.arange = array, asarray, arange
    jnp.stack, jnp.concatenate, jnp.einsum, jnp.tensordot = stack, concatenate, einsum, tensordot
    jnp.pi = np.pi
    jnp.inf = np.inf
    jnp.float32, jnp.int32, jnp.float64, jnp.int64 = np.float32, np.int32, np.float64, np.int64
    jnp.uint8 = np.uint8
    jnp.bool_ = np.bool_
    jnp.float_ = np.float32
    jnp.ndarray = Arr
    jnp.finfo = np.finfo

    linalg = types.ModuleType("jax.numpy.linalg")

    def norm(x, axis=None, keepdims=False):
        return _wrap(np.linalg.norm(np.asarray(x), axis=axis, keepdims=keepdims))
    linalg.norm = norm
    jnp.linalg = linalg

    fft = types.ModuleType("jax.numpy.fft")
    fft.fft2 = lambda a: _wrap(np.fft.fft2(np.asarray(a)))
    fft.ifft2 = lambda a: _wrap(np.fft.ifft2(np.asarray(a)))
    fft.fft = lambda a, **k: _wrap(np.fft.fft(np.asarray(a), **k))
    fft.ifft = lambda a, **k: _wrap(np.fft.ifft(np.asarray(a), **k))
    fft.fftfreq = lambda n, d=1.0: _wrap(np.fft.fftfreq(n, d).astype(np.float32))
    jnp.fft = fft
    return jnp


# ----------------------------------------------------------------------------- pytrees
def _tree_stack(items):
    first = items[0]
    if first is None:
        return None
    if dataclasses.is_dataclass(first) and not isinstance(first, type):
        meta = getattr(type(first), "_shim_meta_fields", ())
        kw = {}
        for f in dataclasses.fields(first):
            vals = [getattr(i, f.name) for i in items]
            kw[f.name] = vals[0] if f.name in meta else _tree_stack(vals)
        return type(first)(**kw)
    if isinstance(first, tuple):
        return tuple(_tree_stack([i[k] for i in items]) for k in range(len(first)))
    if isinstance(first, list):
        return [_tree_stack([i[k] for i in items]) for k in range(len(first))]
    return _wrap(np.stack([np.asarray(i) for i in items]))


def _tree_index(tree, i):
    if tree is None:
        return None
    if dataclasses.is_dataclass(tree) and not isinstance(tree, type):
        meta = getattr(type(tree), "_shim_meta_fields", ())
        return type(tree)(**{f.name: (getattr(tree, f.name) if f.name in meta else _tree_index(getattr(tree, f.name), i))
                             for f in dataclasses.fields(tree)})
    if isinstance(tree, (tuple, list)):
        return type(tree)(_tree_index(t, i) for t in tree)
    return tree[i]


def _leading_len(tree):
    if dataclasses.is_dataclass(tree) and not isinstance(tree, type):
        for f in dataclasses.fields(tree):
            v = getattr(tree, f.name)
            if v is not None and f.name not in getattr(type(tree), "_shim_meta_fields", ()):
                return _leading_len(v)
    if isinstance(tree, (tuple, list)):
        for t in tree:
            if t is not None:
                return _leading_len(t)
    return np.asarray(tree).shape[0]


# ----------------------------------------------------------------------------- jax
def _make_jax():
    jax = types.ModuleType("jax")
    jnp = _make_jnp()
    jax.numpy = jnp
    jax.Array = Arr

    def jit(fn=None, **kw):
        if fn is None:
            return lambda f: f
        return fn
    jax.jit = jit

    def vmap(fn, in_axes=0, out_axes=0):
        def g(*args):
            axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
            n = None
            for a, ax in zip(args, axes):
                if ax is not None:
                    n = _leading_len(a)
                    break
            outs = []
            for i in range(n):
                call = [(_tree_index(a, i) if ax is not None else a) for a, ax in zip(args, axes)]
                outs.append(fn(*call))
            return _tree_stack(outs)
        return g
    jax.vmap = vmap

    lax = types.ModuleType("jax.lax")

    def scan(f, init, xs=None, length=None):
        carry = init
        ys = []
        n = length if xs is None else _leading_len(xs)
        for i in range(n):
            x = None if xs is None else _tree_index(xs, i)
            carry, y = f(carry, x)
            ys.append(y)
        if len(ys) == 0 or ys[0] is None:
            return carry, None
        return carry, _tree_stack(ys)

    def fori_loop(lo, hi, body, init):
        v = init
        for i in range(lo, hi):
            v = body(i, v)
        return v
    lax.scan = scan
    lax.fori_loop = fori_loop
    lax.stop_gradient = lambda x: x
    jax.lax = lax

    tree_util = types.ModuleType("jax.tree_util")

    def register_dataclass(cls, meta_fields=(), data_fields=()):
        cls._shim_meta_fields = tuple(meta_fields)
        if not hasattr(cls, "__replace__"):
            cls.__replace__ = lambda self, **kw: dataclasses.replace(self, **kw)
        return cls
    tree_util.register_dataclass = register_dataclass
    tree_util.tree_map = lambda f, *t: f(*t)
    jax.tree_util = tree_util

    scipy = types.ModuleType("jax.scipy")
    ndimage = types.ModuleType("jax.scipy.ndimage")

    def map_coordinates(inp, coordinates, order, mode="constant", cval=0.0):
        assert order == 1 and mode == "wrap"
        inp = np.asarray(inp)
        coords = [np.asarray(c, dtype=np.float32) for c in coordinates]
        per_axis = []
        for c, size in zip(coords, inp.shape):
            lower = np.floor(c)
            upper_w = (c - lower).astype(np.float32)
            lower_w = (np.float32(1) - upper_w).astype(np.float32)
            idx = lower.astype(np.int32)
            per_axis.append([(np.mod(idx, size), lower_w), (np.mod(idx + 1, size), upper_w)])
        outs = []
        for items in itertools.product(*per_axis):
            indices = tuple(i for i, _ in items)
            weights = [w for _, w in items]
            w = functools.reduce(lambda a, b: (a * b).astype(np.float32), weights)
            outs.append((w * inp[indices]).astype(np.float32))
        res = functools.reduce(lambda a, b: (a + b).astype(np.float32), outs)
        return _wrap(res.astype(inp.dtype))
    ndimage.map_coordinates = map_coordinates
    scipy.ndimage = ndimage
    jax.scipy = scipy

    image = types.ModuleType("jax.image")

    def resize(x, shape, method, **k):
        # method="nearest" as JAX's image resize evaluates it: along every axis whose size
        # changes from m to n, output index o reads input floor((o + 0.5) * m / n), computed
        # in float32.  (The linear method is used only when the fluid grid differs from the
        # domain grid, which the fixtures do not do.)
        if method == "linear":
            return _wrap(_resize_linear(np.asarray(x), shape))
        if method != "nearest":
            raise NotImplementedError("jax.image.resize(method=%r) is not restated" % method)
        x = np.asarray(x)
        for d, (m, n) in enumerate(zip(x.shape, shape)):
            if m == n:
                continue
            o = ((np.arange(n, dtype=np.float32) + np.float32(0.5)) * np.float32(m)) / np.float32(n)
            idx = np.floor(o).astype(np.int32)
            x = np.take(x, idx, axis=d)
        return _wrap(x)
    image.resize = resize
    jax.image = image

    # jax.random: NOT JAX's threefry stream.  Keys are uint32 pairs; draws come from a
    # numpy Generator seeded by the key.  The gym fixtures use keys only where the drawn
    # value is multiplied by zero (energy_walk_std = 0) or not at all.
    rnd = types.ModuleType("jax.random")

    def PRNGKey(seed):
        return np.array([0, int(seed) & 0xffffffff], np.uint32)

    def _gen(key):
        return np.random.default_rng([int(v) for v in np.asarray(key, np.uint32).ravel()])

    def split(key, num=2):
        return _gen(key).integers(0, 2 ** 32, size=(num, 2), dtype=np.uint64).astype(np.uint32)

    def normal(key, shape=(), dtype=None):
        return _wrap(_gen(key).standard_normal(shape).astype(np.float32))

    def uniform(key, shape=(), dtype=None, minval=0.0, maxval=1.0):
        u = _gen(key).random(shape).astype(np.float32)
        return _wrap((np.asarray(minval, np.float32) + u * (np.asarray(maxval, np.float32)
                                                            - np.asarray(minval, np.float32))).astype(np.float32))
    rnd.PRNGKey, rnd.key, rnd.split, rnd.normal, rnd.uniform = PRNGKey, PRNGKey, split, normal, uniform
    jax.random = rnd

    jax.config = types.SimpleNamespace(update=lambda *a, **k: None)
    return jax


def _linear_weights(m, n):
    """JAX's linear resize weights, input m -> output n (antialiased: the triangle kernel
    is widened by 1/scale when downsampling), float32: (m, n)."""
    inv = np.float32(1.0 / (n / m))
    ks = np.maximum(inv, np.float32(1.0))
    sf = (np.arange(n, dtype=np.float32) + np.float32(0.5)) * inv - np.float32(0.5)
    x = np.abs(sf[None, :] - np.arange(m, dtype=np.float32)[:, None]) / ks
    w = np.maximum(np.float32(0.0), np.float32(1.0) - np.abs(x))
    tot = np.sum(w, axis=0, keepdims=True)
    w = np.where(np.abs(tot) > np.float32(1000.0 * np.finfo(np.float32).eps), w / np.where(tot != 0, tot, 1), 0)
    inside = (sf >= -0.5) & (sf <= m - 0.5)
    return np.where(inside[None, :], w, 0).astype(np.float32)


def _resize_linear(x, shape):
    """jax.image.resize(x, shape, "linear"): every axis whose size changes is contracted
    with its weight matrix (in axis order; JAX contracts them in one einsum)."""
    out = x.astype(np.float32)
    for d, (m, n) in enumerate(zip(x.shape, shape)):
        if m == n:
            continue
        w = _linear_weights(m, n)
        out = np.moveaxis(np.tensordot(np.moveaxis(out, d, -1), w, axes=([-1], [0])), -1, d).astype(np.float32)
    return out


def install():
    """Install the shim as `jax`, `jax.numpy`, ... in sys.modules (idempotent)."""
    if "jax" in sys.modules and getattr(sys.modules["jax"], "_is_numpy_shim", False):
        return sys.modules["jax"]
    jax = _make_jax()
    jax._is_numpy_shim = True
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jax.numpy
    sys.modules["jax.numpy.linalg"] = jax.numpy.linalg
    sys.modules["jax.numpy.fft"] = jax.numpy.fft
    sys.modules["jax.lax"] = jax.lax
    sys.modules["jax.tree_util"] = jax.tree_util
    sys.modules["jax.scipy"] = jax.scipy
    sys.modules["jax.scipy.ndimage"] = jax.scipy.ndimage
    sys.modules["jax.image"] = jax.image
    sys.modules["jax.random"] = jax.random
    return jax
