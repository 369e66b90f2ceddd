"""A NumPy-backed stand-in for the parts of ``jax`` that JAXIGA's setup and
basis-evaluation code touches, so that the reference's own functions can run
in a container where jax/jaxlib (pinned 0.11.1 by the reference) are absent.

This is test infrastructure for generating golden fixtures only:

* ``jax.numpy`` is NumPy, with ``ndarray.at[...].set/add`` provided by an
  ndarray subclass (``add`` is ``np.add.at``, i.e. sequential accumulation).
* ``jax.vmap`` is a Python loop followed by ``np.stack``.
* ``jax.pure_callback`` calls the host function directly.
* Transformations that need automatic differentiation (``grad``, ``jvp``,
  ``hessian``, ``jacfwd``) raise; the fixture script never reaches them.
"""

from __future__ import annotations

import sys
import types

import numpy as np


class _AtIndexer:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def set(self, values):
        out = np.array(self.arr, copy=True).view(JArray)
        out[self.idx] = values
        return out

    def add(self, values):
        out = np.array(self.arr, copy=True).view(JArray)
        np.add.at(out, self.idx, values)
        return out

    def get(self):
        return np.asarray(self.arr)[self.idx]


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIndexer(self.arr, idx)


class JArray(np.ndarray):
    """ndarray with the functional ``.at[]`` update syntax."""

    @property
    def at(self):
        return _At(self)


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, JArray):
        return x.view(JArray)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


class _NumpyProxy(types.ModuleType):
    def __init__(self, name, base):
        super().__init__(name)
        self._base = base

    def __getattr__(self, name):
        attr = getattr(self._base, name)
        if callable(attr) and not isinstance(attr, type):
            def fn(*a, **k):
                return _wrap(attr(*a, **k))
            return fn
        return attr


def _tree_map(f, tree, *rest, is_leaf=None):
    if is_leaf is not None and is_leaf(tree):
        return f(tree, *rest)
    if isinstance(tree, dict):
        return {k: _tree_map(f, tree[k], *[r[k] for r in rest], is_leaf=is_leaf) for k in tree}
    if isinstance(tree, (list, tuple)):
        out = [_tree_map(f, t, *[r[i] for r in rest], is_leaf=is_leaf) for i, t in enumerate(tree)]
        return type(tree)(out)
    if tree is None:
        return None
    return f(tree, *rest)


def _tree_leaves(tree, is_leaf=None):
    out = []

    def visit(t):
        if is_leaf is not None and is_leaf(t):
            out.append(t)
        elif isinstance(t, dict):
            for k in t:
                visit(t[k])
        elif isinstance(t, (list, tuple)):
            for v in t:
                visit(v)
        elif t is not None:
            out.append(t)

    visit(tree)
    return out


def _slice(arg, ax, i):
    if ax is None:
        return arg
    if isinstance(ax, dict):
        return {k: _slice(arg[k], ax[k], i) for k in arg}
    if isinstance(ax, (list, tuple)):
        return type(arg)(_slice(a, x, i) for a, x in zip(arg, ax))
    v = np.take(np.asarray(arg), i, axis=ax)
    return v.view(JArray) if isinstance(v, np.ndarray) and v.ndim else v


def _size(arg, ax):
    if ax is None:
        return None
    if isinstance(ax, dict):
        for k in ax:
            n = _size(arg[k], ax[k])
            if n is not None:
                return n
        return None
    if isinstance(ax, (list, tuple)):
        for a, x in zip(arg, ax):
            n = _size(a, x)
            if n is not None:
                return n
        return None
    return np.shape(arg)[ax]


def _stack(outs, ax):
    first = outs[0]
    if first is None:
        return None
    if isinstance(first, tuple):
        axes = ax if isinstance(ax, (tuple, list)) else (ax,) * len(first)
        return tuple(_stack([o[j] for o in outs], axes[j]) for j in range(len(first)))
    return np.stack([np.asarray(o) for o in outs], axis=ax).view(JArray)


def vmap(f, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            n = _size(a, ax)
            if n is not None:
                break
        outs = [f(*[_slice(a, ax, i) for a, ax in zip(args, axes)]) for i in range(n)]
        return _stack(outs, out_axes)

    return mapped


def _no_ad(*a, **k):
    raise NotImplementedError("automatic differentiation is not available in the jax stub")


class _CustomVJP:
    def __init__(self, fun, nondiff_argnums=()):
        self.fun = fun

    def defvjp(self, fwd, bwd):
        return None

    def __call__(self, *a, **k):
        return self.fun(*a, **k)


def custom_vjp(fun=None, nondiff_argnums=()):
    if fun is None:
        return lambda f: _CustomVJP(f, nondiff_argnums)
    return _CustomVJP(fun, nondiff_argnums)


class _Tracer:  # never instantiated; only used in isinstance checks
    pass


def install():
    """Register the stub as ``jax`` (and submodules) in ``sys.modules``."""
    jax = types.ModuleType("jax")
    jnp = _NumpyProxy("jax.numpy", np)
    jnp.linalg = _NumpyProxy("jax.numpy.linalg", np.linalg)
    jnp.ndarray = np.ndarray
    jax.numpy = jnp

    tree_util = types.ModuleType("jax.tree_util")
    tree_util.register_dataclass = lambda cls: cls
    tree_util.register_pytree_node_class = lambda cls: cls
    tree_util.tree_map = _tree_map
    tree_util.tree_leaves = _tree_leaves
    jax.tree_util = tree_util

    core = types.ModuleType("jax.core")
    core.Tracer = _Tracer
    jax.core = core

    config = types.SimpleNamespace(update=lambda *a, **k: None, values={})
    jax.config = config

    jax.vmap = vmap
    jax.grad = jax.jvp = jax.hessian = jax.jacfwd = jax.jacrev = _no_ad
    jax.checkpoint = lambda f, *a, **k: f
    jax.custom_vjp = custom_vjp
    jax.pure_callback = lambda host, shape, *args, **k: host(*args)
    jax.ShapeDtypeStruct = lambda *a, **k: None
    jax.default_backend = lambda: "cpu"
    jax.jit = lambda f, *a, **k: f

    lax = types.ModuleType("jax.lax")
    lax.custom_linear_solve = _no_ad
    lax.while_loop = _no_ad
    jax.lax = lax

    experimental = types.ModuleType("jax.experimental")
    sparse = types.ModuleType("jax.experimental.sparse")
    sparse.BCOO = None
    experimental.sparse = sparse
    jax.experimental = experimental

    scipy_mod = types.ModuleType("jax.scipy")
    scipy_sparse = types.ModuleType("jax.scipy.sparse")
    scipy_linalg = types.ModuleType("jax.scipy.sparse.linalg")
    scipy_linalg.cg = scipy_linalg.bicgstab = scipy_linalg.gmres = _no_ad
    scipy_sparse.linalg = scipy_linalg
    scipy_mod.sparse = scipy_sparse
    jax.scipy = scipy_mod

    mods = {
        "jax": jax,
        "jax.numpy": jnp,
        "jax.numpy.linalg": jnp.linalg,
        "jax.tree_util": tree_util,
        "jax.core": core,
        "jax.lax": lax,
        "jax.experimental": experimental,
        "jax.experimental.sparse": sparse,
        "jax.scipy": scipy_mod,
        "jax.scipy.sparse": scipy_sparse,
        "jax.scipy.sparse.linalg": scipy_linalg,
    }
    sys.modules.update(mods)
    return jax


def load_reference(src_dir):
    """Import ``jaxiga`` submodules from ``src_dir`` without its ``__init__``.

    The package ``__init__`` pulls in optional subsystems (gmsh, optax,
    plotting); the fixture script only needs the setup and evaluation modules,
    whose subpackage ``__init__`` files are empty.
    """
    install()
    pkg = types.ModuleType("jaxiga")
    pkg.__path__ = [f"{src_dir}/jaxiga"]
    sys.modules["jaxiga"] = pkg
    import importlib

    names = [
        "jaxiga.config",
        "jaxiga.space.bernstein",
        "jaxiga.geometry.nurbs",
        "jaxiga.geometry.primitives",
        "jaxiga.space.function_space",
        "jaxiga.space.pointset",
        "jaxiga.space.evaluation",
        "jaxiga.forms.problem",
        "jaxiga.forms.materials",
        "jaxiga.forms.library",
        "jaxiga.solvers.linear",
        "jaxiga.methods._common",
        "jaxiga.methods.galerkin",
    ]
    return {n.split(".")[-1]: importlib.import_module(n) for n in names}
