"""NumPy-backed stand-in for the small part of the ``jax`` API that the
ZhenMode solver sources use.

Test infrastructure only: ``tests/golden/make_golden.py`` puts the parent
folder on ``sys.path`` so that the reference solver, imported unmodified from
its source tree, runs eagerly in float64 NumPy in a container without JAX.
Nothing in the product imports it.

Semantics follow JAX with ``jax_enable_x64`` on: immutable arrays updated
through ``x.at[idx].set/add/multiply`` (returning copies), ``jit`` is the
identity, ``lax.scan`` is a Python loop that stacks per-iteration outputs.
"""
from __future__ import annotations

import types

import numpy as _np

from . import numpy  # noqa: F401  (jax.numpy)
from . import lax  # noqa: F401
from . import scipy  # noqa: F401
from .numpy import JArray as Array  # noqa: F401

__version__ = "0.0-numpy-shim"


def jit(fn=None, **_kwargs):
    if fn is None:
        return lambda f: f
    return fn


def grad(_fn, *args, **kwargs):  # pragma: no cover - not on the shimmed paths
    raise NotImplementedError("jax.grad is not available in the NumPy shim")


def devices(*_args):
    return ["cpu"]


def default_backend():
    return "cpu"


class _Config:
    def update(self, *_args, **_kwargs):
        return None


config = _Config()


def _tree_map(fn, tree, *rest):
    if tree is None:
        return None
    if isinstance(tree, tuple) and hasattr(tree, "_fields"):
        return type(tree)(*[_tree_map(fn, t, *[r[i] for r in rest]) for i, t in enumerate(tree)])
    if isinstance(tree, (tuple, list)):
        out = [_tree_map(fn, t, *[r[i] for r in rest]) for i, t in enumerate(tree)]
        return type(tree)(out)
    if isinstance(tree, dict):
        return {k: _tree_map(fn, v, *[r[k] for r in rest]) for k, v in tree.items()}
    return fn(tree, *rest)


tree = types.SimpleNamespace(map=_tree_map)
tree_util = types.SimpleNamespace(tree_map=_tree_map)
