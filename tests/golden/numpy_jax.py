"""A NumPy stand-in for the small part of ``jax`` that CFD-demo uses.

CFD-demo (the reference) imports ``jax``, ``jax.numpy`` and ``jax.lax``; JAX is
not installed in the container that generates the golden fixtures. The
reference's arithmetic is all array code, so evaluating it eagerly in NumPy
float64 runs the reference's own source unchanged (up to summation-order
round-off against XLA, about 1e-15 relative).

Mapping: ``jit`` -> identity, ``jax.numpy`` -> ``numpy``,
``lax.fori_loop`` / ``lax.cond`` -> Python control flow,
``lax.optimization_barrier`` -> identity, ``jax.tree.map`` -> map over the
fields of a NamedTuple, ``config.update`` -> no-op. ``vmap`` and ``grad`` are
not provided (nothing in the fixture generator calls them).

Used only by ``make_golden.py``; never imported by the product.
"""

from __future__ import annotations

import sys
import types

import numpy as np


def install() -> None:
    """Register ``jax``, ``jax.numpy`` and ``jax.lax`` stand-ins in sys.modules."""
    if "jax" in sys.modules and getattr(sys.modules["jax"], "__numpy_stand_in__", False):
        return

    jax = types.ModuleType("jax")
    jax.__numpy_stand_in__ = True

    class _Config:
        def update(self, *_args, **_kwargs):
            return None

    jax.config = _Config()
    jax.Array = np.ndarray

    def jit(function=None, **_kwargs):
        if function is None:
            return lambda f: f
        return function

    jax.jit = jit

    def tree_map(function, tree, *rest):
        if isinstance(tree, tuple) and hasattr(tree, "_fields"):
            return type(tree)(*(tree_map(function, *items) for items in zip(tree, *rest)))
        if isinstance(tree, (tuple, list)):
            return type(tree)(tree_map(function, *items) for items in zip(tree, *rest))
        if isinstance(tree, dict):
            return {key: tree_map(function, tree[key], *(r[key] for r in rest)) for key in tree}
        return function(tree, *rest)

    jax.tree = types.SimpleNamespace(map=tree_map)

    lax = types.ModuleType("jax.lax")

    def fori_loop(lower, upper, body, init):
        value = init
        for index in range(int(lower), int(upper)):
            value = body(index, value)
        return value

    def cond(predicate, true_fn, false_fn, *operands):
        return true_fn(*operands) if bool(predicate) else false_fn(*operands)

    lax.fori_loop = fori_loop
    lax.cond = cond
    lax.optimization_barrier = lambda value: value
    jax.lax = lax
    jax.numpy = np

    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = np
    sys.modules["jax.lax"] = lax
