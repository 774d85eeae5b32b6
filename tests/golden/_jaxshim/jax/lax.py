"""``jax.lax`` stand-in (eager Python loops).  Test infrastructure only."""
from __future__ import annotations

import numpy as _np

from .numpy import _j


def _stack_trees(items):
    first = items[0]
    if first is None:
        return None
    if isinstance(first, tuple) and hasattr(first, "_fields"):
        return type(first)(*[_stack_trees([it[i] for it in items]) for i in range(len(first))])
    if isinstance(first, (tuple, list)):
        return type(first)(_stack_trees([it[i] for it in items]) for i in range(len(first)))
    return _j(_np.stack([_np.asarray(it) for it in items]))


def scan(fn, init, xs=None, length=None, reverse=False):
    if length is None:
        length = len(xs)
    carry = init
    outputs = []
    order = range(length - 1, -1, -1) if reverse else range(length)
    for index in order:
        x = None if xs is None else xs[index]
        carry, out = fn(carry, x)
        outputs.append(out)
    if reverse:
        outputs = outputs[::-1]
    return carry, (_stack_trees(outputs) if outputs else None)


def fori_loop(lower, upper, body, init):
    value = init
    for index in range(int(lower), int(upper)):
        value = body(index, value)
    return value


def cond(pred, true_fn, false_fn, *operands):
    return true_fn(*operands) if bool(pred) else false_fn(*operands)


def associative_scan(fn, elems, axis=0, reverse=False):
    values = _np.asarray(elems)
    values = _np.moveaxis(values, axis, 0)
    if reverse:
        values = values[::-1]
    out = _np.empty_like(values)
    running = values[0]
    out[0] = running
    for index in range(1, values.shape[0]):
        running = _np.asarray(fn(running, values[index]))
        out[index] = running
    if reverse:
        out = out[::-1]
    return _j(_np.moveaxis(out, 0, axis))
