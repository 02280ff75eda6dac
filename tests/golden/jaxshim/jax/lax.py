"""Test-only stand-in for ``jax.lax.scan`` / ``jax.lax.map``: plain Python
loops over the leading axis, outputs stacked leaf by leaf."""

from __future__ import annotations

import numpy as _np

from . import numpy as _jnp
from . import tree as _tree


def _stack(ys):
    if not ys:
        return None
    first = ys[0]
    return _tree.map(lambda *leaves: _jnp.asarray(_np.stack([_np.asarray(v) for v in leaves])),
                     first, *ys[1:])


def scan(f, init, xs=None, length=None, reverse=False, unroll=1):
    leaves = _tree.leaves(xs) if xs is not None else []
    n = length if length is not None else (len(leaves[0]) if leaves else 0)
    carry = init
    ys = []
    order = range(n - 1, -1, -1) if reverse else range(n)
    for i in order:
        x = _tree.map(lambda a: a[i], xs) if xs is not None else None
        carry, y = f(carry, x)
        ys.append(y)
    if reverse:
        ys.reverse()
    return carry, _stack(ys)


def map(f, xs):  # noqa: A001 - mirrors jax.lax.map
    leaves = _tree.leaves(xs)
    n = len(leaves[0])
    return _stack([f(_tree.map(lambda a: a[i], xs)) for i in range(n)])
