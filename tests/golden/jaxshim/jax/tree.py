"""Test-only stand-in for ``jax.tree`` (pytrees of dict / tuple / list /
NamedTuple / None, leaves are everything else)."""

from __future__ import annotations


def _is_namedtuple(x):
    return isinstance(x, tuple) and hasattr(x, "_fields")


def map(f, tree, *rest):  # noqa: A001 - mirrors jax.tree.map
    if tree is None:
        return None
    if isinstance(tree, dict):
        return {k: map(f, tree[k], *(r[k] for r in rest)) for k in tree}
    if _is_namedtuple(tree):
        return type(tree)(*(map(f, v, *(r[i] for r in rest)) for i, v in enumerate(tree)))
    if isinstance(tree, (tuple, list)):
        out = [map(f, v, *(r[i] for r in rest)) for i, v in enumerate(tree)]
        return type(tree)(out)
    return f(tree, *rest)


def leaves(tree):
    out = []
    map(lambda x: out.append(x), tree)
    return out
