"""Test-only stand-in for the parts of ``jax`` that the reference's forward
solvers use, so that ``tests/golden/make_golden.py`` can execute the
reference's own source on the CPU (numpy float64/float32 arithmetic) and
write golden vectors. Automatic differentiation is not provided."""

from __future__ import annotations

from . import lax, nn, numpy, scipy, tree  # noqa: F401

Array = numpy.ndarray


class _Config:
    def update(self, *args, **kwargs):
        return None


config = _Config()


def checkpoint(fun, *args, **kwargs):
    return fun


def jit(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


def vmap(fun, in_axes=0, out_axes=0):
    def run(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = next(len(a) for a, ax in zip(args, axes) if ax is not None)
        outs = [fun(*(a if ax is None else a[i] for a, ax in zip(args, axes))) for i in range(n)]
        return lax._stack(outs)

    return run


def grad(*args, **kwargs):
    raise NotImplementedError("the golden-vector jax stand-in has no autodiff")


def value_and_grad(*args, **kwargs):
    raise NotImplementedError("the golden-vector jax stand-in has no autodiff")
