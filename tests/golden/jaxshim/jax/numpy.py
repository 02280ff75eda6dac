"""Test-only stand-in for ``jax.numpy``: numpy arrays that also carry JAX's
functional ``.at[idx].add/.set/...`` update syntax (each returns a copy).

This exists only so that ``tests/golden/make_golden.py`` can run the
reference's own, unmodified ``simulate_tm`` / ``simulate_3d`` source on the
CPU to write golden vectors. It is not part of the library, and nothing under
``gradenna_b200/`` can import it.

Semantics kept from JAX:
  * ``.at[idx].add(v)`` is a scatter-add (repeated indices accumulate, as
    ``np.add.at``); ``.set`` assigns; the update is cast to the array dtype.
  * Type promotion follows numpy 2 (NEP 50), which matches JAX with x64
    enabled for the cases the reference uses: Python scalars are weak,
    numpy scalars and arrays are strong.
"""

from __future__ import annotations

import numpy as _np


class ndarray(_np.ndarray):
    """numpy array with JAX's ``.at`` property."""

    @property
    def at(self):
        return _At(self)

    def __array_finalize__(self, obj):  # noqa: D401 - numpy hook
        pass


Array = ndarray


def _wrap(x):
    if isinstance(x, _np.ndarray) and not isinstance(x, ndarray):
        return x.view(ndarray)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self._arr, idx)


class _AtIdx:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def _copy(self):
        return _np.array(self._arr, copy=True).view(ndarray)

    def set(self, v):
        out = self._copy()
        out[self._idx] = _np.asarray(v).astype(out.dtype, copy=False)
        return out

    def add(self, v):
        out = self._copy()
        _np.add.at(out, self._idx, _np.asarray(v).astype(out.dtype, copy=False))
        return out

    def multiply(self, v):
        out = self._copy()
        _np.multiply.at(out, self._idx, _np.asarray(v).astype(out.dtype, copy=False))
        return out

    def get(self):
        return _wrap(self._arr[self._idx])


def asarray(a, dtype=None):
    return _wrap(_np.asarray(a, dtype=dtype))


def array(a, dtype=None, copy=True):
    return _wrap(_np.array(a, dtype=dtype, copy=copy))


def __getattr__(name):
    obj = getattr(_np, name)
    if callable(obj) and not isinstance(obj, type):
        def fn(*args, **kwargs):
            return _wrap(obj(*args, **kwargs))

        fn.__name__ = name
        return fn
    return obj
