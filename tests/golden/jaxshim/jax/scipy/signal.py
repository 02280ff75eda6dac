"""Test-only stand-in for ``jax.scipy.signal.fftconvolve`` (scipy's FFT
convolution, the algorithm JAX's version implements)."""

import numpy as _np
import scipy.signal as _sig

from .. import numpy as _jnp


def fftconvolve(a, b, mode="full", axes=None):
    return _jnp.asarray(_sig.fftconvolve(_np.asarray(a), _np.asarray(b), mode=mode, axes=axes))
