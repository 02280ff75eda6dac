"""Test-only stand-in for ``jax.scipy``."""
from . import signal  # noqa: F401
