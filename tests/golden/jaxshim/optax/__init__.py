"""Test-only placeholder for ``optax`` so the reference's ``topopt`` module
imports; its optimiser is never called by the golden-vector script."""


def __getattr__(name):
    raise NotImplementedError(f"optax.{name} is not available in the golden-vector stand-in")
