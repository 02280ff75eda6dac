"""Load the reference's own modules (``src/gradenna/*.py``, unmodified) on the
CPU through the numpy stand-in for ``jax`` in ``tests/golden/jaxshim``.

Used only by ``tests/golden/make_golden.py`` in a checkout that has the
reference source next to it; the golden vectors it writes are committed, so
neither the tests nor the library read the reference at run time. The
package ``__init__`` of the reference is not executed (it imports optional
modules); each submodule is imported on its own from the reference tree.
"""

from __future__ import annotations

import importlib
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "jaxshim")
DEFAULT_REF = "/root/reference"


def reference_root() -> str:
    return os.environ.get("GRADENNA_REFERENCE", DEFAULT_REF)


def load(*names: str):
    """Import ``gradenna.<name>`` for each name from the reference tree."""
    src = os.path.join(reference_root(), "src", "gradenna")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference source not found at {src}")
    if SHIM not in sys.path:
        sys.path.insert(0, SHIM)
    import jax  # noqa: F401  (must resolve to the stand-in)

    if not getattr(jax, "__file__", "").startswith(SHIM):
        raise RuntimeError(f"'jax' resolves to {jax.__file__}, not the stand-in")
    pkg = sys.modules.get("gradenna")
    if pkg is None:
        pkg = types.ModuleType("gradenna")
        pkg.__path__ = [src]
        sys.modules["gradenna"] = pkg
    mods = [importlib.import_module(f"gradenna.{n}") for n in names]
    return mods[0] if len(mods) == 1 else mods
