"""Every module of the package, the benchmark and the oracle imports on a
machine without a GPU (no CUDA work happens at import time)."""

import importlib
import pkgutil

import pytest

import gradenna_b200

MODULES = sorted(m.name for m in pkgutil.iter_modules(gradenna_b200.__path__, "gradenna_b200.")
                 if not m.name.split(".")[-1].startswith("lib"))  # the CUDA library itself


@pytest.mark.parametrize("name", MODULES + ["bench", "oracle.unet_torch", "oracle.fdtd2d_ad"])
def test_module_imports(name):
    importlib.import_module(name)
