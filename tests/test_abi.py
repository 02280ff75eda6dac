"""CPU checks of the C-ABI library: it loads, exports every declared symbol,
its struct layouts match the ctypes mirrors, and bad arguments come back as
status codes (no device work is launched by these tests)."""

import ctypes
import os
import re
import shutil
import subprocess

import pytest

from tests.conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]


def _declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(gdn_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    syms = _declared_symbols()
    assert "gdn_tm_run_f32" in syms and "gdn_tm_run_f64" in syms
    assert "gdn_version" in syms and "gdn_last_error" in syms


def test_library_exports_every_declared_symbol():
    from gradenna_b200 import _native

    lib = _native.load()
    missing = [s for s in _declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"symbols declared in include/*.h but not exported: {missing}"
    assert lib.gdn_version().startswith(b"gradenna_b200")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs a host C++ compiler")
def test_struct_layouts_match_ctypes(tmp_path):
    from gradenna_b200 import _native

    src = tmp_path / "sz.cpp"
    src.write_text(
        '#include "gradenna_b200.h"\n#include <cstdio>\n'
        "int main(){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(GdnTmParams),"
        " sizeof(GdnTmBuffers), sizeof(GdnTmPoints), sizeof(GdnYeeParams), sizeof(GdnYeePoints),"
        " sizeof(GdnYeeBuffers), sizeof(GdnDftMonitor), sizeof(GdnTmObjective));}\n")
    exe = tmp_path / "sz"
    subprocess.run(["g++", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                            check=True).stdout.split()]
    from gradenna_b200 import fdtd3d, objectives

    assert sizes == [ctypes.sizeof(_native.TmParams), ctypes.sizeof(_native.TmBuffers),
                     ctypes.sizeof(_native.TmPoints), ctypes.sizeof(fdtd3d.YeeParams),
                     ctypes.sizeof(fdtd3d.YeePoints), ctypes.sizeof(fdtd3d.YeeBuffers),
                     ctypes.sizeof(_native.DftMonitor), ctypes.sizeof(objectives.TmObjective)]


def test_bad_arguments_return_status_not_abort():
    from gradenna_b200 import _native

    lib = _native.load()
    p = _native.TmParams()
    p.nx, p.ny, p.npml = 2, 2, 0
    nbytes = ctypes.c_size_t(0)
    assert lib.gdn_tm_workspace_size(ctypes.byref(p), None, 0, ctypes.byref(nbytes)) == 1
    assert b"grid" in lib.gdn_last_error()
    # A grid too small for its CPML is rejected before any device work.
    p.nx, p.ny, p.npml, p.n_steps = 20, 20, 10, 5
    p.dt = p.dx = p.dy = p.dz = 1.0
    pts = _native.TmPoints()
    bufs = _native.TmBuffers()
    st = lib.gdn_tm_run_f32(ctypes.byref(p), ctypes.byref(pts), ctypes.byref(bufs), None)
    assert st == 1
    assert b"too small" in lib.gdn_last_error()
    # Out-of-range port index.
    p.npml = 2
    p.n_ports = 1
    pi = (ctypes.c_int32 * 1)(0)
    pj = (ctypes.c_int32 * 1)(5)
    pts.port_i, pts.port_j = pi, pj
    st = lib.gdn_tm_run_f32(ctypes.byref(p), ctypes.byref(pts), ctypes.byref(bufs), None)
    assert st == 1
    assert b"port" in lib.gdn_last_error()
