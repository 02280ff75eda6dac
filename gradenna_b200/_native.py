"""ctypes binding of the in-tree CUDA library (include/gradenna_b200.h).

This replaces the reference's loader of the Rust cdylib
(src/gradenna/native.py:58-170): the library is loaded once under a lock and
every entry point returns a status code that is turned into an exception
here. There is no fallback: if the library cannot be loaded, or no CUDA
device is present, the call raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgradenna_b200.so")

_LOCK = threading.Lock()
_LIB = None

c_int32 = ctypes.c_int32
c_void_p = ctypes.c_void_p
c_double = ctypes.c_double
P_i32 = ctypes.POINTER(ctypes.c_int32)
P_f64 = ctypes.POINTER(ctypes.c_double)


class GdnError(RuntimeError):
    """A non-zero status returned by the CUDA library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"gradenna_b200 status {status}: {message}")
        self.status = status


class TmParams(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("npml", c_int32), ("n_steps", c_int32),
        ("n_sources", c_int32), ("n_ports", c_int32), ("n_mx", c_int32), ("n_my", c_int32),
        ("n_probes", c_int32), ("n_freq", c_int32), ("record_energy", c_int32),
        ("dft_f64", c_int32), ("cw_sources", c_int32), ("n_monitors", c_int32),
        ("dt", c_double), ("dx", c_double), ("dy", c_double), ("dz", c_double),
        ("mu0", c_double),
    ]


class DftMonitor(ctypes.Structure):
    _fields_ = [("comp", c_int32), ("lo", c_int32 * 3), ("hi", c_int32 * 3), ("out", c_void_p)]


class TmPoints(ctypes.Structure):
    _fields_ = [
        ("src_i", P_i32), ("src_j", P_i32),
        ("port_i", P_i32), ("port_j", P_i32),
        ("mx_i", P_i32), ("mx_j", P_i32),
        ("my_i", P_i32), ("my_j", P_i32),
        ("probe_i", P_i32), ("probe_j", P_i32),
        ("monitors", ctypes.POINTER(DftMonitor)),
    ]


_TM_BUF_PTRS_A = [
    "ca", "cb", "eps", "inv_kx_e", "inv_ky_e", "inv_kx_h", "inv_ky_h",
    "b_ezx_lo", "c_ezx_lo", "b_ezx_hi", "c_ezx_hi",
    "b_ezy_lo", "c_ezy_lo", "b_ezy_hi", "c_ezy_hi",
    "b_hyx_lo", "c_hyx_lo", "b_hyx_hi", "c_hyx_hi",
    "b_hxy_lo", "c_hxy_lo", "b_hxy_hi", "c_hxy_hi",
]
_TM_BUF_PTRS_B = [
    "cb_src", "src_cur", "cb_vs", "port_vs", "mx_cur", "my_cur",
    "cw_env", "src_w", "mx_w", "my_w", "ph_e", "ph_h",
    "ez", "hx", "hy", "out_probe", "out_v", "out_i", "out_energy",
    "dft_ez", "dft_hx", "dft_hy", "workspace",
]


class TmBuffers(ctypes.Structure):
    _fields_ = (
        [(n, c_void_p) for n in _TM_BUF_PTRS_A]
        + [("dt_mu", c_double), ("inv_dx", c_double), ("inv_dy", c_double)]
        + [(n, c_void_p) for n in _TM_BUF_PTRS_B]
        + [("workspace_bytes", ctypes.c_size_t)]
    )


def _configure(lib) -> None:
    lib.gdn_version.restype = ctypes.c_char_p
    lib.gdn_version.argtypes = []
    lib.gdn_last_error.restype = ctypes.c_char_p
    lib.gdn_last_error.argtypes = []
    lib.gdn_kernel_launches.restype = ctypes.c_uint64
    lib.gdn_kernel_launches.argtypes = []
    lib.gdn_tm_loop_stats.restype = ctypes.c_int
    lib.gdn_tm_loop_stats.argtypes = [P_f64, P_f64, ctypes.POINTER(ctypes.c_int64), c_int32]
    lib.gdn_tm_workspace_size.restype = ctypes.c_int
    lib.gdn_tm_workspace_size.argtypes = [
        ctypes.POINTER(TmParams), ctypes.POINTER(TmPoints), ctypes.c_int,
        ctypes.POINTER(ctypes.c_size_t)]
    for name in ("gdn_tm_run_f32", "gdn_tm_run_f64"):
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.POINTER(TmParams), ctypes.POINTER(TmPoints),
                       ctypes.POINTER(TmBuffers), c_void_p]
    _configure_extra(lib)


_EXTRA = []  # (name, restype, argtypes) registered by other modules


def register(name: str, restype, argtypes) -> None:
    """Declare an extra entry point's signature (applied at load time)."""
    _EXTRA.append((name, restype, argtypes))
    if _LIB:
        fn = getattr(_LIB, name)
        fn.restype = restype
        fn.argtypes = argtypes


def _configure_extra(lib) -> None:
    for name, restype, argtypes in _EXTRA:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes


def load():
    """Load the CUDA library (raising if it is missing or unloadable)."""
    global _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"gradenna_b200 CUDA library not built ({LIB_PATH} missing); "
                "run `python -m gradenna_b200.build`"
            )
        # torch first, so the library binds to the same CUDA runtime.
        import torch  # noqa: F401

        lib = ctypes.CDLL(LIB_PATH)
        _configure(lib)
        _LIB = lib
        return lib


def check(status: int) -> None:
    if status != 0:
        msg = load().gdn_last_error().decode(errors="replace")
        raise GdnError(status, msg)


def require_cuda(device=None):
    """Resolve the CUDA device to run on; raise if there is none."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("gradenna_b200 needs a CUDA device (no CPU fallback)")
    dev = torch.device("cuda") if device is None else torch.device(device)
    if dev.type != "cuda":
        raise ValueError(f"gradenna_b200 runs on CUDA devices only, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def ptr(t) -> int | None:
    """Device pointer of a tensor (None for None)."""
    return None if t is None else t.data_ptr()


def kernel_launches() -> int:
    """Kernels this library has launched in this process (gdn_kernel_launches)."""
    return int(load().gdn_kernel_launches())


def tm_loop_stats(reset: bool = True):
    """(ms, cell_steps, blocks) of the 2D time loops since the last reset
    (gdn_tm_loop_stats): device time between events recorded on the run's
    stream around each time loop."""
    ms, cs = ctypes.c_double(), ctypes.c_double()
    nb = ctypes.c_int64()
    check(load().gdn_tm_loop_stats(ctypes.byref(ms), ctypes.byref(cs), ctypes.byref(nb),
                                   int(reset)))
    return ms.value, cs.value, nb.value
