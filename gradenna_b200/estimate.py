"""Memory estimates: size a run against a GPU before launching it.

Two kinds of figures, in GiB:

* The reference's memory model of a reverse-mode-differentiated 3D run
  (src/gradenna/estimate.py:44-152), with the same function names and
  result keys, so code that sizes runs with it keeps working: six Yee
  fields, coefficient arrays, twelve CPML psi arrays (full grid or PML
  strips), running-DFT accumulators, and the naive and sqrt(N)-checkpointed
  reverse sweeps.
* This library's own footprint on B200 (keys starting with ``b200_``), from
  its layouts: the 2D runner's padded ping-pong planes (8 ghost rows and 32
  ghost columns a side, two slots of Ez/Hx/Hy and of the four psi planes,
  ca/cb), the 3D runner's full-volume fields, psi and coefficients, the DFT
  accumulators, the monitor ring, the adjoint's stored phasors, and the
  design-cell Ez histories of the time-domain adjoint. Gradients here need
  no reverse-mode tape: the frequency-domain adjoint keeps the forward
  design phasors during the adjoint run, the time-domain adjoint keeps two
  n_steps x design-cell histories.

All figures are first-order array sizes; leave headroom (``fits_gpu``
defaults to 85 % of the memory).
"""

from __future__ import annotations

import numpy as np

__all__ = ["fdtd3d_memory_estimate", "fdtd2d_memory_estimate", "fits_gpu", "gpu_fit_report",
           "COMMON_VRAM_GB", "B200_VRAM_GB"]

_GIB = float(1 << 30)

#: Consumer VRAM sizes [GB] of the reference's fit report.
COMMON_VRAM_GB = (24.0, 16.0, 8.0)
#: One B200 (nvidia-smi reports 183,359 MiB).
B200_VRAM_GB = 179.0


def _itemsize(dtype) -> int:
    return int(np.dtype(str(dtype).replace("torch.", "")).itemsize)


def fdtd3d_memory_estimate(grid, n_steps: int, *, checkpoint_segments: int | None = None,
                           n_dft_freqs: int = 0, dtype="float32", cpml_thickness: int = 10,
                           dft_dtype=None, design_cells: int = 0) -> dict:
    """Peak memory of a differentiated 3D run (reference keys, see the module
    docstring) plus this library's ``b200_forward_gb`` (one gdn_yee_run with
    full-grid DFT) and ``b200_gradient_gb`` (frequency-domain adjoint: the
    adjoint run while the forward design phasors of ``design_cells`` cells
    are kept). ``dft_dtype`` is the accumulator dtype of this library's runs
    (default: complex of the field dtype)."""
    if n_steps < 1:
        raise ValueError("n_steps must be >= 1")
    if n_dft_freqs < 0:
        raise ValueError("n_dft_freqs must be >= 0")
    k = int(round(np.sqrt(n_steps))) if checkpoint_segments is None else int(checkpoint_segments)
    if k < 1:
        raise ValueError("checkpoint_segments must be >= 1")
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    cells = nx * ny * nz
    b = _itemsize(dtype)
    # Yee components on their staggered lattices.
    comp = ((nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1)
            + nx * (ny - 1) * (nz - 1) + (nx - 1) * ny * (nz - 1) + (nx - 1) * (ny - 1) * nz)
    fields = comp * b
    materials = 4 * cells * b
    psi_full = 12 * cells * b
    t = min(cpml_thickness, nx // 2, ny // 2, nz // 2)
    # a psi array of axis a lives in the 2 t planes of that axis' slabs
    psi_strip = int(4 * cells * b * 2 * t * (1.0 / nx + 1.0 / ny + 1.0 / nz))
    dft = n_dft_freqs * comp * 2 * b
    state_full = fields + psi_full + dft
    state_strip = fields + psi_strip + dft
    per_seg = float(n_steps) / k
    out = {
        "n_cells": cells, "bytes_per_value": b, "n_steps": int(n_steps),
        "checkpoint_segments": k,
        "fields_gb": fields / _GIB, "materials_gb": materials / _GIB,
        "psi_full_gb": psi_full / _GIB, "psi_strip_gb": psi_strip / _GIB,
        "dft_monitor_gb": dft / _GIB,
        "state_full_gb": state_full / _GIB, "state_strip_gb": state_strip / _GIB,
        "forward_gb": (state_full + materials) / _GIB,
        # reverse sweeps: every step's carry, or K snapshots plus one replayed
        # segment of n_steps / K steps (estimate.py:144-149)
        "adjoint_naive_gb": state_full * n_steps / _GIB,
        "adjoint_checkpoint_gb": (k + per_seg) * state_full / _GIB,
        "adjoint_checkpoint_strip_gb": (k + per_seg) * state_strip / _GIB,
    }
    # This library: 6 fields + 12 psi full volumes, ca / cb / eps per node,
    # full-grid complex accumulators, a 32-slot ring of monitored cells.
    acc = _itemsize(dft_dtype) if dft_dtype is not None else 2 * b
    b200_fwd = (6 + 12 + 3) * cells * b + n_dft_freqs * comp * acc
    b200_fwd += (32 * comp * b) if n_dft_freqs else 0
    phasors = 3 * design_cells * max(n_dft_freqs, 1) * acc
    out["b200_forward_gb"] = b200_fwd / _GIB
    out["b200_gradient_gb"] = (b200_fwd + phasors) / _GIB
    return out


def fdtd2d_memory_estimate(grid, n_steps: int, *, n_dft_freqs: int = 0, dtype="float32",
                           dft_dtype=None, design_cells: int = 0, monitor_cells: int | None = None,
                           time_adjoint: bool = False) -> dict:
    """This library's 2D footprint: ``b200_forward_gb`` of one gdn_tm_run
    (padded ping-pong field and psi planes, ca / cb, DFT accumulators of
    ``monitor_cells`` cells (default: the full grid, three components) and
    their 32-slot ring), ``b200_freq_gradient_gb`` (plus the forward design
    phasors kept during the adjoint run) and, with ``time_adjoint``,
    ``b200_time_gradient_gb`` (plus the forward and adjoint Ez histories of
    the design cells, n_steps x design_cells each)."""
    if n_steps < 1:
        raise ValueError("n_steps must be >= 1")
    nx, ny = grid.nx, grid.ny
    b = _itemsize(dtype)
    acc = _itemsize(dft_dtype) if dft_dtype is not None else 2 * b
    plane = (nx + 16) * (ny + 64)
    # 2 slots x (Ez, Hx, Hy, 4 psi) + ca, cb
    planes = (2 * 7 + 2) * plane * b
    mon = (3 * nx * ny) if monitor_cells is None else int(monitor_cells)
    dft = n_dft_freqs * mon * acc
    ring = 32 * mon * b if n_dft_freqs else 0
    fwd = planes + dft + ring
    phasors = design_cells * max(n_dft_freqs, 1) * acc
    out = {
        "n_cells": nx * ny, "bytes_per_value": b, "n_steps": int(n_steps),
        "b200_planes_gb": planes / _GIB, "b200_dft_gb": dft / _GIB, "b200_ring_gb": ring / _GIB,
        "b200_forward_gb": fwd / _GIB,
        "b200_freq_gradient_gb": (fwd + phasors) / _GIB,
    }
    if time_adjoint:
        out["b200_history_gb"] = 2 * n_steps * design_cells * b / _GIB
        out["b200_time_gradient_gb"] = out["b200_forward_gb"] + out["b200_history_gb"]
    return out


def fits_gpu(required_gb: float, vram_gb: float, usable_fraction: float = 0.85) -> bool:
    """True when ``required_gb`` fits in ``usable_fraction`` of ``vram_gb``."""
    if not 0.0 < usable_fraction <= 1.0:
        raise ValueError("usable_fraction must be in (0, 1]")
    return required_gb <= usable_fraction * vram_gb


def gpu_fit_report(estimate: dict, *, key: str = "adjoint_checkpoint_gb",
                   vram_sizes_gb=COMMON_VRAM_GB, usable_fraction: float = 0.85) -> dict:
    """{vram_gb: fits} of ``estimate[key]`` against each memory size (pass
    ``vram_sizes_gb=(B200_VRAM_GB,)`` and a ``b200_*`` key for a B200)."""
    need = float(estimate[key])
    return {float(v): fits_gpu(need, float(v), usable_fraction) for v in vram_sizes_gb}
