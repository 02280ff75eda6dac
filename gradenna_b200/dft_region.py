"""Region-limited running-DFT monitors for the 3D solver
(src/gradenna/dft_region.py:1-257): per-component static slabs, their
union, the design / port / NTFF-box helpers and the scatter back to full
grids. On B200 each slab becomes one GdnDftMonitor of the C ABI, so only the
slab cells are folded into accumulators.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np
import torch


class FieldSlab(NamedTuple):
    """A static half-open index box [lo, hi) in one component's coordinates."""

    lo: tuple
    hi: tuple

    @property
    def shape(self):
        return tuple(h - l for l, h in zip(self.lo, self.hi))

    def slices(self):
        return tuple(slice(l, h) for l, h in zip(self.lo, self.hi))


class DFTRegions(NamedTuple):
    """One optional FieldSlab per component (None: not accumulated)."""

    ex: FieldSlab | None
    ey: FieldSlab | None
    ez: FieldSlab | None
    hx: FieldSlab | None
    hy: FieldSlab | None
    hz: FieldSlab | None


class RegionDFTMonitor(NamedTuple):
    """Slab spectra returned by simulate_3d with dft_regions (dft_region.py:74-92)."""

    freqs: torch.Tensor
    regions: DFTRegions
    ex: torch.Tensor | None
    ey: torch.Tensor | None
    ez: torch.Tensor | None
    hx: torch.Tensor | None
    hy: torch.Tensor | None
    hz: torch.Tensor | None


def full_field_shapes(nx: int, ny: int, nz: int):
    """The six component shapes (dft_region.py:95-104)."""
    return ((nx - 1, ny, nz), (nx, ny - 1, nz), (nx, ny, nz - 1),
            (nx, ny - 1, nz - 1), (nx - 1, ny, nz - 1), (nx - 1, ny - 1, nz))


def union_slab(a, b):
    """Smallest slab covering both (dft_region.py:107-120)."""
    if a is None:
        return b
    if b is None:
        return a
    return FieldSlab(tuple(min(x, y) for x, y in zip(a.lo, b.lo)),
                     tuple(max(x, y) for x, y in zip(a.hi, b.hi)))


def union_regions(a: DFTRegions, b: DFTRegions) -> DFTRegions:
    return DFTRegions(*(union_slab(x, y) for x, y in zip(a, b)))


def _norm(s: slice, n: int):
    if s.step not in (None, 1):
        raise ValueError(f"design/monitor region slices must have step 1, got {s}")
    a, b, _ = s.indices(n)
    return int(a), int(b)


def design_region_to_slabs(design_region, full_shapes) -> DFTRegions:
    """Cell slice applied unchanged to Ex/Ey/Ez, clamped to each shape (dft_region.py:139-165)."""
    if len(design_region) != 3:
        raise ValueError("design_region must be a 3-tuple of slices")

    def slab(shape):
        bounds = [_norm(design_region[d], shape[d]) for d in range(3)]
        return FieldSlab(tuple(b[0] for b in bounds), tuple(b[1] for b in bounds))

    return DFTRegions(slab(full_shapes[0]), slab(full_shapes[1]), slab(full_shapes[2]),
                      None, None, None)


def field_regions(monitor_region, full_shapes) -> DFTRegions:
    return design_region_to_slabs(monitor_region, full_shapes)


def port_regions(port_ijk, full_shapes) -> DFTRegions:
    """Slabs covering what the 3D port rebuild reads (dft_region.py:168-184)."""
    i, j, k = (int(v) for v in np.asarray(port_ijk).reshape(3))
    return DFTRegions(None, None, FieldSlab((i, j, k), (i + 1, j + 1, k + 1)),
                      FieldSlab((i, j - 1, k), (i + 1, j + 1, k + 1)),
                      FieldSlab((i - 1, j, k), (i + 1, j + 1, k + 1)), None)


def ntff_box_regions(grid, box_margin, full_shapes) -> DFTRegions:
    """Bounding slabs of everything ntff_3d reads (dft_region.py:187-227)."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    m = int(box_margin)
    i0, i1, j0, j1, k0, k1 = m, nx - 1 - m, m, ny - 1 - m, m, nz - 1 - m

    def clamp(lo, hi, shape):
        return FieldSlab(tuple(max(0, lo[d]) for d in range(3)),
                         tuple(min(shape[d], hi[d]) for d in range(3)))

    return DFTRegions(
        clamp((i0, j0, k0), (i1, j1 + 1, k1 + 1), full_shapes[0]),
        clamp((i0, j0, k0), (i1 + 1, j1, k1 + 1), full_shapes[1]),
        clamp((i0, j0, k0), (i1 + 1, j1 + 1, k1), full_shapes[2]),
        clamp((i0, j0 - 1, k0 - 1), (i1 + 1, j1 + 1, k1 + 1), full_shapes[3]),
        clamp((i0 - 1, j0, k0 - 1), (i1 + 1, j1 + 1, k1 + 1), full_shapes[4]),
        clamp((i0 - 1, j0 - 1, k0), (i1 + 1, j1 + 1, k1 + 1), full_shapes[5]),
    )


def scatter_full(mon: RegionDFTMonitor, full_shapes):
    """Zero-fill each slab spectrum onto its full component (dft_region.py:230-257)."""
    from gradenna_b200.fdtd3d import DFTMonitor

    n_freq = mon.freqs.shape[0]
    comps = (mon.ex, mon.ey, mon.ez, mon.hx, mon.hy, mon.hz)
    dev = next((c.device for c in comps if c is not None), None)
    dt = next((c.dtype for c in comps if c is not None), torch.complex128)
    out = []
    for slab, arr, shape in zip(mon.regions, comps, full_shapes):
        full = torch.zeros((n_freq,) + tuple(shape), dtype=dt, device=dev)
        if slab is not None and arr is not None:
            full[(slice(None),) + slab.slices()] = arr
        out.append(full)
    return DFTMonitor(mon.freqs, *out)


# ---------------------------------------------------------------------------
# Exact monitor boxes (several per component) for the 3D GdnDftMonitor list.
# The reference's DFTRegions allow one bounding slab per component, which for
# the NTFF box is the whole box volume; recording only the face layers that
# ntff_3d reads gives the same phasors for a fraction of the DFT traffic.
# A box is (comp, lo (3), hi (3)), half-open, in the component's indices.
# ---------------------------------------------------------------------------


def region_boxes(regions: DFTRegions):
    """DFTRegions slabs as a box list."""
    return [(c, tuple(s.lo), tuple(s.hi)) for c, s in enumerate(regions) if s is not None]


def ntff_face_boxes(grid, box_margin):
    """Every sample ntff_3d reads (src/gradenna/ntff.py:345-395): per face the
    tangential E layer and the two tangential H layers around it."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    m = int(box_margin)
    i0, i1, j0, j1, k0, k1 = m, nx - 1 - m, m, ny - 1 - m, m, nz - 1 - m
    out = []
    for i in (i1, i0):
        out += [(1, (i, j0, k0), (i + 1, j1, k1 + 1)), (2, (i, j0, k0), (i + 1, j1 + 1, k1)),
                (4, (i - 1, j0, k0), (i + 1, j1 + 1, k1)), (5, (i - 1, j0, k0), (i + 1, j1, k1 + 1))]
    for j in (j1, j0):
        out += [(0, (i0, j, k0), (i1, j + 1, k1 + 1)), (2, (i0, j, k0), (i1 + 1, j + 1, k1)),
                (3, (i0, j - 1, k0), (i1 + 1, j + 1, k1)), (5, (i0, j - 1, k0), (i1, j + 1, k1 + 1))]
    for k in (k1, k0):
        out += [(0, (i0, j0, k), (i1, j1 + 1, k + 1)), (1, (i0, j0, k), (i1 + 1, j1, k + 1)),
                (3, (i0, j0, k - 1), (i1 + 1, j1, k + 1)), (4, (i0, j0, k - 1), (i1, j1 + 1, k + 1))]
    return out


def boxes_to_full(freqs, boxes, tensors, full_shapes):
    """Zero-filled full-grid DFTMonitor from per-box spectra (n_freq, *box)."""
    from gradenna_b200.fdtd3d import DFTMonitor

    n_freq = freqs.shape[0]
    dev = tensors[0].device if tensors else None
    dt = tensors[0].dtype if tensors else torch.complex128
    full = [torch.zeros((n_freq,) + tuple(s), dtype=dt, device=dev) for s in full_shapes]
    for (c, lo, hi), t in zip(boxes, tensors):
        full[c][(slice(None),) + tuple(slice(a, b) for a, b in zip(lo, hi))] = t
    return DFTMonitor(freqs, *full)
