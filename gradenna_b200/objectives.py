"""Built-in 2D objectives with a fused device evaluation.

``RadiatedPowerS11`` is L = w_prad sum_k P_k + w_s11 sum_k |S11_k|^2: the
Poynting flux through a dual-grid contour (monitors.py:20-70) and the
Kurokawa S11 of one port rebuilt from the field phasors (freq_adjoint.py:
536-558, sparams.py:68-79). Called on FreqPhasors it is an ordinary torch
objective. Inside ``freq_adjoint_gradient`` its ``fused_tm`` method replaces
the generic objective path (phasors scattered onto full grids, torch
autograd, a scan for the nonzero cotangents) with one kernel launch,
``gdn_tm_objective_prad_s11``, that reads the forward run's monitor outputs
and writes the value and the adjoint run's CW source weights.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200.constants import EPS0, MU0
from gradenna_b200.fdtd2d import DZ
from gradenna_b200.monitors import port_monitors, poynting_box_monitors, poynting_flux_box_2d
from gradenna_b200.sparams import s11_power_wave

__all__ = ["RadiatedPowerS11"]


class TmObjective(ctypes.Structure):
    _fields_ = [("n_freq", ctypes.c_int32), ("box", ctypes.c_int32 * 4),
                ("port", ctypes.c_int32 * 2), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("n_monitors", ctypes.c_int32),
                ("monitors", ctypes.POINTER(_native.DftMonitor)),
                ("freqs", ctypes.POINTER(ctypes.c_double))] + [
        (n, ctypes.c_double) for n in ("dx", "dy", "dt", "dz", "resistance", "w_prad", "w_s11",
                                       "eps0", "mu0")] + [
        ("value", ctypes.c_void_p), ("p_rad", ctypes.c_void_p), ("s11", ctypes.c_void_p),
        ("w_ez", ctypes.c_void_p), ("w_hx", ctypes.c_void_p), ("w_hy", ctypes.c_void_p)]


_P = ctypes.POINTER
_native.register("gdn_tm_objective_cells", ctypes.c_int, [
    _P(TmObjective), _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_int32),
    _native.P_i32, _native.P_i32, _native.P_i32])
_native.register("gdn_tm_objective_prad_s11", ctypes.c_int, [_P(TmObjective), ctypes.c_void_p])


class RadiatedPowerS11:
    """w_prad * sum_k P_rad,k + w_s11 * sum_k |S11_k|^2 (2D TM).

    ``box`` = (il, ir, jb, jt) is the flux contour (poynting_flux_box_2d),
    ``port_ij`` the Ez cell of the port whose S11 is taken against
    ``resistance``, ``freqs`` the DFT frequencies of the run. ``monitors()``
    lists the DFT boxes the objective reads (pass them as
    ``objective_monitors``)."""

    def __init__(self, grid, box, port_ij, freqs, resistance: float = 50.0,
                 w_prad: float = 1.0, w_s11: float = -1.0):
        self.grid = grid
        self.freqs = tuple(float(f) for f in freqs)
        self.box = tuple(int(v) for v in box)
        self.port_ij = tuple(int(v) for v in port_ij)
        self.resistance = float(resistance)
        self.w_prad = float(w_prad)
        self.w_s11 = float(w_s11)
        self._cells = None

    def monitors(self):
        return poynting_box_monitors(self.box) + port_monitors(self.port_ij)

    def __call__(self, ph):
        from gradenna_b200.freq_adjoint import ports_from_fields

        p = poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, self.grid, self.box)
        v, i = ports_from_fields(ph.dft_ez, ph.dft_hx, ph.dft_hy, self.grid, [self.port_ij],
                                 self.freqs)
        s = s11_power_wave(v[:, 0], i[:, 0], self.resistance)
        return self.w_prad * p.sum() + self.w_s11 * (s.real ** 2 + s.imag ** 2).sum()

    def _desc(self, freqs, mons, outs):
        g = self.grid
        d = TmObjective()
        d.n_freq = len(freqs)
        d.box[:] = self.box
        d.port[:] = self.port_ij
        d.nx, d.ny = g.nx, g.ny
        arr = (_native.DftMonitor * max(len(mons), 1))()
        for k, ((c, lo0, lo1, hi0, hi1), t) in enumerate(zip(mons, outs)):
            arr[k].comp = c
            arr[k].lo[0], arr[k].lo[1], arr[k].hi[0], arr[k].hi[1] = lo0, lo1, hi0, hi1
            arr[k].out = t.data_ptr() if t is not None else None
        d.n_monitors = len(mons)
        d.monitors = arr
        fr = (ctypes.c_double * len(freqs))(*freqs)
        d.freqs = fr
        d.dx, d.dy, d.dt, d.dz = g.dx, g.dy, g.dt, DZ
        d.resistance, d.w_prad, d.w_s11 = self.resistance, self.w_prad, self.w_s11
        d.eps0, d.mu0 = EPS0, MU0
        return d, (arr, fr)

    def cells(self):
        """Host (n, 2) int32 cell lists (Ez, Hx, Hy) of the adjoint weights' rows
        (computed once per objective: they depend on the geometry only)."""
        if self._cells is not None:
            return [c.copy() for c in self._cells]
        lib = _native.load()
        d, keep = self._desc(self.freqs, [], [])
        n = [ctypes.c_int32() for _ in range(3)]
        _native.check(lib.gdn_tm_objective_cells(ctypes.byref(d), *(ctypes.byref(v) for v in n),
                                                 None, None, None))
        lists = [np.zeros((v.value, 2), np.int32) for v in n]
        _native.check(lib.gdn_tm_objective_cells(
            ctypes.byref(d), None, None, None,
            *(a.ctypes.data_as(_native.P_i32) for a in lists)))
        self._cells = lists
        return [c.copy() for c in lists]

    def fused_tm(self, mons, outs, device):
        """(value, p_rad, s11, [(ez_idx, W), (hx_idx, W), (hy_idx, W)]) from the
        forward run's monitors ``mons`` (boxes) and their complex128 outputs
        ``outs``, in one launch; W are (cells, n_freq) complex128."""
        if any(t is None or t.dtype != torch.complex128 for t in outs):
            raise ValueError("the fused objective reads complex128 monitor phasors")
        lib = _native.load()
        freqs = self.freqs
        K = len(freqs)
        lists = self.cells()
        value = torch.empty(1, dtype=torch.float64, device=device)
        p_rad = torch.empty(K, dtype=torch.float64, device=device)
        s11 = torch.empty(K, dtype=torch.complex128, device=device)
        ws = [torch.empty((len(c), K), dtype=torch.complex128, device=device) for c in lists]
        outs = [t.contiguous() for t in outs]
        d, keep = self._desc(freqs, mons, outs)
        d.value, d.p_rad, d.s11 = value.data_ptr(), p_rad.data_ptr(), s11.data_ptr()
        d.w_ez, d.w_hx, d.w_hy = (w.data_ptr() for w in ws)
        stream = torch.cuda.current_stream(device).cuda_stream
        with torch.cuda.device(device):
            _native.check(lib.gdn_tm_objective_prad_s11(ctypes.byref(d), stream))
        del keep
        return value[0], p_rad, s11, list(zip(lists, ws))
