"""The CPU oracles against golden vectors written by the reference's own code.

``tests/golden/*.npz`` hold the outputs of the reference's unmodified
``simulate_tm`` / ``simulate_3d``, ``poynting_flux_box_2d``, ``port_dft`` +
``s11_power_wave``, ``port_impedance``, ``ntff_3d`` / ``directivity_3d``,
``conic_filter`` / ``tanh_projection`` / ``DesignTransform`` and
``axis_coefficients`` on seeded inputs (``tests/golden/make_golden.py``).
Here the numpy oracle (and the C oracle for 2D) must reproduce them:

  float64: <= 1e-12 peak-normalised on every output (the numpy oracle
           reproduces the reference's float64 arithmetic; in practice 0);
  float32: <= 1e-5 on records, phasors, P_rad and S11, <= 1e-4 on final
           fields in 2D (the reference's own float32 bars,
           tests/test_native.py:50-51) and <= 2e-3 on 3D final fields
           (tests/test_native3d.py:63-64).

This pins the oracle, which every GPU parity test then uses as its checker.
"""

import types

import numpy as np
import pytest

from oracle import fdtd2d_np as o2
from oracle import fdtd3d_np as o3
from oracle import ntff_np as on
from tests.golden import cases as gc

RTOL = {np.float64: 1e-12, np.float32: 1e-5}
RTOL_FIELD = {np.float64: 1e-12, np.float32: 1e-4}
RTOL_FIELD_3D = {np.float64: 1e-12, np.float32: 2e-3}
FIELDS = ("ez", "hx", "hy", "ex", "ey", "hz", "energy")


def tol(case, key):
    if key in FIELDS:
        return (RTOL_FIELD_3D if case["kind"] == "yee" else RTOL_FIELD)[case["dtype"]]
    return RTOL[case["dtype"]]


def check(case, got, want):
    sel = gc.select(case, got)
    missing = set(want) - set(sel)
    assert not missing, f"{case['name']}: outputs missing {sorted(missing)}"
    errs = {k: gc.rel(sel[k], want[k]) for k in want}
    bad = {k: e for k, e in errs.items() if e > tol(case, k)}
    assert not bad, f"{case['name']}: {bad}"
    return errs


ORACLE2 = types.SimpleNamespace(
    Grid2D=o2.Grid2D, CPMLSpec=o2.CPMLSpec, Port=o2.Port, simulate_tm=o2.simulate_tm,
    poynting_flux_box_2d=o2.poynting_flux_box_2d, port_dft=o2.port_dft,
    s11_power_wave=o2.s11_power_wave)


@pytest.mark.parametrize("case", gc.tm_cases(), ids=lambda c: c["name"])
def test_numpy_oracle_2d(case):
    want = gc.load(case["name"], case)
    got = gc.run_tm(ORACLE2, case, oracle=True)
    check(case, got, want)


def _c_api():
    from oracle import tm2d_c

    tm2d_c.build()

    def sim(g, *, dtype, dft_dtype=None, **kw):
        return tm2d_c.simulate_tm_c(g, dtype=dtype, **kw)[0]

    return types.SimpleNamespace(**{**vars(ORACLE2), "simulate_tm": sim})


@pytest.mark.parametrize("case", gc.tm_cases(), ids=lambda c: c["name"])
def test_c_oracle_2d(case):
    """The C restatement (the timed CPU baseline and the checker of the
    large GPU cases) reproduces the same fixtures. Its DFT accumulates in
    double, so float32 phasors meet the float32 bar rather than bit-level
    equality."""
    want = gc.load(case["name"], case)
    got = gc.run_tm(_c_api(), case, oracle=True)
    check(case, got, want)


_COMPS = ("ex", "ey", "ez", "hx", "hy", "hz")


def _oracle3_api():
    from gradenna_b200 import dft_region as dr

    def simulate_3d(g, *, cpml, dtype, dft_dtype=None, dft_regions=None, **kw):
        regs = None
        if dft_regions is not None:
            regs = {c: (tuple(s.lo), tuple(s.hi)) for c, s in zip(_COMPS, dft_regions)
                    if s is not None}
        r = o3.simulate_3d(g, cpml=cpml, dtype=dtype, dft_regions=regs, **kw)
        mon = None
        if r.dft is not None:
            mon = types.SimpleNamespace(freqs=np.asarray(kw["dft_freqs"]), regions=dft_regions,
                                        **{c: r.dft.get(c) for c in _COMPS})
        return r._replace(dft=mon)

    def scatter_full(mon, shapes):
        full = {}
        for c, s, shp in zip(_COMPS, mon.regions, shapes):
            a = np.zeros((len(mon.freqs),) + tuple(shp), complex)
            if s is not None and getattr(mon, c) is not None:
                a[(slice(None),) + s.slices()] = getattr(mon, c)
            full[c] = a
        return types.SimpleNamespace(freqs=mon.freqs, **full)

    def ntff_3d(mon, g, m, freqs, th, ph):
        d = {c: np.asarray(getattr(mon, c)) for c in _COMPS}
        return on.ntff_3d(d, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, m, freqs, th, ph)

    return types.SimpleNamespace(
        Grid3D=o3.Grid3D, CPMLSpec=o2.CPMLSpec, simulate_3d=simulate_3d,
        port_impedance=o3.port_impedance, ntff_3d=ntff_3d,
        design_region_to_slabs=dr.design_region_to_slabs, port_regions=dr.port_regions,
        ntff_box_regions=dr.ntff_box_regions, union_regions=dr.union_regions,
        full_field_shapes=dr.full_field_shapes, scatter_full=scatter_full)


@pytest.mark.parametrize("case", gc.yee_cases(), ids=lambda c: c["name"])
def test_numpy_oracle_3d(case):
    want = gc.load(case["name"], case)
    got = gc.run_yee(_oracle3_api(), case, oracle=True)
    if "e_theta" in got:
        th, ph = case["ntff"][1], case["ntff"][2]
        got["directivity"] = on.directivity_3d(got["e_theta"], got["e_phi"], th, ph)
    check(case, got, want)


def test_cpml_tables_match_reference():
    """gradenna_b200.cpml.axis_coefficients (the tables the CUDA kernels read)
    equals the reference's cpml.axis_coefficients."""
    import gradenna_b200 as gb

    allc = gc.cpml_cases()
    want = gc.load("cpml_tables", allc)
    for q, c in enumerate(allc):
        spec = gb.CPMLSpec(thickness=c["thickness"])
        for half in (False, True):
            for dt_ in (np.float64, np.float32):
                a = gb.axis_coefficients(c["n"], c["delta"], c["dt"], spec, half=half, dtype=dt_)
                tag = f"{q}_{'h' if half else 'e'}_{np.dtype(dt_).name}"
                for nm, v in (("b", a.b), ("c", a.c), ("ik", a.inv_kappa)):
                    v = np.asarray(v.cpu() if hasattr(v, "cpu") else v)
                    w = want[f"{nm}_{tag}"]
                    assert v.dtype == w.dtype, (tag, nm, v.dtype, w.dtype)
                    e = gc.rel(v, w)
                    assert e <= (1e-15 if dt_ is np.float64 else 1e-7), (tag, nm, e)


def test_design_transform_cpu_matches_reference():
    """The library's torch design transform (sigmoid -> conic filter ->
    tanh projection, float64 on the CPU) equals the reference's
    fftconvolve-based DesignTransform; the filtered and projected fields
    alone match conic_filter and tanh_projection."""
    import torch

    from gradenna_b200 import topopt

    allc = gc.design_cases()
    want = gc.load("design_transform", allc)
    for c in allc:
        th = torch.tensor(c["theta"], dtype=torch.float64)
        rho = torch.sigmoid(th)
        filt = topopt.conic_filter(rho, c["radius"])
        proj = topopt.tanh_projection(filt, c["beta"], c["eta"])
        full = topopt.DesignTransform(c["radius"], c["eta"])(th, c["beta"])
        for nm, v in (("filtered", filt), ("projected", proj), ("transform", full)):
            e = gc.rel(v.numpy(), want[f"{c['name']}__{nm}"])
            assert e <= 1e-12, (c["name"], nm, e)
