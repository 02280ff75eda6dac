#!/usr/bin/env python
"""Write the golden vectors in ``tests/golden/*.npz`` from the reference's own
code.

The reference (s-hosomi/gradenna, ``src/gradenna``) is imported unmodified
through the numpy stand-in for ``jax`` (``tests/golden/jaxshim``, see
``refload.py``): its ``simulate_tm`` / ``simulate_3d`` scans become Python
loops over numpy arrays, its ``.at[]`` updates become copies with
scatter-add/assign. Every case's inputs come from ``cases.py``; each fixture
stores the outputs and a digest of the inputs.

Usage (needs the reference source, by default at /root/reference; override
with GRADENNA_REFERENCE):

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py tm_readme   # names starting with ...

Runs on the CPU in under a minute. The float64 fixtures are the reference's
float64 arithmetic exactly; the float32 fixtures follow its float32
operation order under numpy rounding (XLA may fuse differently; the
reference itself documents 1e-5 reassociation drift between its two
float32 back ends, tests/test_native.py:44-51).
"""

from __future__ import annotations

import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import cases  # noqa: E402
import refload  # noqa: E402


def ref_apis():
    (fdtd2d, cpml, grid, monitors, sparams, fdtd3d, ntff, dft_region, topopt) = refload.load(
        "fdtd2d", "cpml", "grid", "monitors", "sparams", "fdtd3d", "ntff", "dft_region", "topopt")
    api2 = types.SimpleNamespace(
        Grid2D=grid.Grid2D, CPMLSpec=cpml.CPMLSpec, Port=fdtd2d.Port,
        simulate_tm=fdtd2d.simulate_tm, poynting_flux_box_2d=monitors.poynting_flux_box_2d,
        port_dft=sparams.port_dft, s11_power_wave=sparams.s11_power_wave)
    api3 = types.SimpleNamespace(
        Grid3D=grid.Grid3D, CPMLSpec=cpml.CPMLSpec, simulate_3d=fdtd3d.simulate_3d,
        port_impedance=fdtd3d.port_impedance, ntff_3d=ntff.ntff_3d,
        design_region_to_slabs=dft_region.design_region_to_slabs,
        port_regions=dft_region.port_regions, ntff_box_regions=dft_region.ntff_box_regions,
        union_regions=dft_region.union_regions, full_field_shapes=dft_region.full_field_shapes,
        scatter_full=dft_region.scatter_full)
    return api2, api3, topopt, cpml, ntff


def main(prefixes):
    api2, api3, topopt, cpml, ntff = ref_apis()

    def wanted(name):
        return not prefixes or any(name.startswith(p) for p in prefixes)

    for case in cases.tm_cases() + cases.yee_cases():
        if not wanted(case["name"]):
            continue
        t0 = time.time()
        if case["kind"] == "tm":
            out = cases.run_tm(api2, case)
        else:
            out = cases.run_yee(api3, case)
            if "e_theta" in out:
                th, ph = case["ntff"][1], case["ntff"][2]
                out["directivity"] = np.asarray(ntff.directivity_3d(
                    out["e_theta"], out["e_phi"], np.asarray(th), np.asarray(ph)))
        cases.save(case["name"], case, out)
        print(f"{case['name']}: {sorted(cases.select(case, out))} ({time.time() - t0:.1f} s)")

    if wanted("design"):
        outs = {}
        allc = cases.design_cases()
        for c in allc:
            th = c["theta"]
            rho = 1.0 / (1.0 + np.exp(-th))
            filt = np.asarray(topopt.conic_filter(rho, c["radius"]))
            proj = np.asarray(topopt.tanh_projection(filt, c["beta"], c["eta"]))
            full = np.asarray(topopt.DesignTransform(c["radius"], c["eta"])(th, c["beta"]))
            outs[c["name"] + "__filtered"] = filt
            outs[c["name"] + "__projected"] = proj
            outs[c["name"] + "__transform"] = full
        cases.save("design_transform", allc, outs)
        print("design_transform:", len(outs), "arrays")

    if wanted("cpml"):
        outs = {}
        allc = cases.cpml_cases()
        for q, c in enumerate(allc):
            spec = cpml.CPMLSpec(thickness=c["thickness"])
            for half in (False, True):
                for dt_ in (np.float64, np.float32):
                    a = cpml.axis_coefficients(c["n"], c["delta"], c["dt"], spec, half=half,
                                               dtype=dt_)
                    tag = f"{q}_{'h' if half else 'e'}_{np.dtype(dt_).name}"
                    outs[f"b_{tag}"] = np.asarray(a.b)
                    outs[f"c_{tag}"] = np.asarray(a.c)
                    outs[f"ik_{tag}"] = np.asarray(a.inv_kappa)
        cases.save("cpml_tables", allc, outs)
        print("cpml_tables:", len(outs), "arrays")


if __name__ == "__main__":
    main(sys.argv[1:])
