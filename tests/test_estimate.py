"""CPU checks of gradenna_b200.estimate.

The reference-compatible 3D figures meet the reference's own sizing checks
(tests/test_topopt3d.py:271-330 of the reference): an 82x82x51 float32 run
of 2000 steps needs a few tens of MB forward, tens of GB for a naive
reverse sweep and low single-digit GB checkpointed; strip psi storage is
cheaper than full; DFT memory scales with frequencies and dtype; the
default checkpoint count is round(sqrt(N)); the fit report keys and
monotonicity. The B200 figures cover this library's runs: the benchmark's
2D (1024^2, K = 4) and 3D patch (160 x 160 x 64, K = 11) workloads and the
280 x 280 antenna's time-domain adjoint fit one B200 with a wide margin.
"""

import numpy as np
import pytest


def test_reference_sizing_checks():
    import gradenna_b200 as gb
    from gradenna_b200.estimate import fdtd3d_memory_estimate, fits_gpu, gpu_fit_report

    g = gb.Grid3D(82, 82, 51, 1.3e-3, 1.3e-3, 1.3e-3)
    est = fdtd3d_memory_estimate(g, 2000, n_dft_freqs=0, dtype="float32", cpml_thickness=10)
    assert 0.005 < est["fields_gb"] < 0.05 and 0.01 < est["forward_gb"] < 0.1
    assert 10.0 < est["adjoint_naive_gb"] < 100.0
    assert 0.5 < est["adjoint_checkpoint_gb"] < 5.0
    assert est["adjoint_checkpoint_gb"] < 0.2 * est["adjoint_naive_gb"]
    e1 = fdtd3d_memory_estimate(g, 2000, n_dft_freqs=1, dtype="float32", cpml_thickness=10)
    assert 0.0 < e1["psi_strip_gb"] < e1["psi_full_gb"]
    assert e1["adjoint_checkpoint_strip_gb"] < e1["adjoint_checkpoint_gb"]
    gs = gb.Grid3D(40, 40, 20, 1e-3, 1e-3, 1e-3)
    e0, e1, e4 = (fdtd3d_memory_estimate(gs, 1000, n_dft_freqs=k) for k in (0, 1, 4))
    assert e0["dft_monitor_gb"] == 0.0
    np.testing.assert_allclose(e4["dft_monitor_gb"], 4 * e1["dft_monitor_gb"], rtol=1e-12)
    e64 = fdtd3d_memory_estimate(gs, 1000, n_dft_freqs=1, dtype="float64")
    np.testing.assert_allclose(e64["fields_gb"], 2 * e1["fields_gb"], rtol=1e-12)
    assert fdtd3d_memory_estimate(gs, 2500)["checkpoint_segments"] == 50
    rep = gpu_fit_report(est)
    assert set(rep) == {24.0, 16.0, 8.0}
    if rep[8.0]:
        assert rep[16.0] and rep[24.0]
    assert fits_gpu(1.0, 24.0) and not fits_gpu(100.0, 24.0)
    with pytest.raises(ValueError):
        fdtd3d_memory_estimate(gs, 0)


def test_b200_figures():
    import gradenna_b200 as gb
    from gradenna_b200.estimate import (B200_VRAM_GB, fdtd2d_memory_estimate,
                                        fdtd3d_memory_estimate, gpu_fit_report)

    c2 = fdtd2d_memory_estimate(gb.Grid2D(1024, 1024, 1e-3, 1e-3), 8000, n_dft_freqs=4,
                                dft_dtype="complex128", design_cells=512 * 512)
    # 16 padded planes of ~1.1 M floats, 4 complex128 accumulators per cell
    # of three components, a 32-slot ring: well under 1 GB
    assert 0.05 < c2["b200_planes_gb"] < 0.1
    assert 0.3 < c2["b200_forward_gb"] < 1.0
    assert c2["b200_freq_gradient_gb"] > c2["b200_forward_gb"]
    c3 = fdtd3d_memory_estimate(gb.Grid3D(160, 160, 64, 5e-4, 5e-4, 5e-4), 6000,
                                n_dft_freqs=11, dft_dtype="complex128", design_cells=96 * 96)
    assert c3["b200_gradient_gb"] < c3["adjoint_checkpoint_gb"] < c3["adjoint_naive_gb"]
    assert gpu_fit_report(c3, key="b200_gradient_gb", vram_sizes_gb=(B200_VRAM_GB,))[B200_VRAM_GB]
    hero = fdtd2d_memory_estimate(gb.Grid2D(280, 280, 1e-3, 1e-3), 7000, n_dft_freqs=1,
                                  design_cells=104 * 104, time_adjoint=True)
    # two float32 histories of 7000 x 10816: 0.56 GiB
    np.testing.assert_allclose(hero["b200_history_gb"], 2 * 7000 * 10816 * 4 / 2**30, rtol=1e-12)
    assert hero["b200_time_gradient_gb"] < 0.05 * B200_VRAM_GB
