"""GPU parity of the 2D TM CUDA path against the CPU oracle.

The cases are those the reference uses to pin its native kernel against
simulate_tm (tests/test_native.py:66-153): CPML + probes + energy, two line
sources + two RVS ports + DFT, magnetic-current sources, and a PEC box. The
tolerances are the reference's (tests/test_native.py:50-51), peak-normalised:

  float64: <= 1e-12 on every output;
  float32: <= 1e-5 on probes, port V/I and DFT phasors, <= 1e-4 on final fields.

Each float32 result is also compared against the float64 oracle, and the
error is reported (the float32-vs-float64 gap is the physics of single
precision, bounded here at 1e-3).
"""

import numpy as np
import pytest
import torch

from oracle import fdtd2d_np as ref

pytestmark = pytest.mark.gpu

RTOL = {np.float64: 1e-12, np.float32: 1e-5}
RTOL_FIELD = {np.float64: 1e-12, np.float32: 1e-4}


def _np(x):
    return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def rel(a, b):
    a, b = _np(a), _np(b)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


def _gauss(grid, n_steps, dtype):
    t = (np.arange(n_steps) + 0.5) * grid.dt
    return np.asarray(ref.gaussian_derivative(t, 20 * grid.dt, 6 * grid.dt), dtype)


def _run_both(dtype, g_ref, kw_ref, kw_gpu):
    import gradenna_b200 as gb

    r_gpu = gb.simulate_tm(gb.Grid2D(g_ref.nx, g_ref.ny, g_ref.dx, g_ref.dy), **kw_gpu,
                           dtype=dtype)
    r_ref = ref.simulate_tm(g_ref, **kw_ref, dtype=dtype)
    r_64 = ref.simulate_tm(g_ref, **kw_ref, dtype=np.float64) if dtype == np.float32 else r_ref
    torch.cuda.synchronize()
    return r_gpu, r_ref, r_64


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_basic_cpml(dtype):
    import gradenna_b200 as gb

    g = ref.Grid2D(48, 52, 1e-3, 1e-3)
    n_steps = 400
    src = _gauss(g, n_steps, dtype)
    probe = ((12, 14), (30, 34))
    kw = dict(source_ij=(24, 26), source_current=src, probe_ij=probe, record_energy=True)
    r_gpu, r_ref, r_64 = _run_both(
        dtype, g, dict(kw, cpml=ref.CPMLSpec(thickness=8)), dict(kw, cpml=gb.CPMLSpec(thickness=8)))
    assert rel(r_gpu.probe_ez, r_ref.probe_ez) <= RTOL[dtype]
    assert rel(r_gpu.energy, r_ref.energy) <= RTOL[dtype]
    assert rel(r_gpu.ez, r_ref.ez) <= RTOL_FIELD[dtype]
    assert rel(r_gpu.hx, r_ref.hx) <= RTOL_FIELD[dtype]
    assert rel(r_gpu.hy, r_ref.hy) <= RTOL_FIELD[dtype]
    assert rel(r_gpu.probe_ez, r_64.probe_ez) <= 1e-3


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("dft_dtype", [None, np.complex128])
def test_multi_source_ports_dft(dtype, dft_dtype):
    import gradenna_b200 as gb

    g = ref.Grid2D(44, 40, 2e-3, 2e-3)
    n_steps = 500
    freqs = (3e9, 5e9)
    base = _gauss(g, n_steps, dtype)
    srcs = np.stack([base, 0.3 * base], axis=1).astype(dtype)
    vs = (0.5 * base).astype(dtype)
    common = dict(source_ij=((15, 18), (25, 22)), source_current=srcs,
                  probe_ij=((10, 12), (30, 30)), dft_freqs=freqs, dft_dtype=dft_dtype)
    r_gpu, r_ref, r_64 = _run_both(
        dtype, g,
        dict(common, cpml=ref.CPMLSpec(8), ports=[ref.Port((20, 20), 50.0, vs), ref.Port((22, 24), 75.0, None)]),
        dict(common, cpml=gb.CPMLSpec(8), ports=[gb.Port((20, 20), 50.0, vs), gb.Port((22, 24), 75.0, None)]),
    )
    for name in ("probe_ez", "port_v", "port_i", "dft_ez", "dft_hx", "dft_hy"):
        e = rel(getattr(r_gpu, name), getattr(r_ref, name))
        assert e <= RTOL[dtype], f"{name}: {e:.2e}"
        assert rel(getattr(r_gpu, name), getattr(r_64, name)) <= 1e-3
    assert rel(r_gpu.ez, r_ref.ez) <= RTOL_FIELD[dtype]
    want = torch.complex128 if (dft_dtype is not None or dtype == np.float64) else torch.complex64
    assert r_gpu.dft_ez.dtype == want


def test_magnetic_current_sources():
    import gradenna_b200 as gb

    dtype = np.float64
    g = ref.Grid2D(40, 40, 2e-3, 2e-3)
    n_steps = 300
    base = _gauss(g, n_steps, dtype)
    kw = dict(source_ij=(20, 20), source_current=base,
              mx_ij=((18, 20), (22, 18)), mx_current=np.stack([base, 0.5 * base], 1),
              my_ij=(20, 22), my_current=0.7 * base, probe_ij=((15, 15),),
              dft_freqs=(4e9,), dft_dtype=np.complex128)
    r_gpu, r_ref, _ = _run_both(dtype, g, dict(kw, cpml=ref.CPMLSpec(8)), dict(kw, cpml=gb.CPMLSpec(8)))
    assert rel(r_gpu.probe_ez, r_ref.probe_ez) <= RTOL[dtype]
    assert rel(r_gpu.dft_ez, r_ref.dft_ez) <= RTOL[dtype]
    assert rel(r_gpu.dft_hx, r_ref.dft_hx) <= RTOL[dtype]
    assert rel(r_gpu.dft_hy, r_ref.dft_hy) <= RTOL[dtype]


def test_no_pml_pec_box():
    import gradenna_b200 as gb

    dtype = np.float64
    g = ref.Grid2D(36, 36, 1e-3, 1e-3)
    src = _gauss(g, 250, dtype)
    kw = dict(source_ij=(18, 18), source_current=src, probe_ij=((10, 10),))
    r_gpu, r_ref, _ = _run_both(dtype, g, dict(kw, cpml=ref.CPMLSpec(0)), dict(kw, cpml=gb.CPMLSpec(0)))
    assert rel(r_gpu.probe_ez, r_ref.probe_ez) <= RTOL[dtype]
    assert rel(r_gpu.ez, r_ref.ez) <= RTOL[dtype]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_ragged_tiles_and_edge_probes(dtype):
    """Grid sizes that are not tile multiples, sources/ports/probes at tile
    seams and on the PEC ring, a step count not a multiple of the DFT block."""
    import gradenna_b200 as gb

    g = ref.Grid2D(37, 71, 1.5e-3, 1e-3)
    n_steps = 97
    base = _gauss(g, n_steps, dtype)
    kw = dict(source_ij=((8, 31), (16, 32), (16, 32)),
              source_current=np.stack([base, -base, 0.5 * base], 1),
              probe_ij=((0, 0), (36, 70), (8, 31), (7, 32), (15, 63)),
              dft_freqs=(2e9, 7e9, 11e9), record_energy=True)
    r_gpu, r_ref, _ = _run_both(
        dtype, g,
        dict(kw, cpml=ref.CPMLSpec(5), ports=[ref.Port((9, 32), 25.0, base), ref.Port((9, 32), 100.0, None)]),
        dict(kw, cpml=gb.CPMLSpec(5), ports=[gb.Port((9, 32), 25.0, base), gb.Port((9, 32), 100.0, None)]),
    )
    for name in ("probe_ez", "port_v", "port_i", "dft_ez", "dft_hx", "dft_hy", "energy"):
        e = rel(getattr(r_gpu, name), getattr(r_ref, name))
        assert e <= RTOL[dtype], f"{name}: {e:.2e}"
    assert np.all(_np(r_gpu.probe_ez)[:, 0] == 0.0)
    for name in ("ez", "hx", "hy"):
        assert rel(getattr(r_gpu, name), getattr(r_ref, name)) <= RTOL_FIELD[dtype]


def test_dft_region_matches_full_grid():
    import gradenna_b200 as gb

    g = gb.Grid2D(64, 64, 2e-3, 2e-3)
    src = _gauss(g, 200, np.float32)
    kw = dict(source_ij=(30, 30), source_current=src, dft_freqs=(3e9, 4e9), cpml=gb.CPMLSpec(8))
    full = gb.simulate_tm(g, **kw)
    part = gb.simulate_tm(g, **kw, dft_region=((10, 12, 40, 50), None, (5, 6, 7, 60)))
    assert part.dft_hx is None
    assert torch.equal(part.dft_ez, full.dft_ez[:, 10:40, 12:50])
    assert torch.equal(part.dft_hy, full.dft_hy[:, 5:7, 6:60])


def test_zero_steps_and_bad_args():
    import gradenna_b200 as gb

    g = gb.Grid2D(20, 20, 1e-3, 1e-3)
    r = gb.simulate_tm(g, source_ij=(10, 10), source_current=np.zeros(0, np.float32),
                       cpml=gb.CPMLSpec(4))
    assert r.probe_ez.shape == (0, 0) and float(r.ez.abs().max()) == 0.0
    with pytest.raises(ValueError):
        gb.simulate_tm(g, source_ij=(0, 10), source_current=np.zeros(5), cpml=gb.CPMLSpec(4))
    with pytest.raises(ValueError):
        gb.simulate_tm(g, source_ij=(10, 10), source_current=np.zeros(5), cpml=gb.CPMLSpec(9))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_heterogeneous_eps_sigma_and_metal(dtype):
    """Media beyond the reference's native cases: eps_r in [1, 4] and sigma
    from lossy (up to 5 S/m, where c_a turns negative) to metal (1e5 S/m),
    with a source, a probe and a DFT."""
    import gradenna_b200 as gb

    g = ref.Grid2D(48, 44, 1e-3, 1e-3)
    rng = np.random.default_rng(4)
    n_steps = 600
    src = _gauss(g, n_steps, dtype)
    eps_r = 1.0 + 3.0 * rng.uniform(0, 1, (48, 44))
    sigma = 10.0 ** (-4 + 9 * rng.uniform(0, 1, (48, 44)))
    sigma[:, :20] = rng.uniform(0, 5, (48, 20))
    kw = dict(source_ij=(24, 30), source_current=src, probe_ij=((12, 14), (30, 34)),
              dft_freqs=(3e9,))
    r_gpu, r_ref, r_64 = _run_both(
        dtype, g, dict(kw, eps_r=eps_r, sigma=sigma, cpml=ref.CPMLSpec(8)),
        dict(kw, eps_r=torch.as_tensor(eps_r), sigma=torch.as_tensor(sigma),
             cpml=gb.CPMLSpec(8)))
    for name in ("probe_ez", "dft_ez", "dft_hx", "dft_hy"):
        assert rel(getattr(r_gpu, name), getattr(r_ref, name)) <= RTOL[dtype], name
        assert rel(getattr(r_gpu, name), getattr(r_64, name)) <= 1e-3, name
    assert rel(r_gpu.ez, r_ref.ez) <= RTOL_FIELD[dtype]
