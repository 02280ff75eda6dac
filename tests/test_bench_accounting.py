"""The benchmark's byte accounting on the CPU (no GPU needed).

The JSON line's roofline carries two fractions: the fields' algorithmic
bytes (2D: 8 words per cell-step, 3D: 14) and the same plus the survey's DFT
term, the complex128 accumulators of every monitored cell read and written
per step and frequency. These tests pin the monitored-cell counts the second
figure uses to the monitor boxes the gradient actually records.
"""

import types

import numpy as np

import bench


def _args(workload, steps):
    return types.SimpleNamespace(workload=workload, grid=bench.N_GRID, time_steps=steps,
                                 dtype="f32", gpus=1)


def test_2d_dft_cells_are_the_design_plus_half_the_objective_boxes():
    case = bench.make_case(_args("tm2d", 40), 0)
    w = case["w"]
    design = int(np.asarray(w["sigma_d"]).size)
    mons = bench.monitors_for(w)
    obj = sum((hi0 - lo0) * (hi1 - lo1) for _, lo0, lo1, hi0, hi1 in mons)
    # the design's Ez is recorded in both runs, the objective boxes in the
    # forward run only
    assert case["dft_cells"] == design + obj / 2
    assert case["n_freq"] == len(bench.FREQS) and case["tb"] == 4 and case["words"] == 8
    # Poynting contour strips and lines plus the ports' cells: a few thousand
    assert 0 < obj < 20000


def test_3d_dft_cells_count_component_cells_of_every_box():
    from gradenna_b200 import dft_region as dr
    from gradenna_b200.freq_adjoint3d import _objective_boxes

    case = bench.make_case(_args("patch3d", 10), 0)
    w = case["w"]
    g = w["grid"]
    shapes = dr.full_field_shapes(g.nx, g.ny, g.nz)
    design = dr.region_boxes(dr.design_region_to_slabs(w["design"], shapes))
    obj = _objective_boxes(g, ("port", "ntff_box"), port_ijk=w["port"], box_margin=bench.P3_BOX)

    def cells(boxes):
        return sum(int(np.prod(np.subtract(hi, lo))) for _, lo, hi in boxes)

    assert case["dft_cells"] == cells(design) + cells(obj) / 2
    assert case["n_freq"] == len(bench.P3_FREQS) and case["tb"] == 1 and case["words"] == 14
    # the NTFF box faces dominate: four tangential components on six faces
    assert cells(obj) > 10 * cells(design)


def test_lpt_partition_is_deterministic_and_balanced_on_the_population():
    specs = bench.population(0, n_problems=64, max_steps=50)
    costs = [bench.pop_cells([sp]) for sp in specs]
    a = bench.lpt_partition(costs, 4)
    assert a == bench.lpt_partition(costs, 4)
    loads = [sum(costs[i] for i in p) for p in a]
    assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / 4, max(costs))
