"""Host side of the fused 2D objective (gdn_tm_objective_cells): the rows of
the adjoint weight lists are exactly the cells the Poynting contour and the
port rebuild read (monitors.py:20-70, freq_adjoint.py:536-558), each once."""

import numpy as np
import pytest

from gradenna_b200.grid import Grid2D
from gradenna_b200.objectives import RadiatedPowerS11


def _expected(box, port):
    il, ir, jb, jt = box
    ez, hx, hy = set(), set(), set()
    for j in range(jb + 1, jt + 1):
        for i in (ir, il):
            ez |= {(i, j), (i + 1, j)}
            hy.add((i, j))
    for i in range(il + 1, ir + 1):
        for j in (jt, jb):
            ez |= {(i, j), (i, j + 1)}
            hx.add((i, j))
    pi, pj = port
    ez.add((pi, pj))
    hy |= {(pi, pj), (pi - 1, pj)}
    hx |= {(pi, pj), (pi, pj - 1)}
    return ez, hx, hy


@pytest.mark.parametrize("box,port", [((3, 9, 4, 12), (5, 6)), ((10, 30, 8, 25), (20, 8)),
                                      ((2, 5, 2, 5), (12, 12))])
def test_cell_lists_cover_what_the_objective_reads(box, port):
    g = Grid2D(40, 36, 1e-3, 1e-3)
    obj = RadiatedPowerS11(g, box, port, freqs=(2e9, 3e9))
    lists = obj.cells()
    for got, want in zip(lists, _expected(box, port)):
        rows = [tuple(r) for r in got.tolist()]
        assert len(rows) == len(set(rows))
        assert set(rows) == want


def test_invalid_geometry_is_refused():
    g = Grid2D(40, 36, 1e-3, 1e-3)
    with pytest.raises(RuntimeError, match="contour"):
        RadiatedPowerS11(g, (5, 3, 4, 12), (5, 6), freqs=(2e9,)).cells()
    with pytest.raises(RuntimeError, match="port"):
        RadiatedPowerS11(g, (3, 9, 4, 12), (0, 6), freqs=(2e9,)).cells()
    assert np.all(RadiatedPowerS11(g, (3, 9, 4, 12), (5, 6), freqs=(2e9,)).cells()[0] >= 0)
