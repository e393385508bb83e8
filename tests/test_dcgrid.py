"""DC grid construction (host code in libmlods) against the Python
restatement of generateFromPoints + uniformizeFromPoints (no GPU needed)."""
import numpy as np
import pytest

from mlodsurfaces_b200 import DCGrid, synth
from oracle import dcgrid


@pytest.mark.parametrize("depth", [3, 5, 6])
def test_grid_matches_restatement(depth):
    p, _ = synth.torus(4000, seed=depth)
    p = synth.normalize_like_pn(p)
    g = DCGrid(p, depth)
    o = dcgrid.grid_from_points(p, depth)
    assert g.max_depth == depth
    assert np.array_equal(g.cells, o)


def test_grid_of_torus_knot_matches_restatement():
    p, _ = synth.torus_knot(3000, seed=4)
    p = synth.normalize_like_pn(p)
    g = DCGrid(p, 6)
    assert np.array_equal(g.cells, dcgrid.grid_from_points(p, 6))


def test_grid_is_complete_and_sorted():
    p, _ = synth.torus(2000, seed=9)
    g = DCGrid(synth.normalize_like_pn(p), 5)
    cells = [tuple(c) for c in g.cells]
    keys = [dcgrid.key(c) for c in cells]
    assert keys == sorted(keys) and len(set(cells)) == len(cells)
    s = set(cells)
    for c in cells:  # every non-root cell has its parent and all its siblings
        if c[0] > 0:
            par = dcgrid.parent(c)
            assert par in s
            assert all(dcgrid.child(par, k) in s for k in range(8))
