"""Host-side parts of the path against the reference's OWN code, compiled from
its sources into oracle/_ref (oracle/ref_dc_shim.cpp + oracle/Makefile):

* the points-driven dual-contouring grid (OctreeGenerator::generateFromPoints
  + uniformizeFromPoints, upsample.cpp:128-144, :253-260, with grade /
  regularize_up / regularize_siblings and sorted_octree from octree.h),
  bit for bit;
* Pn::load of the reference's three shipped clouds with and without
  Pn::normalize (Pn.cpp:102-164, :262-290), bit for bit;
* Pn::order (Pn.cpp:388-445): the same Morton code sequence, and the same
  points inside every code (the reference sorts with the unstable std::sort,
  so the order inside one code is not defined by its source).

Skipped where the checkers were not built (they need the reference sources
once; the built library and data copies travel with the tree)."""
import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import io, synth
from mlodsurfaces_b200.apss import DCGrid

pytestmark = pytest.mark.skipif(not oracle.refdc_available(), reason="reference DC checker not built")

CLOUDS = ["Face.ply", "gargoyle_0.ply", "half-igea.ply"]


def _unit(pts, scale=0.9):
    return (pts / np.abs(pts).max() * scale).astype(np.float32)


@pytest.mark.parametrize("depth", [4, 6, 7])
def test_points_grid_equals_reference_code(depth):
    pts, _ = synth.torus(20000, seed=3)
    pts = _unit(pts)
    ref = oracle.RefDCGrid.from_points(pts, depth)
    g = DCGrid(pts, depth, device=False)
    assert np.array_equal(ref.cells(), g.cells)
    assert ref.max_depth == g.max_depth
    assert np.array_equal(ref.xform(), g.xform.ravel())


def test_points_grid_equals_reference_code_on_torus_knot_with_holes():
    pts, _ = synth.torus_knot(60000, seed=4)
    pts = _unit(pts, 0.97)
    ref = oracle.RefDCGrid.from_points(pts, 7)
    assert np.array_equal(ref.cells(), DCGrid(pts, 7, device=False).cells)


@pytest.mark.parametrize("name", CLOUDS)
@pytest.mark.parametrize("normalize", [True, False])
def test_cloud_load_equals_reference_pn_load(name, normalize):
    path = oracle.ref_data(name)
    if path is None:
        pytest.skip("reference data not copied")
    ref = oracle.refpn_load(path, normalize)
    pts, nrm, off, norme = io.load_cloud(path, normalize)
    assert np.array_equal(ref["pts"], pts)
    assert np.array_equal(ref["nrm"], nrm)
    if normalize:
        assert np.array_equal(ref["offset"], off)
        assert ref["norme"] == norme


def _ref_codes(p, grid):
    """Pn::order's cell of every point (Pn.cpp:400-414), float arithmetic."""
    f = np.float32
    mini = f(min(p[:, 0].min(), p[:, 1].min(), p[:, 2].min()))
    maxi = f(max(p[:, 0].max(), p[:, 1].max(), p[:, 2].max()))
    norme = f(maxi - mini)
    c = np.floor((p - mini) / norme * f(grid)).astype(np.int64)
    return np.clip(c, 0, grid - 1)


def _interleave(c):
    code = np.zeros(len(c), np.uint64)
    for b in range(10):
        for a in range(3):
            # _pdep_u32 masks 0x92492492 (x), 0x49249249 (y), 0x24924924 (z):
            # bit b of x lands at 3b + 1, of y at 3b, of z at 3b + 2
            pos = 3 * b + (1, 0, 2)[a]
            code |= (((c[:, a] >> b) & 1).astype(np.uint64) << np.uint64(pos))
    return code


@pytest.mark.parametrize("grid", [16, 64])
def test_morton_order_equals_reference_up_to_ties(grid):
    pts, _ = synth.torus(20000, seed=5)
    q = synth.perturbed_queries(pts, 0.01, seed=6).astype(np.float32)
    ref = oracle.refpn_order(q, grid)
    ours = q[io.morton_order(q, grid)]
    rc = _interleave(_ref_codes(ref, grid))
    oc = _interleave(_ref_codes(ours, grid))
    # same code at every position, non-decreasing
    assert np.array_equal(rc, oc)
    assert (np.diff(rc.astype(np.int64)) >= 0).all()
    # and the same points inside every code
    starts = np.flatnonzero(np.r_[True, rc[1:] != rc[:-1]])
    ends = np.r_[starts[1:], len(rc)]
    for s, e in zip(starts, ends):
        a = np.sort(ref[s:e].view("V12").ravel())
        b = np.sort(ours[s:e].view("V12").ravel())
        assert np.array_equal(a, b)
