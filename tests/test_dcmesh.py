"""Dual-contouring mesh extraction, smoothing and subdivision (host code of
the library) against the pure-Python restatement of the reference
(oracle/dcmesh.py): identical vertex order and triangle lists; the mesh of a
closed surface is a closed, consistently oriented 2-manifold."""
from collections import Counter

import numpy as np
import pytest

from mlodsurfaces_b200 import DCGrid, Mesh
from mlodsurfaces_b200 import _capi as capi
from oracle import dcmesh


def sphere_points(n, r, seed, center=(0.05, -0.03, 0.02)):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (v * r + np.asarray(center)).astype(np.float32)


def corner_field(grid, r, center=(0.05, -0.03, 0.02), nan_every=0):
    """Signed distance to a sphere at every cell corner (lattice of the
    deepest level, mapped through the grid's xform), float32."""
    md = grid.max_depth
    d = grid.cells[:, 0].astype(np.int64)
    delta = (np.int64(1) << (md - d))[:, None]
    bits = np.array([[k & 1, (k >> 1) & 1, (k >> 2) & 1] for k in range(8)], np.int64)
    lat = (grid.cells[:, None, 1:4].astype(np.int64) + bits[None]) * delta[:, :, None]
    u = lat.astype(np.float64) / (1 << md)
    w = u @ grid.xform[:, :3].T.astype(np.float64) + grid.xform[:, 3]
    f = (np.linalg.norm(w - np.asarray(center), axis=2) - r).astype(np.float32)
    if nan_every:
        key = (lat[..., 0] * 73856093) ^ (lat[..., 1] * 19349669) ^ (lat[..., 2] * 39349693)
        f[key % nan_every == 0] = np.nan
    return f, lat


def cell_vertices(grid):
    width = 1.0 / (np.int64(1) << grid.cells[:, 0].astype(np.int64))
    jitter = ((grid.cells[:, 1:4] * np.array([3, 5, 7])) % 11) / 11.0
    return ((grid.cells[:, 1:4] + 0.25 + 0.5 * jitter) * width[:, None]).astype(np.float32)


def oracle_mesh(grid, cf, lat, vx):
    values = {}
    for i in range(len(grid.cells)):
        for k in range(8):
            values[tuple(lat[i, k])] = cf[i, k]
    by_cell = {tuple(c): vx[i] for i, c in enumerate(grid.cells.tolist())}
    tree, order, verts, tris = dcmesh.extract(grid.cells.tolist(), lambda c: values[tuple(c)],
                                              lambda c: by_cell[tuple(c)])
    return np.array(verts, np.float32).reshape(-1, 3), np.array(tris, np.int64).reshape(-1, 3)


@pytest.fixture(scope="module", params=[(4, 0.55), (5, 0.4)])
def sphere_grid(request):
    depth, r = request.param
    g = DCGrid(sphere_points(4000, r, seed=depth), depth)
    return g, r


def test_extraction_matches_reference_order(sphere_grid):
    g, r = sphere_grid
    cf, lat = corner_field(g, r)
    vx = cell_vertices(g)
    v, n, t = Mesh.extract(g.cells, cf, vx).arrays()
    ov, ot = oracle_mesh(g, cf, lat, vx)
    assert len(t) > 100
    assert np.array_equal(t.astype(np.int64), ot)
    assert np.array_equal(v, ov)
    assert np.all(n == 0)  # the reference's zero normal field


def test_sphere_mesh_is_closed_and_oriented(sphere_grid):
    g, r = sphere_grid
    cf, _ = corner_field(g, r)
    v, _, t = Mesh.extract(g.cells, cf, cell_vertices(g)).arrays()
    directed = Counter()
    for a, b, c in t.tolist():
        for e in ((a, b), (b, c), (c, a)):
            directed[e] += 1
    assert all(cnt == 1 for cnt in directed.values())  # no edge used twice in one direction
    assert all(directed[(b, a)] == 1 for (a, b) in directed)  # every edge has its opposite
    assert len(np.unique(t)) == len(v)  # every vertex is used


def test_nan_corners_skip_edges_like_the_reference(sphere_grid):
    g, r = sphere_grid
    cf, lat = corner_field(g, r, nan_every=7)
    vx = cell_vertices(g)
    v, _, t = Mesh.extract(g.cells, cf, vx).arrays()
    ov, ot = oracle_mesh(g, cf, lat, vx)
    assert np.array_equal(t.astype(np.int64), ot) and np.array_equal(v, ov)


def test_smooth_and_subdivide_match_reference():
    g = DCGrid(sphere_points(3000, 0.5, seed=9), 4)
    cf, _ = corner_field(g, 0.5)
    m = Mesh.extract(g.cells, cf, cell_vertices(g))
    v, _, t = m.arrays()
    m.transform(g.xform)
    v = v @ g.xform[:, :3].T + g.xform[:, 3]
    v0, _, _ = m.arrays()
    assert np.allclose(v0, v, atol=1e-6)
    ref_v, ref_t = v0, t
    for _ in range(2):
        m.smooth()
        m.subdivide()
        ref_v = dcmesh.smooth(ref_v, ref_t.tolist())
        ref_v, ref_t = dcmesh.subdivide(ref_v, ref_t.tolist())
        ref_t = np.array(ref_t, np.int64)
        mv, mn, mt = m.arrays()
        assert np.array_equal(mt.astype(np.int64), ref_t)
        assert np.array_equal(mv, ref_v)
        assert mn.shape == mv.shape


def test_extract_rejects_unregularized_grids():
    cells = np.array([[0, 0, 0, 0], [1, 0, 0, 0], [1, 1, 0, 0]], np.int32)  # 2 of 8 children
    with pytest.raises(capi.MlodsError):
        Mesh.extract(cells, np.zeros((3, 8), np.float32), np.zeros((3, 3), np.float32))
    unsorted = np.array([[1, 1, 0, 0], [0, 0, 0, 0]], np.int32)
    with pytest.raises(capi.MlodsError):
        Mesh.extract(unsorted, np.zeros((2, 8), np.float32), np.zeros((2, 3), np.float32))
