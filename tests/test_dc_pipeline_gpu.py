"""The projection-driven DC grid and the whole DC mesh pipeline on the GPU.

* adaptive grid: the library's generator against the Python restatement of
  OctreeGenerator::generate + uniformize fed with the same projections;
* pipeline: mlods_dc_mesh against the same steps composed from the parts
  (corner field, extraction, transform, projections, smooth, subdivide), the
  connectivity against the restatement of the extraction, and the refined
  vertices against the FP64 oracle projection of the same mesh.
"""
from collections import Counter

import numpy as np
import pytest

import oracle
from oracle import dcgrid as odg
from oracle import dcmesh
from mlodsurfaces_b200 import APSSOctree, DCGrid, Fastapss, Mesh, synth
from conftest import TOL_DIAG, make_kernel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FLT_MAX = float(np.finfo(np.float32).max)


@pytest.fixture(scope="module")
def torus_apss():
    pts, nrm = synth.torus(30000, seed=71)
    pts = synth.make_tie_free(synth.normalize_like_pn(pts))
    diag = synth.bbox_diag(pts)
    k = make_kernel("singular", diag)
    t = APSSOctree()
    t.build(pts, nrm)
    f = Fastapss(t, k)
    f.setScalingProtectionSphere(2.0)
    return pts, nrm, diag, k, f


def projector(f):
    def project(centres):
        q = torch.from_numpy(np.ascontiguousarray(centres, np.float32)).cuda()
        p = torch.empty_like(q)
        n = torch.empty_like(q)
        f.project_device(q, p, n, 1, stepMaxSize=FLT_MAX)
        torch.cuda.synchronize()
        return p.cpu().numpy(), n.cpu().numpy()
    return project


@pytest.mark.parametrize("depth,cut", [(4, False), (5, True)])
def test_adaptive_grid_matches_restatement(torus_apss, depth, cut):
    pts, nrm, diag, k, f = torus_apss
    g = DCGrid.adaptive(f, depth, cut=cut)
    total = odg.generate(depth, projector(f))
    cells, nd, no = odg.uniformize(total, depth, cut=cut)
    assert np.array_equal(g.cells, cells)
    want = np.zeros((3, 4), np.float32)
    for a in range(3):
        want[a, a] = 2.0 * nd
        want[a, 3] = 2.0 * no[a] - 1.0
    assert np.array_equal(g.xform, want)
    assert g.n_projected > 0
    # the grid hugs the surface: its deepest cells contain the points
    assert g.max_depth >= depth


def unpaired_fraction(t):
    """Share of directed edges that are repeated or have no opposite (0 for a
    closed, consistently oriented 2-manifold)."""
    directed = Counter()
    for a, b, c in t.tolist():
        for e in ((a, b), (b, c), (c, a)):
            directed[e] += 1
    bad = sum(1 for (a, b), v in directed.items() if v != 1 or directed.get((b, a), 0) != 1)
    return bad / max(1, len(directed))


def test_dc_mesh_on_adaptive_grid_equals_parts(torus_apss):
    """The device extraction on a shifted, projection-driven grid equals the
    host extraction of the same field."""
    pts, nrm, diag, k, f = torus_apss
    g = DCGrid.adaptive(f, 5)
    mesh = f.dc_mesh(g, refine_rounds=1)
    v, n, t = mesh.arrays()
    cf, vx, nc, _ = f.dc_evaluate(g.cells, g.max_depth, g.xform)
    m = Mesh.extract(g.cells, cf, vx)
    m.transform(g.xform)
    m.project(f, 3)
    m.smooth()
    m.subdivide()
    m.project(f, 3)
    pv, pn, pt = m.arrays()
    assert len(t) > 1000
    assert np.array_equal(t, pt) and np.array_equal(v, pv) and np.array_equal(n, pn)
    st = mesh.stage_ms()
    assert st["extract"] > 0 and st["project"] > 0


def test_device_resident_mesh(torus_apss):
    """A dc_mesh result stays in device memory: the mesh functions run there
    (one refinement round by hand equals refine_rounds=1), and the host copy,
    the pinned host copy and the device views agree."""
    pts, nrm, diag, k, f = torus_apss
    g = DCGrid.adaptive(f, 5)
    want = f.dc_mesh(g, refine_rounds=1).arrays()
    m = f.dc_mesh(g, refine_rounds=0)
    assert m.stage_ms()["download"] == 0.0
    m.smooth()
    m.subdivide()
    m.project(f, 3)
    got = m.arrays()
    pinned = m.arrays(pinned=True)
    dv, dn, dt = m.device_arrays()
    for a, b in zip(want, got):
        assert np.array_equal(a, b)
    for a, b in zip(got, pinned):
        assert np.array_equal(a, b)
    assert np.array_equal(dv.cpu().numpy(), got[0]) and np.array_equal(dn.cpu().numpy(), got[1])
    assert np.array_equal(dt.cpu().numpy().view(np.uint32), got[2])
    # a moved transform on the device equals the same map applied to the copy
    xf = np.array([[2, 0, 0, 0.5], [0, 1, 0, -0.25], [0, 0, 0.5, 1]], np.float32)
    m.transform(xf)
    v2 = m.arrays()[0]
    ref = got[0] @ xf[:, :3].T + xf[:, 3]
    assert np.allclose(v2, ref, rtol=0, atol=1e-6)


def test_host_mesh_has_no_device_arrays(torus_apss):
    pts, nrm, diag, k, f = torus_apss
    g = DCGrid(pts, 4)
    cf, vx, nc, _ = f.dc_evaluate(g.cells, g.max_depth, g.xform)
    m = Mesh.extract(g.cells, cf, vx)
    from mlodsurfaces_b200._capi import MlodsError
    with pytest.raises(MlodsError):
        m.device_arrays()


def test_dc_mesh_pipeline(torus_apss):
    pts, nrm, diag, k, f = torus_apss
    g = DCGrid(pts, 5)
    v, n, t = f.dc_mesh(g).arrays()

    # same steps composed from the parts
    cf, vx, nc, _ = f.dc_evaluate(g.cells, g.max_depth, g.xform)
    m = Mesh.extract(g.cells, cf, vx)
    v0, _, t0 = m.arrays()
    m.transform(g.xform)
    m.project(f, 3)
    for _ in range(2):
        m.smooth()
        m.subdivide()
        m.project(f, 3)
    pv, pn, pt = m.arrays()
    assert np.array_equal(t, pt) and np.array_equal(v, pv) and np.array_equal(n, pn)

    # extraction connectivity equals the restatement's on the same corner values
    md = g.max_depth
    values = {}
    for i, (d, x, y, z) in enumerate(g.cells.tolist()):
        s = 1 << (md - d)
        for kk in range(8):
            values[((x + (kk & 1)) * s, (y + ((kk >> 1) & 1)) * s, (z + ((kk >> 2) & 1)) * s)] = cf[i, kk]
    _, order, _, tris = dcmesh.extract(g.cells.tolist(), lambda c: values[tuple(c)], lambda c: None)
    assert np.array_equal(t0.astype(np.int64), np.array(tris, np.int64).reshape(-1, 3))

    # a torus inside the grid gives an (almost everywhere) closed, consistently
    # oriented mesh; dual contouring leaves a few non-manifold spots where a
    # cell holds two sheets, exactly as the reference's extraction does
    frac = unpaired_fraction(t)
    assert len(t) > 1000 and frac < 0.01, frac
    assert len(v) == len(np.unique(t))
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-4)

    # the last projection step: one more 3-iteration projection of the
    # smoothed, subdivided mesh by the FP64 oracle lands within tolerance
    m2 = Mesh.extract(g.cells, cf, vx)
    m2.transform(g.xform)
    m2.project(f, 3)
    for r in range(2):
        m2.smooth()
        m2.subdivide()
        if r == 1:
            before, _, _ = m2.arrays()
        else:
            m2.project(f, 3)
    ot = oracle.OracleTree(pts, nrm, 12)
    o64, _ = ot.project_mlod(before, 3, k, rule=0, cutoff=2.0)
    err = np.linalg.norm(v.astype(np.float64) - o64, axis=1) / diag
    assert err.max() < TOL_DIAG
