"""The dual-contouring path against the reference's OWN code (oracle/_ref/
libmlods_refdc.so: scene/upsample.cpp, dual-contouring/octree.h and
dual_contouring.h compiled from the reference sources, plus a restatement of
the glue of scene::computeDualContouring).

The reference code asks for every projection through a callback, which the
tests answer with this library's projection of the same tree, so the grid
generation, the corner field, the extraction (minimal-edge order, vertex
numbering, triangles, mass-point vertices) and the refinement loop (smooth,
subdivide, project) are compared bit for bit with the library's device
implementations."""
import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import APSSOctree, DCGrid, Fastapss, Mesh, synth
from conftest import make_kernel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.refdc_available(), reason="reference DC checker not built")]
torch = pytest.importorskip("torch")


def ref_projector(f):
    """Answers the reference code's projections with the library's: APSS::project
    (GPU blend rule, the tree's kernel and options) or APSS::projectCPU."""
    calls = {"project": 0, "projectCPU": 0}

    def project(pts, iters, step_max, cpu_rule):
        if cpu_rule:
            calls["projectCPU"] += 1
            return f.projectCPU(pts, iters, stepMaxSize=step_max)
        calls["project"] += 1
        q = torch.from_numpy(np.ascontiguousarray(pts, np.float32)).cuda()
        p = torch.empty_like(q)
        n = torch.empty_like(q)
        f.project_device(q, p, n, iters, stepMaxSize=step_max)
        torch.cuda.synchronize()
        return p.cpu().numpy(), n.cpu().numpy()

    project.calls = calls
    return project


@pytest.fixture(scope="module", params=["singular", "multi"])
def apss(request):
    pts, nrm = synth.torus(30000, seed=71)
    pts = synth.make_tie_free(synth.normalize_like_pn(pts))
    diag = synth.bbox_diag(pts)
    t = APSSOctree()
    t.build(pts, nrm)
    f = Fastapss(t, make_kernel(request.param, diag))
    f.setScalingProtectionSphere(2.0)
    return pts, f


@pytest.mark.parametrize("depth,cut", [(4, False), (5, False), (6, True)])
def test_adaptive_grid_equals_reference_generate_uniformize(apss, depth, cut):
    pts, f = apss
    proj = ref_projector(f)
    ref = oracle.RefDCGrid.adaptive(proj, depth, cut=cut)
    g = DCGrid.adaptive(f, depth, cut=cut)
    assert proj.calls["project"] > 0 and proj.calls["projectCPU"] == 0
    assert np.array_equal(ref.cells(), g.cells)
    assert ref.max_depth == g.max_depth
    assert np.array_equal(ref.xform(), g.xform.ravel())


def _check_mesh(f, g, ref_grid, refine_rounds):
    proj = ref_projector(f)
    ref = ref_grid.mesh(proj, refine_rounds)
    assert proj.calls["projectCPU"] == 0  # every corner value came from the precomputed map
    cells = g.cells
    # corner field: one value per corner slot, NaN where the projection failed
    cf, vx, nc, _ = f.dc_evaluate(cells, g.max_depth, g.xform)
    md = g.max_depth
    d = cells[:, 0:1]
    corner = np.array([[(c >> 0) & 1, (c >> 1) & 1, (c >> 2) & 1] for c in range(8)], np.int32)
    keys = ((cells[:, None, 1:] + corner[None]) << (md - d)[:, :, None]).reshape(-1, 3)
    assert np.array_equal(keys, ref["corner_keys"])
    rv = ref["corner_vals"]
    ov = cf.reshape(-1)
    assert np.array_equal(np.isnan(rv), np.isnan(ov))
    ok = ~np.isnan(rv)
    assert np.array_equal(rv[ok].view(np.uint32), ov[ok].view(np.uint32))
    # extraction: the reference's vertices (unit frame) and triangles
    m = Mesh.extract(cells, cf, vx)
    v0, _, t0 = m.arrays()
    assert len(t0) > 100
    assert np.array_equal(ref["ext_indices"].reshape(-1, 3), t0)
    assert np.array_equal(ref["ext_vertices"], v0)
    # whole pipeline on the device: transform, project, smooth, subdivide
    v, n, t = f.dc_mesh(g, refine_rounds=refine_rounds).arrays()
    assert np.array_equal(ref["indices"].reshape(-1, 3), t)
    assert np.array_equal(ref["vertices"], v)
    assert np.array_equal(ref["normals"], n)


def test_mesh_on_adaptive_grid_equals_reference(apss):
    pts, f = apss
    g = DCGrid.adaptive(f, 5)
    _check_mesh(f, g, oracle.RefDCGrid.adaptive(ref_projector(f), 5), refine_rounds=2)


def test_mesh_on_points_grid_equals_reference(apss):
    pts, f = apss
    g = DCGrid(pts, 5)
    ref_grid = oracle.RefDCGrid.from_points(pts, 5)
    assert np.array_equal(ref_grid.cells(), g.cells)
    _check_mesh(f, g, ref_grid, refine_rounds=1)


def test_points_grid_on_device_equals_reference_at_depth_9():
    """The -b grid of the dual-contouring workload's cloud shape at its depth,
    on the device, against the reference's generateFromPoints + uniformize."""
    pts, _ = synth.torus_knot(400000, seed=4)
    pts = synth.normalize_like_pn(pts)
    ref = oracle.RefDCGrid.from_points(pts, 9)
    g = DCGrid(torch.from_numpy(pts).cuda(), 9)
    assert np.array_equal(ref.cells(), g.cells)
