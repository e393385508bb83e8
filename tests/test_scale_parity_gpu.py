"""Parity at the full sizes of the benchmark configurations (seeded synthetic
clouds with the configurations' shapes, sizes and value distributions):

* precision configuration: 2M-point 12-blob RBF surface translated 1e3 x diag,
  multi-Gaussian kernel, 10 iterations -- the device octree equals the
  reference's own tree (APSSOctree::build compiled from its sources) and the
  FP64 restatement's, node for node; 65,536 queries against the FP64
  restatement, in world coordinates beyond float32 output rounding (the
  output itself rounds by up to ~5e-5 diag that far from the origin) and in
  the tree's local frame (local_output), both within 1e-5 diag;
* the same data with APSS over the 32 nearest neighbours;
* torus configuration: 100k points, single Gaussian, CPU blend rule,
  queries = the points -- tree equal to the reference's, every query within
  1e-5 diag of FP64;
* dual-contouring configuration: 5M-point torus knot with holes, rational
  kernel, projection-driven grid at depth 9 -- on a 1M-corner sample the
  field has the FP64 restatement's NaN pattern, values within 1e-5 diag and
  identical signs wherever |f| > 1e-5 diag."""
import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import APSSOctree, DCGrid, Fastapss, Kernel, synth
from mlodsurfaces_b200._capi import BLEND_CPU, BLEND_GPU
from conftest import TOL_DIAG, make_kernel, rel_err

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOPOLOGY = ("depth", "parent", "first_child", "n_children", "next_brother", "leaf_off", "leaf_cnt", "perm")


def excess_err(x, x64, diag):
    x = np.asarray(x, np.float64)
    half_ulp = np.abs(np.spacing(x64.astype(np.float32)).astype(np.float64)) / 2
    return np.linalg.norm(np.maximum(np.abs(x - x64) - half_ulp, 0.0), axis=1) / diag


def assert_same_tree(t, pts, nrm):
    ex = t.export()
    ot = oracle.OracleTree(pts, nrm, 12).export()
    for k in TOPOLOGY + ("bmin", "bmax"):
        assert np.array_equal(ex[k], ot[k]), k
    if oracle.ref_available():
        rt = oracle.RefTree(pts, nrm, 12).export()
        for k in TOPOLOGY + ("bmin", "bmax"):
            assert np.array_equal(ex[k], rt[k]), k


def project_all(t, k, q, rule, cutoff, iters=10, local=False):
    f = Fastapss(t, k)
    f.setScalingProtectionSphere(cutoff)
    f.blend_rule = rule
    f.local_output = local
    d_q = torch.from_numpy(q).cuda()
    d_p = torch.empty_like(d_q)
    d_n = torch.empty_like(d_q)
    f.project_device(d_q, d_p, d_n, iters)
    torch.cuda.synchronize()
    return d_p.cpu().numpy(), d_n.cpu().numpy(), f


@pytest.fixture(scope="module")
def precision():
    pts, nrm = synth.rbf_blobs(2_000_000, seed=2)
    pts = synth.make_tie_free(pts)
    q = synth.perturbed_queries(pts, 0.01, seed=3)
    diag = synth.bbox_diag(pts)
    k = Kernel()
    k.type = Kernel.GAUSSIAN_MULTIPLE
    k.sigmas = [0.01 * diag * 2.0**i for i in range(4)]
    t = APSSOctree()
    t.build(pts, nrm)
    return pts, nrm, q, diag, k, t


def test_precision_tree_equals_reference(precision):
    pts, nrm, q, diag, k, t = precision
    assert t.numTies() == 0
    assert_same_tree(t, pts, nrm)


def test_precision_error_vs_fp64_world_and_local(precision):
    pts, nrm, q, diag, k, t = precision
    world, wn, _ = project_all(t, k, q, BLEND_GPU, 3.0)
    local, _, _ = project_all(t, k, q, BLEND_GPU, 3.0, local=True)
    sel = np.random.default_rng(7).choice(len(q), 65536, replace=False)
    x64, n64 = oracle.OracleTree(pts, nrm, 12).project_mlod(q[sel], 10, k, rule=0, cutoff=3.0)
    origin = np.array(t.info().origin[:], np.float64)
    ew = excess_err(world[sel], x64, diag)
    el = np.linalg.norm(local[sel].astype(np.float64) - (x64 - origin), axis=1) / diag
    print(f"\nprecision 2M, 65536 queries vs FP64 / diag: world beyond f32 rounding max {ew.max():.3e} "
          f"p99 {np.percentile(ew, 99):.3e}; local frame max {el.max():.3e} p99 {np.percentile(el, 99):.3e}")
    assert ew.max() < TOL_DIAG
    assert el.max() < TOL_DIAG
    ok = np.linalg.norm(n64, axis=1) > 0.5
    assert ((wn[sel][ok] * n64[ok]).sum(1) > 1 - 1e-4).all()


def test_precision_knn32_error_vs_fp64(precision):
    pts, nrm, q, diag, k, t = precision
    f = Fastapss(t, k)
    t.knnMode(True, 32)
    try:
        sel = np.random.default_rng(8).choice(len(q), 384, replace=False)
        qs = np.ascontiguousarray(q[sel])
        d_q = torch.from_numpy(qs).cuda()
        d_p = torch.empty_like(d_q)
        d_n = torch.empty_like(d_q)
        f.project_device(d_q, d_p, d_n, 10)
        torch.cuda.synchronize()
        x64, _ = oracle.project_apss(pts, nrm, qs, 10, k, 0, k=32, step_max=float(t.radius()))
    finally:
        t.knnMode(False)
    e = excess_err(d_p.cpu().numpy(), x64, diag)
    print(f"\nkNN=32, 384 queries vs FP64 / diag beyond f32 rounding: max {e.max():.3e} p99 {np.percentile(e, 99):.3e}")
    assert e.max() < TOL_DIAG


def test_torus_tree_and_every_query_vs_fp64():
    pts, nrm = synth.torus(100_000, seed=1)
    pts = synth.make_tie_free(pts)
    diag = synth.bbox_diag(pts)
    k = make_kernel("gauss", diag)
    t = APSSOctree()
    t.build(pts, nrm)
    assert_same_tree(t, pts, nrm)
    out, _, _ = project_all(t, k, pts, BLEND_CPU, 3.0)
    x64, _ = oracle.OracleTree(pts, nrm, 12).project_mlod(pts, 10, k, rule=1, cutoff=3.0)
    e = rel_err(out, x64, diag)
    print(f"\ntorus 100k, all queries vs FP64 / diag: max {e.max():.3e} p99 {np.percentile(e, 99):.3e}")
    assert e.max() < TOL_DIAG


def test_dc_workload_field_signs_vs_fp64():
    pts, nrm = synth.torus_knot(5_000_000, seed=4)
    pts = synth.make_tie_free(synth.normalize_like_pn(pts))
    diag = synth.bbox_diag(pts)
    k = make_kernel("singular", diag)
    t = APSSOctree()
    t.build(pts, nrm)
    f = Fastapss(t, k)
    f.setScalingProtectionSphere(2.0)
    g = DCGrid.adaptive(f, 9)
    assert len(g.cells) > 4_000_000
    cf, _, _, n_unique = f.dc_evaluate(g.cells, g.max_depth, g.xform)
    # the lattice corner of every slot, and one slot per unique corner
    md = g.max_depth
    bits = np.array([[c & 1, (c >> 1) & 1, (c >> 2) & 1] for c in range(8)], np.int64)
    d = g.cells[:, 0].astype(np.int64)
    lat = ((g.cells[:, None, 1:].astype(np.int64) + bits[None]) << (md - d)[:, None, None]).reshape(-1, 3)
    b = lat + (1 << 20)  # grade may add cells just outside the grid's root box (negative positions)
    assert b.min() >= 0 and b.max() < (1 << 21)
    key = (b[:, 0] << 42) | (b[:, 1] << 21) | b[:, 2]
    _, first = np.unique(key, return_index=True)
    assert len(first) == n_unique
    sel = np.random.default_rng(9).choice(first, min(1_000_000, len(first)), replace=False)
    # corner position as the library maps it: u = lattice * 2^-md, then the grid's map
    w = np.float32(1.0) / np.float32(1 << md)
    u = lat[sel].astype(np.float32) * w
    xf = g.xform
    wc = np.empty_like(u)
    for r in range(3):
        wc[:, r] = (xf[r, r] * u[:, r]).astype(np.float32) + xf[r, 3]
    x64, n64 = oracle.OracleTree(pts, nrm, 12).project_mlod(wc, 1, k, rule=0, cutoff=2.0)
    f64 = np.empty(len(wc))
    wc64 = np.ascontiguousarray(wc.astype(np.float64))
    oracle.orc().orc_dc_field(oracle._ptr(wc64), oracle._ptr(x64), oracle._ptr(n64), len(wc), oracle._ptr(f64))
    ours = cf.reshape(-1)[sel]
    assert np.array_equal(np.isnan(ours), np.isnan(f64))
    ok = ~np.isnan(f64)
    dev = np.abs(ours[ok] - f64[ok]) / diag
    strong = ok & (np.abs(f64) > TOL_DIAG * diag)
    agree = np.mean((ours[strong] < 0) == (f64[strong] < 0))
    print(f"\nDC depth 9, {len(sel)} unique corners of {n_unique}: |f - f64| / diag max {dev.max():.3e}, "
          f"sign agreement where |f| > 1e-5 diag: {agree:.6f} over {strong.sum()} corners")
    assert dev.max() < TOL_DIAG
    assert agree == 1.0
