"""MLoD projection kernel (b) against the FP64 oracle (both blend rules, all
three weight kernels) and against the reference's own CPU results.

Bar: projected points within 1e-5 of the bounding-box diagonal of the FP64
oracle; normals within 1e-4 in direction."""
import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import APSSOctree, Fastapss, synth
from mlodsurfaces_b200._capi import BLEND_CPU, BLEND_GPU, CONVERGE_EXACT, CONVERGE_OFF, CONVERGE_TOL, MlodsError
from conftest import TOL_DIAG, golden_kernel, make_kernel, rel_err

pytestmark = pytest.mark.gpu


def excess_err(x, x64, diag):
    """Distance to the FP64 result beyond float32 output rounding, / diag."""
    x = np.asarray(x, np.float64)
    x64 = np.asarray(x64, np.float64)
    half_ulp = np.abs(np.spacing(x64.astype(np.float32)).astype(np.float64)) / 2
    e = np.maximum(np.abs(x - x64) - half_ulp, 0.0)
    return np.linalg.norm(e, axis=1) / diag


def run_gpu(pts, nrm, q, kernel, iters=10, cutoff=3.0, rule=BLEND_GPU, min_depth=0, reorder=True, step_max=-1.0,
            depth=12, converge=CONVERGE_OFF, converge_tol=0.0):
    t = APSSOctree()
    t.build(pts, nrm, maxDepth=depth)
    f = Fastapss(t)
    f.copyToGPU(kernel, len(q))
    f.setScalingProtectionSphere(cutoff)
    f.setMinDepth(min_depth)
    f.blend_rule = rule
    f.reorder = reorder
    f.converge = converge
    f.converge_tol = converge_tol
    f.copyPointsToGPU(len(q), q)
    op = np.empty((len(q), 3), np.float32)
    on = np.empty((len(q), 3), np.float32)
    f.project(len(q), op, on, iters, kernel, step_max)
    return op, on, f.last_stats(), t


@pytest.fixture(scope="module")
def torus20k():
    pts, nrm = synth.torus(20000, seed=31)
    pts = synth.make_tie_free(pts)
    q = synth.perturbed_queries(pts, 0.01, seed=32)[:1500]
    return pts, nrm, q, oracle.OracleTree(pts, nrm, 12)


@pytest.mark.parametrize("kind", ["gauss", "multi", "singular"])
@pytest.mark.parametrize("rule", [BLEND_GPU, BLEND_CPU])
def test_projection_matches_fp64_oracle(torus20k, kind, rule):
    pts, nrm, q, ot = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel(kind, diag)
    op, on, st, _ = run_gpu(pts, nrm, q, k, rule=rule)
    rp, rn = ot.project_mlod(q, 10, k, rule=rule, cutoff=3.0)
    err = rel_err(op, rp, diag)
    assert err.max() < TOL_DIAG, (err.max(), np.percentile(err, 99))
    ok = np.linalg.norm(rn, axis=1) > 0.5
    assert ((on[ok] * rn[ok]).sum(1) > 1 - 1e-4).all()
    assert st["overflows"] == 0 and st["node_visits"] > 0


@pytest.mark.parametrize("name", ["gauss", "multi", "singular"])
def test_cpu_rule_matches_reference_golden(golden, name):
    k = golden_kernel(golden, name)
    diag = float(golden["diag"])
    op, _, _, _ = run_gpu(golden["pts"], golden["nrm"], golden["q"], k, rule=BLEND_CPU)
    ref_p = golden[f"mlod_{name}_p"]
    err = rel_err(op, ref_p, diag)
    # where the reference's own float solve is accurate (FP64 oracle within
    # 5e-6 diag of it), the kernel agrees with the reference within 1e-5 diag
    ot = oracle.OracleTree(golden["pts"], golden["nrm"], 12)
    o64, _ = ot.project_mlod(golden["q"], 10, k, rule=1, cutoff=3.0)
    ref_ok = rel_err(o64, ref_p, diag) < 5e-6
    assert ref_ok.mean() > 0.98
    assert err[ref_ok].max() < TOL_DIAG, err[ref_ok].max()
    assert rel_err(op, o64, diag).max() < TOL_DIAG


def test_translated_cloud_matches_fp64_beyond_output_rounding():
    pts, nrm = synth.rbf_blobs(30000, seed=41)
    pts = synth.make_tie_free(pts)
    q = synth.perturbed_queries(pts, 0.01, seed=42)[:800]
    diag = synth.bbox_diag(pts)
    k = make_kernel("multi", diag)
    op, on, st, _ = run_gpu(pts, nrm, q, k)
    rp, rn = oracle.OracleTree(pts, nrm, 12).project_mlod(q, 10, k, rule=0, cutoff=3.0)
    assert excess_err(op, rp, diag).max() < TOL_DIAG
    ok = np.linalg.norm(rn, axis=1) > 0.5
    assert ((on[ok] * rn[ok]).sum(1) > 1 - 1e-4).all()


def test_min_depth_and_step_clamp(torus20k):
    pts, nrm, q, ot = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel("gauss", diag)
    op, _, _, _ = run_gpu(pts, nrm, q[:300], k, iters=3, min_depth=4, step_max=0.002)
    rp, _ = ot.project_mlod(q[:300], 3, k, rule=0, cutoff=3.0, min_depth=4, step_max=0.002)
    assert rel_err(op, rp, diag).max() < TOL_DIAG
    # each step is clamped to 0.002; every iterate is rounded to float (as the
    # reference stores it), which adds up to about one ulp (1.2e-7 here) per step
    assert (np.linalg.norm(op.astype(np.float64) - q[:300], axis=1) <= 3 * 0.002 + 4e-7).all()


def test_far_queries_and_single_query(torus20k):
    pts, nrm, _, ot = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel("singular", diag)
    q = np.array([[5.0, 5.0, 5.0], [0.0, 0.0, 3.0], [1.3, 0.0, 0.0]], np.float32)
    op, _, _, _ = run_gpu(pts, nrm, q, k, iters=4)
    rp, _ = ot.project_mlod(q, 4, k, rule=0, cutoff=3.0)
    assert rel_err(op, rp, diag).max() < TOL_DIAG
    op1, _, _, _ = run_gpu(pts, nrm, q[2:3], k, iters=4)
    assert np.array_equal(op1[0], op[2])


def test_reorder_is_bit_identical(torus20k):
    pts, nrm, q, _ = torus20k
    k = make_kernel("multi", synth.bbox_diag(pts))
    a, an, _, _ = run_gpu(pts, nrm, q, k, reorder=True)
    b, bn, _, _ = run_gpu(pts, nrm, q, k, reorder=False)
    assert np.array_equal(a, b) and np.array_equal(an, bn)


@pytest.mark.parametrize("kind", ["gauss", "multi"])
def test_exact_convergence_is_bit_identical_and_cheaper(torus20k, kind):
    pts, nrm, q, _ = torus20k
    k = make_kernel(kind, synth.bbox_diag(pts))
    a, an, sa, _ = run_gpu(pts, nrm, q, k, iters=30)
    b, bn, sb, _ = run_gpu(pts, nrm, q, k, iters=30, converge=CONVERGE_EXACT)
    assert np.array_equal(a, b) and np.array_equal(an, bn)
    assert sb["node_visits"] < sa["node_visits"]


def test_tolerance_convergence_stays_within_tolerance(torus20k):
    pts, nrm, q, ot = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel("gauss", diag)
    tol = 1e-7 * diag
    b, bn, sb, _ = run_gpu(pts, nrm, q, k, iters=10, converge=CONVERGE_TOL, converge_tol=tol)
    rp, _ = ot.project_mlod(q, 10, k, rule=BLEND_GPU, cutoff=3.0)
    assert rel_err(b, rp, diag).max() < TOL_DIAG
    _, _, sa, _ = run_gpu(pts, nrm, q, k, iters=10)
    assert sb["node_visits"] < sa["node_visits"]
    # every query counts the iterations it evaluated
    assert sa["iterations"] == 10 * len(q)
    assert len(q) <= sb["iterations"] < sa["iterations"]


def test_in_place_protocol_continues_from_last_positions(torus20k):
    pts, nrm, q, _ = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel("gauss", diag)
    t = APSSOctree()
    t.build(pts, nrm)
    f = Fastapss(t, k, len(q))
    f.setScalingProtectionSphere(3.0)
    f.copyPointsToGPU(len(q), q)
    out = np.empty((len(q), 3), np.float32)
    nrmo = np.empty((len(q), 3), np.float32)
    for _ in range(10):  # ten timer ticks of one iteration, as scene::projectPoints
        f.project(len(q), None, None, 1, k)
    f.project(len(q), out, nrmo, 0, k)
    full, _, _, _ = run_gpu(pts, nrm, q, k, iters=10)
    assert rel_err(out, full, diag).max() < TOL_DIAG


def test_nan_query_fails_in_band(torus20k):
    pts, nrm, q, _ = torus20k
    k = make_kernel("gauss", synth.bbox_diag(pts))
    qq = q[:64].copy()
    qq[5] = np.nan
    op, on, _, _ = run_gpu(pts, nrm, qq, k, iters=2)
    assert np.all(on[5] == 0)
    good, _, _, _ = run_gpu(pts, nrm, q[:64], k, iters=2)
    mask = np.ones(64, bool)
    mask[5] = False
    assert np.array_equal(op[mask], good[mask])


def test_protocol_errors(torus20k):
    pts, nrm, q, _ = torus20k
    t = APSSOctree()
    t.build(pts[:1000], nrm[:1000])
    f = Fastapss(t)
    with pytest.raises(MlodsError):
        f.project(10, None, None, 1)  # no kernel, no queries
    f.copyToGPU(make_kernel("gauss", 1.0))
    with pytest.raises(MlodsError):
        f.project(10, None, None, 1)  # no queries uploaded
    f.copyPointsToGPU(10, q[:10])
    with pytest.raises(MlodsError):
        f.project(11, None, None, 1)  # more than uploaded
    f.project(10, None, None, 1)


TINY = {
    "one point": [[0.1, 0.2, 0.3]],
    "two points": [[0, 0, 0], [1, 0.5, 0.25]],
    "three points": [[0, 0, 0], [1, 0, 0], [0, 1, 0]],
    "coincident points": [[0.3, 0.3, 0.3]] * 3,
}


@pytest.mark.parametrize("name", list(TINY))
@pytest.mark.parametrize("rule", [BLEND_GPU, BLEND_CPU])
def test_tiny_clouds(name, rule):
    """Clouds of one to three points: a degenerate fit fails in band (the
    query stays, normal zero) exactly where the oracle's does, otherwise the
    projection matches it.  Coincident points build a multi-point leaf (the
    reference draws a random side for them, CPUUtils.cpp:299-308)."""
    pts = np.array(TINY[name], np.float32)
    nrm = np.tile(np.array([[0, 0, 1]], np.float32), (len(pts), 1))
    q = np.array([[0.2, 0.1, 0.5], [0.5, 0.5, -0.3], [0.1, 0.2, 0.3]], np.float32)
    from mlodsurfaces_b200 import Kernel

    k = Kernel()
    k.type = Kernel.GAUSSIAN
    k.sigma = 0.5
    op, on, _, _ = run_gpu(pts, nrm, q, k, iters=3, cutoff=2.0, rule=rule)
    x64, n64 = oracle.OracleTree(pts, nrm, 12).project_mlod(q, 3, k, rule=rule, cutoff=2.0)
    failed64 = np.all(n64 == 0, axis=1)
    failed = np.all(on == 0, axis=1)
    assert np.array_equal(failed, failed64)
    assert np.array_equal(op[failed], q[failed])
    scale = max(float(np.ptp(pts, axis=0).max()), 1.0)
    assert np.abs(op[~failed] - x64[~failed]).max(initial=0.0) < TOL_DIAG * scale


@pytest.mark.parametrize("kind", ["gauss", "multi", "singular"])
@pytest.mark.parametrize("rule", [BLEND_GPU, BLEND_CPU])
@pytest.mark.parametrize("qpw", [2, 4])
def test_paired_walk_matches_fp64_and_single_walk(torus20k, kind, rule, qpw):
    """Two or four queries per warp: each query's arithmetic is its own
    walk's, only the order of the float sums changes -- FP64 within 1e-5
    diag, and the one-query walk within float rounding of the moments; the
    same query-node visits."""
    pts, nrm, q, ot = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel(kind, diag)
    t = APSSOctree()
    t.build(pts, nrm)
    outs = {}
    for w in (1, qpw):
        f = Fastapss(t)
        f.copyToGPU(k, len(q))
        f.setScalingProtectionSphere(3.0)
        f.blend_rule = rule
        f.queries_per_warp = w
        f.copyPointsToGPU(len(q), q)
        op = np.empty((len(q), 3), np.float32)
        on = np.empty((len(q), 3), np.float32)
        f.project(len(q), op, on, 10, k)
        outs[w] = (op, on, f.last_stats())
    rp, rn = ot.project_mlod(q, 10, k, rule=rule, cutoff=3.0)
    op2, on2, st2 = outs[qpw]
    assert rel_err(op2, rp, diag).max() < TOL_DIAG
    assert rel_err(op2, outs[1][0], diag).max() < 1e-6
    ok = np.linalg.norm(rn, axis=1) > 0.5
    assert ((on2[ok] * rn[ok]).sum(1) > 1 - 1e-4).all()
    assert st2["overflows"] == 0
    assert st2["node_visits"] == outs[1][2]["node_visits"]  # query-node visits: the reference's walk


def test_schedule_tuner_picks_a_timed_schedule(torus20k):
    """mlods_tune_schedule times the 1, 2 and 4 queries-per-warp walks on the
    caller's queries and keeps the fastest; projections with it stay within
    1e-5 diag of FP64."""
    torch = pytest.importorskip("torch")
    pts, nrm, q, ot = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel("multi", diag)
    t = APSSOctree()
    t.build(pts, nrm)
    f = Fastapss(t, k)
    f.setScalingProtectionSphere(3.0)
    d_q = torch.from_numpy(q).cuda()
    res = f.tune_schedule(d_q, 10)
    assert res["queries_per_warp"] in (1, 2, 4)
    assert all(m > 0 for m in res["ms"].values())
    assert res["ms"][res["queries_per_warp"]] == min(res["ms"].values())
    assert f.queries_per_warp == res["queries_per_warp"]
    d_p = torch.empty_like(d_q)
    d_n = torch.empty_like(d_q)
    f.project_device(d_q, d_p, d_n, 10)
    torch.cuda.synchronize()
    rp, _ = ot.project_mlod(q, 10, k, rule=0, cutoff=3.0)
    assert rel_err(d_p.cpu().numpy(), rp, diag).max() < TOL_DIAG


def test_kernel_weight_pruning_is_bounded_and_off_by_default(torus20k):
    """prune_tol = 0 is the reference's walk (bit-identical to no option);
    a small tolerance drops subtrees that can weigh almost nothing: fewer or
    equal visits, results within 1e-5 diag of FP64."""
    torch = pytest.importorskip("torch")
    pts, nrm, q, ot = torus20k
    diag = synth.bbox_diag(pts)
    k = make_kernel("gauss", diag)
    t = APSSOctree()
    t.build(pts, nrm)
    d_q = torch.from_numpy(q).cuda()
    out = {}
    for tol in (0.0, 1e-6, 1e-3):
        f = Fastapss(t, k)
        f.setScalingProtectionSphere(3.0)
        f.prune_tol = tol
        d_p = torch.empty_like(d_q)
        d_n = torch.empty_like(d_q)
        f.project_device(d_q, d_p, d_n, 10)
        torch.cuda.synchronize()
        out[tol] = (d_p.cpu().numpy(), f.last_stats())
    base = Fastapss(t, k)
    base.setScalingProtectionSphere(3.0)
    d_p = torch.empty_like(d_q)
    d_n = torch.empty_like(d_q)
    base.project_device(d_q, d_p, d_n, 10)
    torch.cuda.synchronize()
    assert np.array_equal(out[0.0][0], d_p.cpu().numpy()) and out[0.0][1]["pruned"] == 0
    rp, _ = ot.project_mlod(q, 10, k, rule=0, cutoff=3.0)
    for tol in (1e-6, 1e-3):
        p, st = out[tol]
        assert st["node_visits"] <= out[0.0][1]["node_visits"]
        assert rel_err(p, rp, diag).max() < TOL_DIAG
    assert out[1e-3][1]["pruned"] > 0
