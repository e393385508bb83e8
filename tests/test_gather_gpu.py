"""Neighbour gathers (c) and the APSS projections built on them, against the
oracle and the reference's own kd-tree/APSS results.

kNN sets: exact (same float distance arithmetic as kdTreeNN.h:424) except at
an exact tie between the k-th and (k+1)-th distance.  Projections: within
1e-5 of the bounding-box diagonal."""
import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import APSSOctree, Fastapss, GlobalAPSS, synth
from conftest import TOL_DIAG, golden_kernel, make_kernel, rel_err

pytestmark = pytest.mark.gpu


def tree_of(pts, nrm):
    t = APSSOctree()
    t.build(pts, nrm)
    return t


def assert_knn_sets(pts, q, k, t=None):
    t = t or tree_of(pts, np.tile(np.array([[0, 0, 1]], np.float32), (len(pts), 1)))
    idx, d2 = t.knearest(q, k)
    oi, od, tie = oracle.knn(pts, q, k)
    kk = min(k, len(pts))
    assert np.array_equal(d2[:, :kk].astype(np.float64), od[:, :kk])
    for i in range(len(q)):
        if tie[i]:
            continue
        assert set(idx[i, :kk].tolist()) == set(oi[i, :kk].tolist()), i
    if kk < k:
        assert (idx[:, kk:] == -1).all()
    return idx, d2


@pytest.mark.parametrize("k", [1, 8, 20, 32])
def test_knn_sets_match_bruteforce(k):
    pts, nrm = synth.torus(30000, seed=71)
    q = synth.perturbed_queries(pts, 0.01, seed=72)[:500]
    assert_knn_sets(pts, q, k, tree_of(pts, nrm))


def test_knn_sets_match_reference_kdtree_golden(golden):
    t = tree_of(golden["pts"], golden["nrm"])
    idx, d2 = t.knearest(golden["q"], 32)
    ref = golden["kd_knn32_idx"]
    _, _, tie = oracle.knn(golden["pts"], golden["q"], 32)
    for i in range(len(idx)):
        if not tie[i]:
            assert set(idx[i].tolist()) == set(ref[i].tolist())
    assert np.array_equal(np.sort(d2, 1).astype(np.float64), np.sort(golden["kd_knn32_d2"], 1))


def test_knn_translated_cloud_and_fewer_points_than_k():
    pts, nrm = synth.rbf_blobs(20000, seed=73)
    q = synth.perturbed_queries(pts, 0.01, seed=74)[:300]
    assert_knn_sets(pts, q, 32, tree_of(pts, nrm))
    small = pts[:10]
    assert_knn_sets(small, q[:20], 20)


def apss_gpu(pts, nrm, q, kernel, mode, iters=3, k=32, ball_r=0.1):
    t = tree_of(pts, nrm)
    if mode == "knn":
        t.knnMode(True, k)
    else:
        t.ballMode(True, ball_r)
    f = Fastapss(t, kernel, len(q))
    f.copyPointsToGPU(len(q), q)
    op = np.empty((len(q), 3), np.float32)
    on = np.empty((len(q), 3), np.float32)
    f.project(len(q), op, on, iters, kernel)
    return op, on, t


def test_knn_apss_matches_reference_golden(golden):
    k = golden_kernel(golden, "gauss")
    diag = float(golden["diag"])
    op, on, _ = apss_gpu(golden["pts"], golden["nrm"], golden["q"], k, "knn", iters=3, k=32)
    o64, _ = oracle.project_apss(golden["pts"], golden["nrm"], golden["q"], 3, k, mode=0, k=32,
                                 step_max=float(golden["radius"]))
    assert rel_err(op, o64, diag).max() < TOL_DIAG
    assert rel_err(op, golden["knn32_gauss_p"], diag).max() < TOL_DIAG


def test_ball_apss_matches_reference_golden(golden):
    k = golden_kernel(golden, "gauss")
    diag = float(golden["diag"])
    r = float(golden["ball_r"])
    op, on, _ = apss_gpu(golden["pts"], golden["nrm"], golden["q"], k, "ball", iters=3, ball_r=r)
    o64, _ = oracle.project_apss(golden["pts"], golden["nrm"], golden["q"], 3, k, mode=1, ball_r=r,
                                 step_max=float(golden["radius"]))
    assert rel_err(op, o64, diag).max() < TOL_DIAG
    assert rel_err(op, golden["ball_gauss_p"], diag).max() < TOL_DIAG


@pytest.mark.parametrize("kind", ["multi", "singular"])
def test_knn_apss_matches_oracle(kind):
    pts, nrm = synth.torus(30000, seed=75)
    q = synth.perturbed_queries(pts, 0.01, seed=76)[:400]
    diag = synth.bbox_diag(pts)
    k = make_kernel(kind, diag)
    op, on, t = apss_gpu(pts, nrm, q, k, "knn", iters=5, k=20)
    o64, n64 = oracle.project_apss(pts, nrm, q, 5, k, mode=0, k=20, step_max=t.radius())
    assert rel_err(op, o64, diag).max() < TOL_DIAG


def test_empty_ball_returns_start_point():
    pts, nrm = synth.torus(5000, seed=77)
    k = make_kernel("gauss", synth.bbox_diag(pts))
    q = np.array([[3.0, 3.0, 3.0], [1.35, 0.0, 0.0]], np.float32)
    op, on, _ = apss_gpu(pts, nrm, q, k, "ball", iters=2, ball_r=0.05)
    assert np.array_equal(op[0], q[0]) and np.all(on[0] == 0)
    assert np.linalg.norm(on[1]) > 0.5


def test_global_apss_matches_oracle_and_reference(golden):
    k = golden_kernel(golden, "gauss")
    diag = float(golden["diag"])
    t = tree_of(golden["pts"], golden["nrm"])
    g = GlobalAPSS(t, k)
    q = golden["q"][:100]
    g.copyPointsToGPU(len(q), q)
    op = np.empty((len(q), 3), np.float32)
    on = np.empty((len(q), 3), np.float32)
    g.project(len(q), op, on, 2, k)
    o64, _ = oracle.OracleTree(golden["pts"], golden["nrm"], 12).project_global(q, 2, k)
    assert rel_err(op, o64, diag).max() < TOL_DIAG
    assert rel_err(op, golden["global_gauss_p"], diag).max() < TOL_DIAG


def test_knn_walk_on_a_large_cloud_never_overflows():
    """2M points on the translated RBF surface, k = 32, all 2M queries: the
    walk turns depth-first near its stack capacity, so no query is dropped,
    and sampled results match brute force and the FP64 restatement."""
    pts, nrm = synth.rbf_blobs(2_000_000, seed=2)
    pts = synth.make_tie_free(pts)
    q = synth.perturbed_queries(pts, 0.01, seed=3)
    diag = synth.bbox_diag(pts)
    k = make_kernel("multi", diag)
    t = tree_of(pts, nrm)
    t.knnMode(True, 32)
    f = Fastapss(t, k, len(q))
    f.copyPointsToGPU(len(q), q)
    op = np.empty((len(q), 3), np.float32)
    on = np.empty((len(q), 3), np.float32)
    f.project(len(q), op, on, 3, k)
    assert f.last_stats()["overflows"] == 0
    sel = np.random.default_rng(5).choice(len(q), 48, replace=False)
    o64, _ = oracle.project_apss(pts, nrm, q[sel], 3, k, mode=0, k=32, step_max=t.radius())
    # the cloud sits 1e3 diagonals from the origin: a float32 output is only
    # good to half a unit in the last place there (about 3e-5 diag), so the
    # tolerance applies beyond that rounding
    half_ulp = np.abs(np.spacing(o64.astype(np.float32)).astype(np.float64)) / 2
    excess = np.linalg.norm(np.maximum(np.abs(op[sel].astype(np.float64) - o64) - half_ulp, 0.0), axis=1) / diag
    assert excess.max() < TOL_DIAG
    assert_knn_sets(pts, q[sel], 32, t)


def test_global_apss_split_and_fused_forms():
    """Few queries take the split form (point ranges summed by separate
    blocks, then added in order), many queries the one-launch form; both
    match the FP64 restatement and each other."""
    pts, nrm = synth.torus(20000, seed=91)
    diag = synth.bbox_diag(pts)
    k = make_kernel("multi", diag)
    q = synth.perturbed_queries(np.tile(pts, (31, 1)), 0.01, seed=92)  # 620k queries: the one-launch form
    t = tree_of(pts, nrm)
    g = GlobalAPSS(t, k)
    import torch

    d_q = torch.from_numpy(q).cuda()
    d_p = torch.empty_like(d_q)
    d_n = torch.empty_like(d_q)
    g.project_device(d_q, d_p, d_n, 2)
    full = d_p.cpu().numpy()
    few = q[:300]
    d_q2 = torch.from_numpy(np.ascontiguousarray(few)).cuda()
    d_p2 = torch.empty_like(d_q2)
    d_n2 = torch.empty_like(d_q2)
    g.project_device(d_q2, d_p2, d_n2, 2)
    split = d_p2.cpu().numpy()
    ot = oracle.OracleTree(pts, nrm, 12)
    o64, _ = ot.project_global(few[:64], 2, k)
    assert rel_err(split[:64], o64, diag).max() < TOL_DIAG
    assert rel_err(full[:64], o64, diag).max() < TOL_DIAG
    assert rel_err(split, full[:300], diag).max() < TOL_DIAG
    sel = np.random.default_rng(3).choice(len(q), 64, replace=False)
    o64b, _ = ot.project_global(q[sel], 2, k)
    assert rel_err(full[sel], o64b, diag).max() < TOL_DIAG


@pytest.mark.parametrize("k", [32, 20])
def test_knn_iterations_in_one_call_equal_one_call_per_iteration(k):
    """Inside one call the kNN iteration i > 0 either keeps the k points of
    iteration i - 1, when the step provably leaves them the k nearest, or
    searches from a bound on the (k+1)-th distance taken from iteration i - 1
    (its k points and one other at their new distances, or the (k+1)-th
    distance grown by the step); one call per iteration searches every time
    from the points around the query's Morton position.  The neighbour sets,
    and so the projections, are the same bit for bit, and most later
    iterations keep their neighbours."""
    pts, nrm = synth.rbf_blobs(300_000, seed=7)
    pts = synth.make_tie_free(pts)
    q = synth.perturbed_queries(pts, 0.01, seed=8)[:20000]
    kern = make_kernel("multi", synth.bbox_diag(pts))
    t = tree_of(pts, nrm)
    t.knnMode(True, k)
    f = Fastapss(t, kern, len(q))
    iters = 8
    f.copyPointsToGPU(len(q), q)
    one = np.empty((len(q), 3), np.float32)
    one_n = np.empty((len(q), 3), np.float32)
    f.project(len(q), one, one_n, iters, kern)
    searches = f.last_stats()["iterations"]
    assert len(q) <= searches < len(q) * iters // 2
    f.copyPointsToGPU(len(q), q)
    step = np.empty((len(q), 3), np.float32)
    step_n = np.empty((len(q), 3), np.float32)
    for i in range(iters):
        last = i == iters - 1
        f.project(len(q), step if last else None, step_n if last else None, 1, kern)
        assert f.last_stats()["iterations"] == len(q)
    assert np.array_equal(one, step) and np.array_equal(one_n, step_n)


def test_cpu_sphere_matches_the_reference():
    """APSSOctree.cpuSphere (CPUUtils.cpp:638-663): the sphere fitted to the
    20 nearest samples, against the reference's own on its kd-tree."""
    pts, nrm = synth.torus(20000, seed=93)
    q = synth.perturbed_queries(pts, 0.01, seed=94)[:50]
    k = make_kernel("gauss", synth.bbox_diag(pts))
    t = tree_of(pts, nrm)
    got = np.array([[u0, *u123, u4] for u0, u123, u4 in (t.cpuSphere(x, k) for x in q)], np.float32)
    ref_u = oracle.RefTree(pts, nrm, 12).cpu_sphere(q, k, 20)
    assert np.allclose(got, ref_u, rtol=2e-3, atol=2e-3 * np.abs(ref_u).max(axis=0))
