"""Projection server: requests mixed across trees, sizes and kernels give the
same results as projecting each request alone; waits are bounded;
admission refuses requests beyond the pending limit; closing with queued
work neither hangs nor leaks."""
import threading

import numpy as np
import pytest

from mlodsurfaces_b200 import APSSOctree, Fastapss, ProjectionServer, synth
from mlodsurfaces_b200 import _capi as capi
from mlodsurfaces_b200._capi import BLEND_CPU, MlodsError
from conftest import make_kernel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def projectors():
    out = []
    for i, (pts, nrm) in enumerate([synth.torus(40000, seed=61), synth.torus_knot(30000, seed=62),
                                    synth.rbf_blobs(20000, seed=63, translate=0.0)]):
        t = APSSOctree()
        t.build(pts, nrm)
        diag = synth.bbox_diag(pts)
        f = Fastapss(t, make_kernel(["gauss", "singular", "multi"][i], diag))
        f.setScalingProtectionSphere([3.0, 2.0, 2.5][i])
        if i == 2:
            f.blend_rule = BLEND_CPU
        out.append((f, pts, diag))
    return out


def direct(f, q, iters, kernel=None):
    """The request projected alone through the reference-facing protocol."""
    if kernel is not None:
        f.updateKernel(kernel)
    f.copyPointsToGPU(len(q), q)
    p = np.empty_like(q)
    n = np.empty_like(q)
    f.project(len(q), p, n, iters)
    return p, n


def make_requests(projectors, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for j in range(count):
        ti = int(rng.integers(0, len(projectors)))
        f, pts, diag = projectors[ti]
        n = int(np.exp(rng.uniform(np.log(50), np.log(20000))))
        q = synth.perturbed_queries(pts, 0.01, seed=1000 + j)[:n]
        iters = int(rng.integers(1, 8))
        kernel = make_kernel(["gauss", "multi", "singular"][j % 3], diag) if j % 4 == 0 else None
        reqs.append((ti, q, iters, kernel))
    return reqs


def expected(projectors, reqs):
    out = []
    for ti, q, iters, kernel in reqs:
        f, pts, diag = projectors[ti]
        p, n = direct(f, q, iters, kernel)
        if kernel is not None:
            restore_kernels(projectors)
        out.append((p, n))
    return out


def restore_kernels(projectors):
    for i, (f, pts, diag) in enumerate(projectors):
        f.updateKernel(make_kernel(["gauss", "singular", "multi"][i], diag))


def test_mixed_requests_equal_projection_alone(projectors):
    reqs = make_requests(projectors, 40, seed=5)
    want = expected(projectors, reqs)
    restore_kernels(projectors)
    srv = ProjectionServer([f for f, _, _ in projectors], n_streams=2, max_batch_queries=60000)
    try:
        tickets = [srv.submit(ti, q, iters, kernel) for ti, q, iters, kernel in reqs]
        for t, (wp, wn) in zip(tickets, want):
            p, n, lat = srv.wait(t, timeout_ms=60000)
            assert np.array_equal(p, wp) and np.array_equal(n, wn)
            assert lat > 0
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["queued"] == 0
        assert st["batches"] < len(reqs)  # requests were batched together
    finally:
        srv.close()


def test_large_requests_run_in_pieces(projectors):
    """With a batch of 4000 queries, requests of up to 20000 run as pieces
    in several batches on both streams while small ones pass them; every
    result is still the request projected alone."""
    reqs = make_requests(projectors, 30, seed=13)
    assert max(len(q) for _, q, _, _ in reqs) > 4000
    want = expected(projectors, reqs)
    restore_kernels(projectors)
    srv = ProjectionServer([f for f, _, _ in projectors], n_streams=2, max_batch_queries=4000)
    try:
        tickets = [srv.submit(ti, q, iters, kernel) for ti, q, iters, kernel in reqs]
        for t, (wp, wn) in zip(tickets, want):
            p, n, lat = srv.wait(t, timeout_ms=60000)
            assert np.array_equal(p, wp) and np.array_equal(n, wn)
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["queued"] == 0
        assert st["queries"] == sum(len(q) for _, q, _, _ in reqs)
        assert st["batches"] > sum(len(q) for _, q, _, _ in reqs) // 4000
    finally:
        srv.close()


def test_concurrent_submitters(projectors):
    reqs = make_requests(projectors, 24, seed=9)
    want = expected(projectors, reqs)
    restore_kernels(projectors)
    srv = ProjectionServer([f for f, _, _ in projectors], n_streams=3)
    results = {}
    errors = []

    def client(idx):
        try:
            for j in idx:
                ti, q, iters, kernel = reqs[j]
                t = srv.submit(ti, q, iters, kernel)
                results[j] = srv.wait(t, timeout_ms=60000)
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    threads = [threading.Thread(target=client, args=(range(k, len(reqs), 4),)) for k in range(4)]
    try:
        for th in threads:
            th.start()
        for th in threads:
            th.join(timeout=120)
        assert not errors and len(results) == len(reqs)
        for j, (wp, wn) in enumerate(want):
            assert np.array_equal(results[j][0], wp) and np.array_equal(results[j][1], wn)
    finally:
        srv.close()


def test_bounded_wait_admission_and_errors(projectors):
    f, pts, diag = projectors[0]
    # room for about 300k queued queries: a request's footprint is its device
    # bytes when it runs plus 36 bytes of pinned staging per query
    budget = ProjectionServer.batch_bytes(300000) + 36 * 300000
    srv = ProjectionServer([f], n_streams=1, max_pending_bytes=budget)
    try:
        q = synth.perturbed_queries(pts, 0.01, seed=77)
        big = np.concatenate([q] * 7)[:280000]
        t = srv.submit(0, big, 10)
        with pytest.raises(TimeoutError):
            srv.wait(t, timeout_ms=0)
        p, n, _ = srv.wait(t, timeout_ms=120000)  # the ticket is still valid after a timeout
        assert np.isfinite(p).all()
        with pytest.raises(MlodsError) as e:
            srv.submit(0, np.concatenate([q] * 8)[:300001], 1)  # beyond max_pending_bytes
        assert e.value.code == capi.MLODS_ERR_CAPACITY
        with pytest.raises(MlodsError):
            srv.wait(987654321)  # unknown ticket
        with pytest.raises(MlodsError):
            srv.submit(5, q[:10], 1)  # no such tree
    finally:
        srv.close()


def test_close_with_queued_work_returns(projectors):
    f, pts, diag = projectors[1]
    srv = ProjectionServer([f], n_streams=1)
    q = synth.perturbed_queries(pts, 0.01, seed=78)
    for _ in range(20):
        srv.submit(0, q, 10)
    srv.close()  # cancels what is queued, finishes the running batch, joins
    srv.close()
    # requests cut into pieces: closing while some of a request's pieces are
    # in flight and the rest are queued waits for those pieces, then returns
    srv = ProjectionServer([f], n_streams=2, max_batch_queries=3000)
    big = np.concatenate([q] * 3)
    for _ in range(6):
        srv.submit(0, big, 10)
    srv.close()


def test_device_budget_bounds_the_batches_in_flight(projectors):
    """Batches are formed within the device budget: with room for only a
    few thousand queries in flight the server still answers every request
    (large ones in pieces, requests waiting for memory to free up), the
    bytes in flight never pass the budget, and results equal the requests
    projected alone."""
    f, pts, diag = projectors[0]
    budget = ProjectionServer.batch_bytes(6000, 8)
    srv = ProjectionServer([f], n_streams=2, max_device_bytes=budget)
    try:
        rng = np.random.default_rng(80)
        q = synth.perturbed_queries(pts, 0.01, seed=80)
        reqs = [q[rng.choice(len(q), int(m), replace=False)] for m in (100, 5000, 17000, 300, 2500, 9000)]
        tickets = [srv.submit(0, r, 6) for r in reqs]
        outs = [srv.wait(t, timeout_ms=120000) for t in tickets]
        mem = srv.memory()
        assert mem["max_device_bytes"] == budget
        assert 0 < mem["peak_in_flight_bytes"] <= budget
        assert mem["in_flight_bytes"] == 0 and mem["pending_bytes"] == 0
        for r, (p, n, _) in zip(reqs, outs):
            want_p = np.empty_like(r)
            want_n = np.empty_like(r)
            f.copyPointsToGPU(len(r), r)
            f.project(len(r), want_p, want_n, 6)
            assert np.array_equal(p, want_p) and np.array_equal(n, want_n)
    finally:
        srv.close()


def test_large_pieces_alone_and_paired_walks(projectors):
    """A piece large enough to fill the GPU many times over runs in a launch
    of its own (the single-tree kernel) beside the shared launch of the
    small ones, with the same results as the requests projected alone.  With
    two queries per warp a request that runs whole is still bit-identical;
    one cut into pieces pairs its queries within each piece, so it agrees
    with the projection alone to float rounding of the moment sums."""
    f, pts, diag = projectors[0]
    q = synth.perturbed_queries(pts, 0.01, seed=81)
    big = np.ascontiguousarray(np.concatenate([q + np.float32(1e-4 * diag * k) for k in range(5)]), np.float32)
    small = q[:3000]
    saved = f.queries_per_warp
    try:
        for qpw in (1, 2):
            f.queries_per_warp = qpw
            want = [direct(f, r, 3) for r in (big, small)]
            srv = ProjectionServer([f], n_streams=1)  # 2^18-query batches: the 200k request runs whole
            try:
                outs = [srv.wait(srv.submit(0, r, 3), timeout_ms=120000) for r in (big, small)]
            finally:
                srv.close()
            for (p, n, _), (wp, wn) in zip(outs, want):
                assert np.array_equal(p, wp) and np.array_equal(n, wn)
        # cut into 60000-query pieces: within the tolerance of the projection alone
        wp, wn = direct(f, big, 3)
        srv = ProjectionServer([f], n_streams=2, max_batch_queries=60000)
        try:
            p, n, _ = srv.wait(srv.submit(0, big, 3), timeout_ms=120000)
        finally:
            srv.close()
        dev = np.linalg.norm(p.astype(np.float64) - wp, axis=1) / diag
        assert dev.max() < 1e-5
        assert ((n * wn).sum(1) > 1 - 1e-4).mean() > 0.999
    finally:
        f.queries_per_warp = saved
