"""Batched projection over several resident trees (one launch) against
per-tree launches: results must be identical bit for bit, with and without
CUDA-graph replay and after launch-shape tuning."""
import ctypes as C

import numpy as np
import pytest

from mlodsurfaces_b200 import APSSOctree, Fastapss, FastapssBatch, synth
from mlodsurfaces_b200 import _capi as capi
from mlodsurfaces_b200._capi import BLEND_CPU, MlodsError
from conftest import make_kernel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _setup():
    clouds = [
        synth.torus(30000, seed=41),
        synth.rbf_blobs(20000, seed=42),
        synth.torus_knot(25000, seed=43),
        synth.torus(500, seed=44),
    ]
    projectors, queries = [], []
    for i, (pts, nrm) in enumerate(clouds):
        t = APSSOctree()
        t.build(pts, nrm, maxDepth=12)
        diag = synth.bbox_diag(pts)
        f = Fastapss(t)
        f.copyToGPU(make_kernel(["gauss", "multi", "singular", "multi"][i], diag))
        f.setScalingProtectionSphere([3.0, 2.0, 3.0, 2.5][i])
        if i == 1:
            f.blend_rule = BLEND_CPU
        if i == 2:
            f.setMinDepth(2)
        projectors.append(f)
        n_q = [4000, 0, 3000, 700][i]
        queries.append(synth.perturbed_queries(pts, 0.01, seed=50 + i)[:n_q])
    return projectors, queries


@pytest.fixture(scope="module")
def setup():
    return _setup()


def _per_tree(projectors, queries, iters):
    outs_p, outs_n = [], []
    for f, q in zip(projectors, queries):
        if len(q) == 0:
            continue
        d_q = torch.from_numpy(q).cuda()
        d_p = torch.empty_like(d_q)
        d_n = torch.empty_like(d_q)
        f.project_device(d_q, d_p, d_n, iters)
        outs_p.append(d_p)
        outs_n.append(d_n)
    torch.cuda.synchronize()
    return torch.cat(outs_p), torch.cat(outs_n)


def _batched(b, queries, iters, use_graph=False, out=None):
    counts = [len(q) for q in queries]
    d_q = torch.from_numpy(np.concatenate(queries)).cuda()
    d_p = torch.full_like(d_q, float("nan")) if out is None else out[0]
    d_n = torch.full_like(d_q, float("nan")) if out is None else out[1]
    b.project_device(counts, d_q, d_p, d_n, iters, use_graph=use_graph)
    torch.cuda.synchronize()
    return d_p, d_n, d_q


def test_batch_equals_per_tree_launches(setup):
    projectors, queries = setup
    ref_p, ref_n = _per_tree(projectors, queries, 6)
    b = FastapssBatch(projectors)
    p, n, _ = _batched(b, queries, 6)
    assert torch.equal(p, ref_p) and torch.equal(n, ref_n)
    st = b.last_stats()
    assert st["overflows"] == 0 and st["node_visits"] > 0 and st["kernel_ms"] > 0


def test_graph_replay_and_tuning(setup):
    projectors, queries = setup
    ref_p, ref_n = _per_tree(projectors, queries, 4)
    b = FastapssBatch(projectors)
    counts = [len(q) for q in queries]
    d_q = torch.from_numpy(np.concatenate(queries)).cuda()
    d_p = torch.empty_like(d_q)
    d_n = torch.empty_like(d_q)
    lib = capi.load()
    for _ in range(3):
        d_p.fill_(float("nan"))
        before = lib.mlods_kernel_launches()
        b.project_device(counts, d_q, d_p, d_n, 4, use_graph=True)
        torch.cuda.synchronize()
        assert lib.mlods_kernel_launches() > before  # each replay counts its kernels
        assert torch.equal(d_p, ref_p) and torch.equal(d_n, ref_n)
    b.tune(counts, d_q, d_p, d_n, 4)
    st = b.last_stats()
    assert st["grid_pct"] in (85, 100) and st["reorder"] in (0, 1)
    assert st["queries_per_warp"] in (1, 2)
    cands = b.tune_results()
    assert len(cands) == 7 and all(c["ms"] > 0 for c in cands)
    best = min(cands, key=lambda c: c["ms"])
    keys = ("queries_per_warp", "reorder", "grid_pct", "line_order", "solo_min_queries")
    assert all(best[k] == st[k] for k in keys)
    d_p.fill_(float("nan"))
    b.project_device(counts, d_q, d_p, d_n, 4, use_graph=True)
    torch.cuda.synchronize()
    # the tuner's schedule applies to every tree: per-tree launches with the
    # same schedule (and the tuned query order) give the same bits
    saved = [f.queries_per_warp for f in projectors]
    saved_order = [f.reorder for f in projectors]
    try:
        for f in projectors:
            f.queries_per_warp = st["queries_per_warp"]
            f.reorder = bool(st["reorder"])
        tuned_p, tuned_n = _per_tree(projectors, queries, 4)
    finally:
        for f, w, r in zip(projectors, saved, saved_order):
            f.queries_per_warp = w
            f.reorder = r
    assert torch.equal(d_p, tuned_p) and torch.equal(d_n, tuned_n)
    # a change of iteration count re-captures
    try:
        for f in projectors:
            f.queries_per_warp = st["queries_per_warp"]
            f.reorder = bool(st["reorder"])
        ref2_p, _ = _per_tree(projectors, queries, 2)
    finally:
        for f, w, r in zip(projectors, saved, saved_order):
            f.queries_per_warp = w
            f.reorder = r
    b.project_device(counts, d_q, d_p, d_n, 2, use_graph=True)
    torch.cuda.synchronize()
    assert torch.equal(d_p, ref2_p)


@pytest.mark.parametrize("by_spec,solo,reorder", [(False, 0, True), (True, 0, True), (True, 1000, True),
                                                   (False, 1000, False)])
def test_batch_with_paired_walks_equals_per_tree(setup, by_spec, solo, reorder):
    """Trees set to two queries per warp: the single launch pairs the same
    queries as each tree's own launch (each tree's slots are padded to a
    multiple of 4), whatever the order of the trees along the launch; trees
    with at least `solo` queries run in launches of their own on their slice
    of the batch order."""
    projectors, queries = setup
    saved = [f.queries_per_warp for f in projectors]
    saved_order = [f.reorder for f in projectors]
    try:
        for f in projectors:
            f.queries_per_warp = 2
            f.reorder = reorder
        ref_p, ref_n = _per_tree(projectors, queries, 5)
        b = FastapssBatch(projectors)
        b.set_schedule(0, reorder, 100, by_specialisation=by_spec, solo_min_queries=solo)
        p, n, _ = _batched(b, queries, 5, use_graph=bool(solo))
        st = b.last_stats()
        assert st["line_order"] == ("by specialisation" if by_spec else "most work first")
        assert st["solo_min_queries"] == solo
        # two trees hold >= 1000 queries (4000 and 3000), one fewer (700), one none
        assert st["walk_launches"] == (3 if solo else 1)
    finally:
        for f, w, r in zip(projectors, saved, saved_order):
            f.queries_per_warp = w
            f.reorder = r
    assert torch.equal(p, ref_p) and torch.equal(n, ref_n)


def test_batch_rejects_bad_input(setup):
    projectors, queries = setup
    b = FastapssBatch(projectors)
    d_q = torch.zeros((10, 3), device="cuda")
    with pytest.raises(ValueError):
        b.project_device([1, 2], d_q, d_q, d_q, 1)
    with pytest.raises(MlodsError):
        b.project_device([0, 0, 0, 0], d_q, d_q, d_q, 1)  # no queries at all
    lib = capi.load()
    off = np.array([1, 2, 3, 4, 5], np.int64)  # offsets[0] != 0
    rc = lib.mlods_batch_project(b._b, capi.ptr(off), capi.ptr(d_q), capi.ptr(d_q), capi.ptr(d_q), 1, 0,
                                 C.c_void_p(0))
    assert rc == capi.MLODS_ERR_INVALID
    off = np.array([0, 5, 3, 6, 8], np.int64)  # decreasing
    rc = lib.mlods_batch_project(b._b, capi.ptr(off), capi.ptr(d_q), capi.ptr(d_q), capi.ptr(d_q), 1, 0,
                                 C.c_void_p(0))
    assert rc == capi.MLODS_ERR_INVALID
    with pytest.raises(MlodsError):
        b.set_schedule(queries_per_warp=3)
    with pytest.raises(MlodsError):
        b.set_schedule(grid_pct=0)
    with pytest.raises(MlodsError):
        b.set_schedule(solo_min_queries=-1)
    g = Fastapss(projectors[0].m_apssOctree)
    g.m_apssOctree.knnMode(True, 8)
    try:
        with pytest.raises(ValueError):
            FastapssBatch([g])
    finally:
        g.m_apssOctree.knnMode(False)
