"""Device octree build (a) against the oracle and the reference golden tree:
topology, breadth-first order and leaf point lists bit-exact; moments and
areas to float precision."""
import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import APSSOctree, synth
from test_oracle import TREE_KEYS

pytestmark = pytest.mark.gpu


def build(pts, nrm, depth=12):
    t = APSSOctree()
    t.build(pts, nrm, maxDepth=depth)
    return t


def assert_same_tree(dev, ora):
    for k in TREE_KEYS:
        assert np.array_equal(dev[k], ora[k]), k
    assert np.array_equal(dev["bmin"], ora["bmin"])
    assert np.array_equal(dev["bmax"], ora["bmax"])


def assert_moments_close(dev, ora, rtol=2e-6):
    """Moments agree to float precision on their physical scales: mass and
    normal sums against the largest node mass, centroids against the box
    extent, cpn against mass x extent, cpp against mass x extent^2."""
    m = ora["mom"]
    # a single point has a zero-extent box: area 0, centroid 0/0 in the
    # reference, the oracle and the device alike
    same_nan = np.isnan(dev["mom"]) & np.isnan(m)
    assert np.array_equal(np.isnan(dev["mom"]), np.isnan(m))
    m = np.where(same_nan, 0.0, m)
    dev = dict(dev, mom=np.where(same_nan, 0.0, dev["mom"]))
    M = float(np.abs(m[:, 0]).max()) or 1.0
    ext = float(np.abs(ora["bmax"][0] - ora["bmin"][0]).max()) or 1.0
    origin = float(np.abs(ora["bmax"][0] + ora["bmin"][0]).max()) / 2
    d = np.abs(dev["mom"] - m)
    assert d[:, [0, 4, 5, 6]].max() <= rtol * M, d[:, [0, 4, 5, 6]].max() / M
    assert d[:, 1:4].max() <= rtol * ext + 1e-7 * origin, d[:, 1:4].max()
    assert d[:, 7].max() <= rtol * M * ext, d[:, 7].max() / (M * ext)
    assert d[:, 8].max() <= rtol * M * ext * ext, d[:, 8].max() / (M * ext * ext)


def test_golden_reference_tree(golden):
    t = build(golden["pts"], golden["nrm"])
    ex = t.export()
    for k in TREE_KEYS:
        assert np.array_equal(ex[k], golden["tree_" + k]), k
    assert t.nbOfNodes() == len(golden["tree_parent"])
    assert t.computeDepth() == int(golden["depth_ref"])
    assert t.numTies() == 0
    assert np.abs(ex["area"] - golden["tree_area"]).max() <= 1e-6 * golden["tree_area"].max()


@pytest.mark.parametrize("n,depth,seed", [(1, 12, 1), (2, 12, 2), (3, 12, 3), (100, 12, 4), (20000, 12, 5),
                                          (20000, 6, 6), (5000, 0, 7), (60000, 12, 8)])
def test_torus_trees_match_oracle(n, depth, seed):
    pts, nrm = synth.torus(n, seed=seed)
    pts = synth.make_tie_free(pts, depth=max(depth, 1))
    t = build(pts, nrm, depth)
    o = oracle.OracleTree(pts, nrm, depth)
    dev, ora = t.export(), o.export()
    assert t.nbOfNodes() == o.n_nodes
    assert_same_tree(dev, ora)
    assert_moments_close(dev, ora)
    assert np.allclose(dev["area"], ora["area"], rtol=1e-6, atol=0)


def test_translated_blobs_tree_matches_oracle():
    pts, nrm = synth.rbf_blobs(30000, seed=9)
    pts = synth.make_tie_free(pts)
    t = build(pts, nrm)
    o = oracle.OracleTree(pts, nrm, 12)
    dev, ora = t.export(), o.export()
    assert_same_tree(dev, ora)
    # centroids of a cloud 5e3 away from the origin still agree to float precision
    assert np.abs(dev["mom"][:, 1:4] - ora["mom"][:, 1:4]).max() < 1e-3
    assert np.allclose(dev["mom"][:, 0], ora["mom"][:, 0], rtol=1e-5)


def test_duplicates_make_multi_point_leaves():
    rng = np.random.default_rng(0)
    base = rng.uniform(-1, 1, (500, 3)).astype(np.float32)
    pts = np.concatenate([base, base[:50], base[:10], base[:3]])
    nrm = np.tile(np.array([[0, 0, 1]], np.float32), (len(pts), 1))
    for depth in (12, 4):
        t = build(pts, nrm, depth)
        o = oracle.OracleTree(pts, nrm, depth)
        dev, ora = t.export(), o.export()
        assert_same_tree(dev, ora)
        assert dev["leaf_cnt"].max() >= 4 if depth == 12 else True
        assert_moments_close(dev, ora)


def test_exact_split_ties_go_low_and_are_counted():
    # x = 0.5 is exactly the first split of [0, 1]
    pts = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.5, 0.25, 0.75], [0.5, 0.8, 0.1]], np.float32)
    nrm = np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))
    t = build(pts, nrm)
    o = oracle.OracleTree(pts, nrm, 12)
    assert t.numTies() > 0 and o.n_ties > 0
    assert_same_tree(t.export(), o.export())


def test_device_build_from_torch_tensors():
    torch = pytest.importorskip("torch")
    pts, nrm = synth.torus(5000, seed=21)
    pts = synth.make_tie_free(pts)
    t = APSSOctree()
    t.build_device(torch.from_numpy(pts).cuda(), torch.from_numpy(nrm).cuda())
    o = oracle.OracleTree(pts, nrm, 12)
    assert_same_tree(t.export(), o.export())


def test_invalid_inputs_are_rejected():
    from mlodsurfaces_b200._capi import MlodsError

    t = APSSOctree()
    with pytest.raises(ValueError):
        t.build(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32))
    with pytest.raises(MlodsError):
        t.build(np.zeros((4, 3), np.float32), np.zeros((4, 3), np.float32), maxDepth=13)
    bad = np.zeros((4, 3), np.float32)
    bad[1, 0] = np.nan
    with pytest.raises(MlodsError):
        t.build(bad, np.zeros((4, 3), np.float32))
