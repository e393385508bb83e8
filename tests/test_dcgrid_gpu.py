"""The points-driven DC grid with its set work on the device
(mlods_dcgrid_from_points_device) against the host version and the Python
restatement of OctreeGenerator::generateFromPoints + uniformizeFromPoints."""
import numpy as np
import pytest

from mlodsurfaces_b200 import DCGrid, synth
from oracle import dcgrid as odg

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_small_grid_matches_restatement():
    pts, _ = synth.torus(2000, seed=51)
    pts = synth.normalize_like_pn(pts)
    g = DCGrid(pts, 5, device=True)
    want = odg.grid_from_points(pts, 5)
    assert np.array_equal(g.cells, want)


@pytest.mark.parametrize("depth", [4, 7, 9])
def test_device_grid_equals_host_grid(depth):
    pts, _ = synth.torus_knot(300_000, seed=4)
    pts = synth.normalize_like_pn(pts)
    dev = DCGrid(pts, depth, device=True)
    host = DCGrid(pts, depth, device=False)
    assert dev.max_depth == host.max_depth == depth
    assert np.array_equal(dev.cells, host.cells)
    assert np.array_equal(dev.xform, host.xform)
    # from a CUDA tensor too
    on_gpu = DCGrid(torch.from_numpy(pts).cuda(), depth)
    assert np.array_equal(on_gpu.cells, host.cells)


def test_points_beyond_the_keys_fall_back_to_the_host():
    pts, _ = synth.torus(5000, seed=52)
    pts = synth.normalize_like_pn(pts)
    far = np.concatenate([pts, np.array([[3e6, 0.0, 0.0]], np.float32)])  # cell index far beyond 2^19
    dev = DCGrid(far, 6, device=True)
    host = DCGrid(far, 6, device=False)
    assert np.array_equal(dev.cells, host.cells)
    deep_dev = DCGrid(pts, 16, device=True)  # deeper than the device keys
    deep_host = DCGrid(pts, 16, device=False)
    assert np.array_equal(deep_dev.cells, deep_host.cells)
