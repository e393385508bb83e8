"""Query generation in octree cells (scene::generateFromOctree,
scene.cpp:733-756) on the device, bit-exact against a numpy restatement of
the same draws and the reference's float cell geometry
(aabb_octree::bounds / center, octree.h:939-955)."""
import numpy as np
import pytest
import torch

from mlodsurfaces_b200 import io
from mlodsurfaces_b200._capi import MlodsError

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def draw(seed, i, k):
    return mix64((seed + 0x9E3779B97F4A7C15 * (i * 4 + k + 1)) & M64)


def restated(cells, n, seed):
    cells = np.asarray(cells, np.int64).reshape(-1, 4)
    out = np.empty((n, 3), np.float32)
    for i in range(n):
        c = cells[(draw(seed, i, 0) * len(cells)) >> 64]
        d = int(c[0])
        w = np.float32(2.0) / np.float32(1 << d)
        move = np.float32(4.0) / np.float32(1 << d)
        for a in range(3):
            lo = np.float32(-1.0) + w * np.float32(c[1 + a])
            hi = np.float32(-1.0) + w * np.float32(c[1 + a] + 1)
            centre = (lo + hi) / np.float32(2.0)
            r = np.float32(draw(seed, i, a + 1) >> 40) * np.float32(1.0 / 16777216.0) - np.float32(0.5)
            out[i, a] = centre + r * move
    return out


def random_cells(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.integers(0, 10, n)
    pos = (rng.random((n, 3)) * (1 << d)[:, None]).astype(np.int64)
    return np.concatenate([d[:, None], pos], 1).astype(np.int32)


@pytest.mark.parametrize("seed", [0, 12345, 2**63 + 7])
def test_matches_restatement(seed):
    cells = random_cells(300, 31)
    p, nrm = io.sample_cells(cells, 3000, seed=seed)
    torch.cuda.synchronize()
    p = p.cpu().numpy()
    assert np.array_equal(p, restated(cells, 3000, seed))
    assert np.array_equal(nrm.cpu().numpy(), p)  # the normal is the point


def test_points_stay_in_the_doubled_cell_and_cells_are_uniform():
    cells = random_cells(64, 32)
    n = 400_000
    p, _ = io.sample_cells(cells, n, seed=9)
    p = p.cpu().numpy().astype(np.float64)
    # which cell produced each point is the first draw; recompute it
    pick = np.array([(draw(9, i, 0) * len(cells)) >> 64 for i in range(0, n, 997)])
    sub = p[::997]
    c = cells[pick].astype(np.float64)
    side = 2.0 / (1 << c[:, 0].astype(np.int64))
    centre = -1.0 + side[:, None] * (c[:, 1:] + 0.5)
    assert (np.abs(sub - centre) <= side[:, None] + 1e-6).all()
    counts = np.bincount(pick, minlength=len(cells))
    expected = len(pick) / len(cells)
    assert ((counts - expected) ** 2 / expected).sum() < 3 * len(cells)  # chi-square, 63 dof


def test_bad_arguments():
    cells = torch.zeros((4, 4), dtype=torch.int32, device="cuda")
    with pytest.raises(MlodsError):
        io.sample_cells(cells[:0], 10)
    p, _ = io.sample_cells(torch.tensor([[40, 0, 0, 0]], dtype=torch.int32), 4)
    assert torch.isnan(p).all()
    p, _ = io.sample_cells(cells, 0)
    assert p.shape == (0, 3)
