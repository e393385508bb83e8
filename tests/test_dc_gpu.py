"""DC corner field and per-cell vertex (d) against the FP64 oracle.

Field: same NaN pattern, values within 1e-5 of the tree's box diagonal, so
signs agree wherever |f| exceeds that; vertex: the reference's zero-normal
QEF (mass point of the crossings) evaluated from the same corner values."""
import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import APSSOctree, DCGrid, Fastapss, synth, unit2bbox
from conftest import TOL_DIAG, make_kernel

pytestmark = pytest.mark.gpu


def unique_corners(cells, max_depth):
    d = cells[:, 0].astype(np.int64)
    delta = (np.int64(1) << (max_depth - d))[:, None]
    bits = np.array([[k & 1, (k >> 1) & 1, (k >> 2) & 1] for k in range(8)], np.int64)
    lat = (cells[:, None, 1:4].astype(np.int64) + bits[None]) * delta[:, :, None]
    return lat  # (n, 8, 3)


def world_of(lat, max_depth):
    w = np.float32(1.0) / np.float32(1 << max_depth)
    u = (lat.astype(np.float32) * w).astype(np.float32)
    m = unit2bbox()
    out = np.empty(u.shape, np.float32)
    for r in range(3):
        out[..., r] = (((m[r, 0] * u[..., 0]).astype(np.float32) + (m[r, 1] * u[..., 1]).astype(np.float32))
                       .astype(np.float32) + (m[r, 2] * u[..., 2]).astype(np.float32)).astype(np.float32) + m[r, 3]
    return out


@pytest.fixture(scope="module")
def dc_setup():
    pts, nrm = synth.torus(20000, seed=81)
    pts = synth.make_tie_free(synth.normalize_like_pn(pts))
    diag = synth.bbox_diag(pts)
    k = make_kernel("singular", diag)
    t = APSSOctree()
    t.build(pts, nrm)
    f = Fastapss(t, k)
    f.setScalingProtectionSphere(2.0)
    g = DCGrid(pts, 6)
    return pts, nrm, diag, k, f, g


def test_corner_field_matches_oracle(dc_setup):
    pts, nrm, diag, k, f, g = dc_setup
    cf, vx, nc, nu = f.dc_evaluate(g.cells, g.max_depth)
    lat = unique_corners(g.cells, g.max_depth)
    flat = lat.reshape(-1, 3)
    uniq, inv = np.unique(flat, axis=0, return_inverse=True)
    assert nu == len(uniq)
    wc = world_of(uniq, g.max_depth)
    ot = oracle.OracleTree(pts, nrm, 12)
    xp, xn = ot.project_mlod(wc, 1, k, rule=0, cutoff=2.0)
    f64 = np.empty(len(wc))
    wc64 = np.ascontiguousarray(wc.astype(np.float64))  # named: must outlive the call
    oracle.orc().orc_dc_field(oracle._ptr(wc64), oracle._ptr(xp), oracle._ptr(xn), len(wc), oracle._ptr(f64))
    ref = f64[inv.reshape(-1)].reshape(-1, 8)
    assert np.array_equal(np.isnan(cf), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert np.abs(cf[ok] - ref[ok]).max() < TOL_DIAG * diag
    strong = ok & (np.abs(ref) > TOL_DIAG * diag)
    assert np.array_equal(cf[strong] < 0, ref[strong] < 0)


def test_vertices_follow_the_zero_normal_qef(dc_setup):
    pts, nrm, diag, k, f, g = dc_setup
    cf, vx, nc, _ = f.dc_evaluate(g.cells, g.max_depth)
    assert nc.max() > 0
    for ci in np.random.default_rng(0).choice(len(g.cells), 400, replace=False):
        d, x, y, z = g.cells[ci]
        width = 1.0 / (1 << d)
        lo = np.array([x, y, z], np.float64) * width
        out = np.empty(3)
        cnt = np.zeros(1, np.int32)
        vals = np.ascontiguousarray(cf[ci].astype(np.float64))
        oracle.orc().orc_dc_vertex(oracle._ptr(lo), width, oracle._ptr(vals), oracle._ptr(out), oracle._ptr(cnt))
        assert nc[ci] == cnt[0]
        assert np.abs(vx[ci] - out).max() <= 1e-6 * width + 1e-7


def test_qef_with_normals_stays_in_its_cell(dc_setup):
    pts, nrm, diag, k, f, g = dc_setup
    cf, vx, nc, _ = f.dc_evaluate(g.cells, g.max_depth, use_normals=True)
    width = 1.0 / (np.int64(1) << g.cells[:, 0].astype(np.int64))
    lo = g.cells[:, 1:4] * width[:, None]
    act = nc > 0
    eps = 1e-6
    assert np.isfinite(vx).all()
    assert ((vx[act] >= lo[act] - eps) & (vx[act] <= lo[act] + width[act, None] + eps)).all()


def test_device_buffers_give_the_host_results(dc_setup):
    """mlods_dc_evaluate_device: cells and results in device memory, the
    same values as the host-buffer call, on two calls in a row (the second
    reuses the library's pooled scratch)."""
    import torch

    from mlodsurfaces_b200._capi import MlodsError

    pts, nrm, diag, k, f, g = dc_setup
    want = f.dc_evaluate(g.cells, g.max_depth)
    d_cells = torch.from_numpy(np.ascontiguousarray(g.cells, np.int32)).cuda()
    for _ in range(2):
        cf, vx, nc, nu = f.dc_evaluate_device(d_cells, g.max_depth)
        torch.cuda.synchronize()
        assert nu == want[3]
        assert np.array_equal(cf.cpu().numpy(), want[0], equal_nan=True)
        assert np.array_equal(vx.cpu().numpy(), want[1]) and np.array_equal(nc.cpu().numpy(), want[2])
    # cells deeper than max_depth or off the lattice are refused on the device path too
    bad = d_cells.clone()
    bad[7, 0] = g.max_depth + 1
    with pytest.raises(MlodsError):
        f.dc_evaluate_device(bad, g.max_depth)
    bad = d_cells.clone()
    bad[3, 1] = 1 << 30
    with pytest.raises(MlodsError):
        f.dc_evaluate_device(bad, g.max_depth)
    # and the host path still works after a refusal, and after the pooled
    # scratch went back to the system
    from mlodsurfaces_b200 import _capi as capi

    capi.check(capi.load().mlods_release_scratch())
    again = f.dc_evaluate(g.cells, g.max_depth)
    assert np.array_equal(again[0], want[0], equal_nan=True)
