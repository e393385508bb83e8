"""Point-set and parameter files (host code of the library): PLY / PN round
trips, PLY variants (ascii, big endian, extra properties and elements),
Pn::normalize against a float32 restatement, and the .params layout against
the reference's own parameter files."""
import json
import struct
from pathlib import Path

import numpy as np
import pytest

from mlodsurfaces_b200 import io, synth
from mlodsurfaces_b200._capi import MlodsError

GOLDEN = Path(__file__).parent / "golden" / "params_reference.json"


def normalize_restated(p):
    """Pn::normalize (Pn.cpp:262-290), float32, sequential sums."""
    p = np.asarray(p, np.float32)
    off = p[0].copy()
    mx = p[0].copy()
    mn = p[0].copy()
    for i in range(1, len(p)):
        off = (off + p[i]).astype(np.float32)
        mx = np.maximum(p[i], mx)
        mn = np.minimum(p[i], mn)
    off = (off / np.float32(len(p))).astype(np.float32)
    mx = (mx - off).astype(np.float32)
    mn = (mn - off).astype(np.float32)
    dd = (mx - mn).astype(np.float32)
    d2 = np.float32(0)
    for a in range(3):
        d2 = np.float32(d2 + np.float32(dd[a] * dd[a]))
    small = np.float32(np.float32(np.sqrt(d2)) * np.float32(0.005))
    mx = (mx + small).astype(np.float32)
    mn = (mn - small).astype(np.float32)
    norme = np.float32(max(abs(mx[0]), abs(mx[1]), abs(mx[2]), abs(mn[0]), abs(mn[1]), abs(mn[2])))
    return ((p - off).astype(np.float32) / norme).astype(np.float32), off, float(norme)


def test_normalize_matches_restatement():
    pts, _ = synth.torus(3000, seed=3)
    pts = (pts * 37.5 + np.float32(1000.25)).astype(np.float32)
    out, off, norme = io.normalize(pts)
    r_out, r_off, r_norme = normalize_restated(pts)
    assert np.array_equal(off, r_off) and norme == r_norme
    assert np.array_equal(out, r_out)
    assert np.abs(out).max() <= 1.0


@pytest.mark.parametrize("ext", ["ply", "pn"])
def test_round_trip(tmp_path, ext):
    pts, nrm = synth.torus(2000, seed=4)
    pts = (pts * 3.0 + 5.0).astype(np.float32)
    path = tmp_path / f"cloud.{ext}"
    npts, off, norme = io.normalize(pts)
    io.save_cloud(path, npts, nrm, off, norme)  # writes p * norme + offset
    raw, rn, roff, rnorme = io.load_cloud(path, normalize=False)
    assert np.array_equal(raw, (npts * np.float32(norme) + off).astype(np.float32))
    assert np.array_equal(rn, nrm)
    assert roff.tolist() == [0, 0, 0] and rnorme == 1.0
    back, _, loff, lnorme = io.load_cloud(path, normalize=True)
    r_back, r_off, r_norme = normalize_restated(raw)
    assert np.array_equal(back, r_back) and np.array_equal(loff, r_off) and lnorme == r_norme


def test_ply_header_written_like_the_reference(tmp_path):
    pts = np.arange(12, dtype=np.float32).reshape(4, 3)
    io.save_cloud(tmp_path / "a.ply", pts)
    head = (tmp_path / "a.ply").read_bytes()
    assert head.startswith(b"ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\n"
                           b"property float y\nproperty float z\nend_header\n")
    assert len(head) == len(b"ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\n"
                            b"property float y\nproperty float z\nend_header\n") + 48
    p, n, _, _ = io.load_cloud(tmp_path / "a.ply", normalize=False)
    assert np.array_equal(p, pts) and n is None


def test_ply_variants(tmp_path):
    pts = np.array([[0.5, -1.25, 2.0], [3.0, 4.5, -6.0], [7.0, 8.0, 9.5]], np.float32)
    nrm = np.array([[1, 0, 0], [0, 1, 0], [0, 0, -1]], np.float32)
    # ascii with an extra colour property and a face element after the vertices
    lines = ["ply", "format ascii 1.0", "comment test", "element vertex 3", "property double x",
             "property double y", "property double z", "property uchar red", "property float nx",
             "property float ny", "property float nz", "element face 1", "property list uchar int vertex_index",
             "end_header"]
    body = [f"{p[0]} {p[1]} {p[2]} 200 {n[0]} {n[1]} {n[2]}" for p, n in zip(pts, nrm)] + ["3 0 1 2"]
    (tmp_path / "a.ply").write_text("\n".join(lines + body) + "\n")
    p, n, _, _ = io.load_cloud(tmp_path / "a.ply", normalize=False)
    assert np.array_equal(p, pts) and np.array_equal(n, nrm)
    # big endian, an element before the vertices, int16 extras
    hdr = ("ply\nformat binary_big_endian 1.0\nelement camera 1\nproperty float view\nproperty list uchar int ids\n"
           "element vertex 3\nproperty float x\nproperty short tag\nproperty float y\nproperty float z\n"
           "end_header\n").encode()
    data = struct.pack(">fBii", 1.5, 2, 7, 8)
    for i, q in enumerate(pts):
        data += struct.pack(">fhff", q[0], i, q[1], q[2])
    (tmp_path / "b.ply").write_bytes(hdr + data)
    p, n, _, _ = io.load_cloud(tmp_path / "b.ply", normalize=False)
    assert np.array_equal(p, pts) and n is None


def test_bad_files(tmp_path):
    (tmp_path / "x.ply").write_text("not a ply\n")
    with pytest.raises(MlodsError):
        io.load_cloud(tmp_path / "x.ply")
    (tmp_path / "y.ply").write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 10\n"
                                     b"property float x\nproperty float y\nproperty float z\nend_header\n" + b"\0" * 20)
    with pytest.raises(MlodsError):
        io.load_cloud(tmp_path / "y.ply")  # truncated
    with pytest.raises(MlodsError):
        io.load_cloud(tmp_path / "missing.pn")
    with pytest.raises(MlodsError):
        io.load_cloud(tmp_path / "z.xyz")


def test_reference_params_files(tmp_path):
    """The reference's own .params files decode to the fields
    scene::loadParameters reads, and write back byte for byte."""
    golden = json.loads(GOLDEN.read_text())
    assert len(golden) >= 5
    for name, entry in golden.items():
        raw = bytes.fromhex(entry["hex"])
        assert len(raw) == 134
        path = tmp_path / f"{name}.params"
        path.write_bytes(raw)
        got = io.load_params(path)
        for key, want in entry["fields"].items():
            if isinstance(want, list):
                assert np.allclose(got[key], want, rtol=0, atol=0), (name, key)
            else:
                assert got[key] == pytest.approx(want, rel=0, abs=0), (name, key)
        io.save_params(tmp_path / "again.params", got)
        assert (tmp_path / "again.params").read_bytes() == raw
        k = io.kernel_from_params(got, radius=2.0)
        assert k.type == got["kernel_type"]
        if got["computed_sigma"]:
            assert len(k.sigmas) == got["n_computed_sigmas"]
            assert k.sigmas[0] == pytest.approx(2.0 * got["beginning_sigma"], rel=1e-6)
    with pytest.raises(MlodsError):
        (tmp_path / "short.params").write_bytes(b"\0" * 100)
        io.load_params(tmp_path / "short.params")


def morton_restated(p, grid=64):
    """Pn::order's codes (Pn.cpp:388-440) and a stable sort."""
    p = np.asarray(p, np.float32)
    lo = np.float32(min(p[:, 0].min(), p[:, 1].min(), p[:, 2].min()))
    hi = np.float32(max(p[:, 0].max(), p[:, 1].max(), p[:, 2].max()))
    norme = np.float32(hi - lo)
    t = np.floor((((p - lo).astype(np.float32) / norme).astype(np.float32) * np.float32(grid)).astype(np.float32))
    c = np.clip(t, 0, grid - 1).astype(np.uint64)
    code = np.zeros(len(p), np.uint64)
    for b in range(6):
        code |= ((c[:, 1] >> b) & 1) << (3 * b) | ((c[:, 0] >> b) & 1) << (3 * b + 1) | ((c[:, 2] >> b) & 1) << (3 * b + 2)
    return np.argsort(code, kind="stable")


def test_morton_order_matches_restatement():
    pts, _ = synth.torus(20000, seed=8)
    perm = io.morton_order(pts)
    assert np.array_equal(perm.astype(np.int64), morton_restated(pts))
    assert sorted(perm.tolist()) == list(range(len(pts)))


def test_sample_around_stays_on_tangent_disks():
    pts, nrm = synth.torus(5000, seed=9)
    q, qn = io.sample_around(pts, nrm, 3000, factor=1.0, seed=3)
    gap = 2.0 * np.cbrt(np.pi / len(pts))
    # every query is within meanGap of some input point, in that point's tangent plane
    from scipy.spatial import cKDTree
    d, k = cKDTree(pts).query(q)
    assert d.max() <= gap * 1.0001
    q2, _ = io.sample_around(pts, nrm, 3000, factor=1.0, seed=3)
    assert np.array_equal(q, q2)  # seeded
    assert np.allclose(np.linalg.norm(qn, axis=1), 1.0, atol=1e-5)
