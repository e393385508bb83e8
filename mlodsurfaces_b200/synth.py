"""Seeded synthetic point clouds for the parity tests and the benchmark.

The reference ships no benchmark data for its projection path; these
generators produce oriented clouds with the shapes, sizes and noise levels of
the workloads the benchmark is quoted on:

* :func:`torus` -- uniform-by-area torus (R, r) with analytic normals.
* :func:`rbf_blobs` -- zero level set of sum_j exp(-|x-c_j|^2/rho_j^2) - tau,
  Newton-projected samples, normals from the analytic gradient, optionally
  translated far from the origin.
* :func:`torus_knot` -- a (p, q) torus-knot tube with spherical holes.
* :func:`perturbed_queries` -- points plus isotropic Gaussian offsets.
* :func:`make_tie_free` -- nudges coordinates that sit exactly on a split
  of the reference octree lattice (the reference breaks such ties with
  rand(), sources/apss/CPUUtils.cpp:299-308), so that every build of the
  same cloud has one topology.

All outputs are float32 arrays of shape (n, 3).
"""
from __future__ import annotations

import numpy as np

F32 = np.float32


def _bbox_diag(p: np.ndarray) -> float:
    p = np.asarray(p, dtype=np.float64)
    return float(np.linalg.norm(p.max(0) - p.min(0)))


def torus(n: int, R: float = 1.0, r: float = 0.35, noise: float = 0.002, seed: int = 1):
    """Points uniform in area on a torus (rejection on the (R + r cos v) factor)."""
    rng = np.random.default_rng(seed)
    us, vs = [], []
    have = 0
    while have < n:
        m = int((n - have) * 1.6) + 64
        u = rng.uniform(0.0, 2 * np.pi, m)
        v = rng.uniform(0.0, 2 * np.pi, m)
        keep = rng.uniform(0.0, 1.0, m) < (R + r * np.cos(v)) / (R + r)
        us.append(u[keep])
        vs.append(v[keep])
        have += int(keep.sum())
    u = np.concatenate(us)[:n]
    v = np.concatenate(vs)[:n]
    nrm = np.stack([np.cos(v) * np.cos(u), np.cos(v) * np.sin(u), np.sin(v)], axis=1)
    ring = np.stack([R * np.cos(u), R * np.sin(u), np.zeros_like(u)], axis=1)
    p = ring + r * nrm
    if noise > 0:
        p = p + rng.normal(0.0, noise, p.shape)
    return p.astype(F32), nrm.astype(F32)


def _blob_field(x, c, rho2):
    """f = sum_j exp(-|x-c_j|^2/rho_j^2) and its gradient (float64)."""
    d = x[:, None, :] - c[None, :, :]
    e = np.exp(-(d * d).sum(-1) / rho2[None, :])
    f = e.sum(1)
    g = (-2.0 * e / rho2[None, :])[:, :, None] * d
    return f, g.sum(1)


def _newton_torch(x, c, rho2, tau, device):
    """The Newton projection of rbf_blobs on a torch device (float64)."""
    import torch

    xt = torch.from_numpy(x).to(device)
    ct = torch.from_numpy(c).to(device)
    rt = torch.from_numpy(rho2).to(device)

    def field(v):
        d = v[:, None, :] - ct[None, :, :]
        e = torch.exp(-(d * d).sum(-1) / rt[None, :])
        return e.sum(1), ((-2.0 * e / rt[None, :])[:, :, None] * d).sum(1)

    for _ in range(30):
        f, g = field(xt)
        gg = (g * g).sum(1).clamp_min(1e-30)
        step = ((f - tau) / gg)[:, None] * g
        done = (f - tau).abs() <= 1e-13
        xt = torch.where(done[:, None], xt, xt - step)
        if bool(done.all()):
            break
    f, g = field(xt)
    return xt.cpu().numpy(), f.cpu().numpy(), g.cpu().numpy()


def rbf_blobs(n: int, n_blobs: int = 12, noise: float = 0.003, seed: int = 2, tau: float = 0.5,
              translate: float = 1e3, batch: int = 1 << 18, device=None):
    """Samples of the level set sum_j exp(-|x-c_j|^2/rho_j^2) = tau.

    Centres ~ U[-1, 1]^3, radii ~ U[0.2, 0.5].  Candidates start on the
    single-blob spheres and are Newton-projected onto the union's level set;
    normals are the normalised negative gradient (outward).  After noise the
    cloud is moved by translate * diag along (1, 1, 1)/sqrt(3).  With a torch
    `device` the Newton iterations run there (same candidates and noise).
    """
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1.0, 1.0, (n_blobs, 3))
    rho = rng.uniform(0.2, 0.5, n_blobs)
    rho2 = rho * rho
    s = np.sqrt(np.log(1.0 / tau))
    pts, nrms = [], []
    have = 0
    while have < n:
        m = min(batch, int((n - have) * 1.5) + 64)
        j = rng.integers(0, n_blobs, m)
        u = rng.normal(size=(m, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        x = c[j] + (rho[j] * s)[:, None] * u
        if device is not None:
            x, f, g = _newton_torch(x, c, rho2, tau, device)
        else:
            act = np.arange(m)
            for _ in range(30):
                f, g = _blob_field(x[act], c, rho2)
                gg = (g * g).sum(1)
                x[act] = x[act] - ((f - tau) / np.maximum(gg, 1e-30))[:, None] * g
                act = act[np.abs(f - tau) > 1e-13]
                if len(act) == 0:
                    break
            f, g = _blob_field(x, c, rho2)
        gn = np.linalg.norm(g, axis=1)
        ok = (np.abs(f - tau) < 1e-9) & (gn > 1e-6) & np.all(np.abs(x) < 4.0, axis=1)
        pts.append(x[ok])
        nrms.append(-g[ok] / gn[ok, None])
        have += int(ok.sum())
    p = np.concatenate(pts)[:n]
    nv = np.concatenate(nrms)[:n]
    if noise > 0:
        p = p + rng.normal(0.0, noise, p.shape)
    if translate:
        diag = _bbox_diag(p)
        p = p + translate * diag / np.sqrt(3.0)
    return p.astype(F32), nv.astype(F32)


def torus_knot(n: int, p: int = 2, q: int = 3, R: float = 1.0, r: float = 0.5, tube: float = 0.15,
               noise: float = 0.002, n_holes: int = 20, removed: float = 0.10, seed: int = 4):
    """Tube of radius `tube` around the (p, q) torus knot
    C(t) = ((R + r cos qt) cos pt, (R + r cos qt) sin pt, r sin qt), with
    `n_holes` random spherical holes removing a `removed` fraction."""
    rng = np.random.default_rng(seed)
    n_gen = int(np.ceil(n / (1.0 - removed))) + 1024

    def curve(t):
        a = R + r * np.cos(q * t)
        return np.stack([a * np.cos(p * t), a * np.sin(p * t), r * np.sin(q * t)], axis=1)

    def dcurve(t):
        a = R + r * np.cos(q * t)
        da = -r * q * np.sin(q * t)
        return np.stack([da * np.cos(p * t) - a * p * np.sin(p * t), da * np.sin(p * t) + a * p * np.cos(p * t),
                         r * q * np.cos(q * t)], axis=1)

    tt = np.linspace(0, 2 * np.pi, 4097)
    vmax = np.linalg.norm(dcurve(tt), axis=1).max()
    ts, ths = [], []
    have = 0
    while have < n_gen:
        m = int((n_gen - have) * 1.5) + 64
        t = rng.uniform(0, 2 * np.pi, m)
        th = rng.uniform(0, 2 * np.pi, m)
        keep = rng.uniform(0, 1, m) < np.linalg.norm(dcurve(t), axis=1) / vmax
        ts.append(t[keep])
        ths.append(th[keep])
        have += int(keep.sum())
    t = np.concatenate(ts)[:n_gen]
    th = np.concatenate(ths)[:n_gen]
    T = dcurve(t)
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    N = np.cross(T, np.array([0.0, 0.0, 1.0]))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    B = np.cross(T, N)
    nv = np.cos(th)[:, None] * N + np.sin(th)[:, None] * B
    pts = curve(t) + tube * nv
    if noise > 0:
        pts = pts + rng.normal(0.0, noise, pts.shape)
    # holes: centres on the cloud, common radius found by bisection
    centres = pts[rng.choice(len(pts), n_holes, replace=False)]
    d2 = np.full(len(pts), np.inf)
    for cc in centres:
        d2 = np.minimum(d2, ((pts - cc) ** 2).sum(1))
    target = len(pts) - n
    order = np.sort(d2)
    rad2 = order[target - 1] if target > 0 else -1.0
    keep = d2 > rad2
    pts, nv = pts[keep][:n], nv[keep][:n]
    return pts.astype(F32), nv.astype(F32)


def perturbed_queries(points: np.ndarray, rel_sigma: float = 0.01, seed: int = 3) -> np.ndarray:
    """points + N(0, (rel_sigma * bbox diagonal)^2), rounded to float32."""
    rng = np.random.default_rng(seed)
    sig = rel_sigma * _bbox_diag(points)
    q = np.asarray(points, np.float64) + rng.normal(0.0, sig, points.shape)
    return q.astype(F32)


def split_tables(lo: float, hi: float, depth: int):
    """Per-axis split values (float64) and child bounds (float32) of the
    reference recursion (CPUUtils.cpp:286-292, :321-323) for one axis: the
    float bounds are added in float, then halved in double."""
    bounds = [np.array([lo, hi], dtype=F32)]
    splits = []
    for _ in range(depth):
        b = bounds[-1]
        s = (b[:-1] + b[1:]).astype(F32).astype(np.float64) / 2.0
        splits.append(s)
        nb = np.empty(2 * len(b) - 1, dtype=F32)
        nb[0::2] = b
        nb[1::2] = s.astype(F32)
        bounds.append(nb)
    return splits, bounds


def count_split_ties(points: np.ndarray, depth: int = 12) -> int:
    """Number of (point, axis) pairs lying exactly on a split of their path."""
    p = np.asarray(points, dtype=F32)
    total = 0
    for a in range(3):
        x = p[:, a].astype(np.float64)
        splits, _ = split_tables(p[:, a].min(), p[:, a].max(), depth)
        k = np.zeros(len(x), dtype=np.int64)
        tie = np.zeros(len(x), dtype=bool)
        for s in splits:
            sv = s[k]
            tie |= x == sv
            k = 2 * k + (x > sv)
        total += int(tie.sum())
    return total


def make_tie_free(points: np.ndarray, depth: int = 12, max_rounds: int = 8) -> np.ndarray:
    """Return a copy where no coordinate equals a split value on its path.

    Axes on which all points are equal are left alone (every split of such an
    axis equals the coordinate)."""
    p = np.array(points, dtype=F32, copy=True)
    for _ in range(max_rounds):
        changed = False
        for a in range(3):
            if p[:, a].min() == p[:, a].max():
                continue  # a flat axis ties everywhere; nudging would only move the box
            x = p[:, a].astype(np.float64)
            splits, _ = split_tables(p[:, a].min(), p[:, a].max(), depth)
            k = np.zeros(len(x), dtype=np.int64)
            tie = np.zeros(len(x), dtype=bool)
            for s in splits:
                sv = s[k]
                tie |= x == sv
                k = 2 * k + (x > sv)
            if tie.any():
                p[tie, a] = np.nextafter(p[tie, a], np.float32(np.inf))
                changed = True
        if not changed:
            return p
    raise RuntimeError("could not remove split ties")


def normalize_like_pn(points: np.ndarray) -> np.ndarray:
    """Pn::normalize (sources/apss/Pn.cpp:262-290) in float: centre on the
    mean, pad the box by 0.5% of its diagonal, divide by the largest absolute
    coordinate, so the cloud fits the [-1, 1]^3 zone of the DC grid."""
    p = np.asarray(points, np.float32)
    off = p.astype(np.float64).mean(0).astype(np.float32)
    mx = (p.max(0) - off).astype(np.float32)
    mn = (p.min(0) - off).astype(np.float32)
    small = np.float32(np.linalg.norm((mx - mn).astype(np.float32)) * np.float32(0.005))
    mx = mx + small
    mn = mn - small
    norme = np.float32(max(np.abs(mx).max(), np.abs(mn).max()))
    return ((p - off) / norme).astype(np.float32)


def bbox_diag(points: np.ndarray) -> float:
    return _bbox_diag(points)
