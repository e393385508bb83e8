"""The rule by which the kNN projection keeps a neighbour set between
iterations, checked on the CPU against brute force.

After a search at iterate w0, every point outside the k found is at least
out_lo = sqrt(L) (1 - 1e-5) away, L being the (k+1)-th squared float
distance (the search's final bound), and the (k+1)-th nearest at most
out_hi = sqrt(L) (1 + 1e-5).  At the next iterate w1, a step of length s
away, the kept points are re-ranked without a search when
sqrt(max new squared distance of the kept points) (1 + 1e-5) <
(out_lo - s) (1 - 1e-5); otherwise the search starts from the smaller of
((out_hi + s) (1 + 1e-5))^2 and the largest new squared distance among the
kept points and one point outside them.  Distances are the reference
kd-tree's (kdTreeNN.h:424): float differences, float products,
left-to-right float sums."""
import numpy as np


def kd_d2(pts, q):
    """Squared distances as float32 operations in the reference's order."""
    d = pts - q.astype(np.float32)
    d2 = d[:, 0] * d[:, 0]
    d2 = d2 + d[:, 1] * d[:, 1]
    return d2 + d[:, 2] * d[:, 2]


def ranked(d2, idx):
    """Indices ordered by (distance, index), as the warp merge keeps them."""
    return idx[np.lexsort((idx, d2[idx]))]


def test_kept_sets_equal_fresh_searches_and_bounds_hold():
    rng = np.random.default_rng(41)
    n, k = 6000, 32
    u = rng.normal(size=(n, 3))
    pts = (u / np.linalg.norm(u, axis=1, keepdims=True) * 1.0 + 1e3).astype(np.float32)
    allidx = np.arange(n)
    kept_count = 0
    trials = 0
    for t in range(400):
        w0 = (pts[rng.integers(n)].astype(np.float64) + rng.normal(scale=0.01, size=3)).astype(np.float32)
        d0 = kd_d2(pts, w0)
        order0 = ranked(d0, allidx)
        kept = order0[:k]
        L = float(d0[order0[k]])
        out_lo = np.sqrt(L) * (1 - 1e-5)
        out_hi = np.sqrt(L) * (1 + 1e-5)
        for scale in (1e-7, 1e-5, 1e-4, 1e-3, 1e-2):
            trials += 1
            w1 = (w0.astype(np.float64) + rng.normal(size=3) * scale).astype(np.float32)
            step = float(np.linalg.norm(w1.astype(np.float64) - w0.astype(np.float64)))
            d1 = kd_d2(pts, w1)
            fresh = ranked(d1, allidx)
            dmax = float(d1[kept].max())
            kth1 = float(d1[fresh[k]])  # the new (k+1)-th squared distance
            if np.sqrt(dmax) * (1 + 1e-5) < (out_lo - step) * (1 - 1e-5):
                kept_count += 1
                assert np.array_equal(ranked(d1, kept), fresh[:k])
            # both starting bounds of a search are at least the (k+1)-th distance
            # (the kernel rounds the first one up to float)
            r = (out_hi + step) * (1 + 1e-5)
            assert r * r >= kth1
            other = np.setdiff1d(allidx, kept)[0]
            assert max(dmax, float(d1[other])) >= kth1
    # the rule does keep sets: the short steps (up to 1e-4 of the radius)
    # keep nearly all of them, steps of 1e-2 almost none
    assert trials // 3 < kept_count < trials
