"""TEST INFRASTRUCTURE ONLY: pure-Python restatement of the reference's
dual-contouring grid for small inputs.

OctreeGenerator::generateFromPoints (sources/scene/upsample.cpp:128-144),
uniformizeFromPoints (:253-260) with grade (:67-93), regularize_up (:40-46)
and regularize_siblings (:48-65); octree_id parent/child/neighbor
(sources/dual-contouring/octree.h:547-602); node_comparator (:147-154);
aabb_octree::enclosing (:957-965).  Cells are (depth, x, y, z) tuples.
"""
from __future__ import annotations

import numpy as np

CORNERS = (0, 2, 6, 8, 18, 20, 24, 26)


def key(c):
    """node_comparator: depth, then z, y, x."""
    return (c[0], c[3], c[2], c[1])


def parent(c):
    d, x, y, z = c
    return (d - 1, x // 2, y // 2, z // 2)  # Python // floors, as octree_id::parent


def child(c, k):
    d, x, y, z = c
    return (d + 1, 2 * x + (k & 1), 2 * y + ((k >> 1) & 1), 2 * z + ((k >> 2) & 1))


def neighbor(c, n):
    z = n // 9
    y = (n - 9 * z) // 3
    x = n - 9 * z - 3 * y
    return (c[0], c[1] + x - 1, c[2] + y - 1, c[3] + z - 1)


def remove_duplicates(v):
    return sorted(set(v), key=key)


def grade(nodes):
    nodes = sorted(nodes, key=key, reverse=True)
    i = 0
    cur = nodes[0][0]
    while i < len(nodes):
        if cur != nodes[i][0]:
            nodes = sorted(set(nodes), key=key, reverse=True)
            cur = nodes[i][0]
        if nodes[i][0] > 0:
            for c in CORNERS:
                nodes.append(parent(neighbor(nodes[i], c)))
        i += 1
    return remove_duplicates(nodes)


def regularize_up(nodes):
    nodes = list(nodes)
    t = 0
    while t < len(nodes):
        if nodes[t][0] != 0:
            nodes.append(parent(nodes[t]))
        t += 1
    return remove_duplicates(nodes)


def regularize_siblings(nodes):
    out = list(nodes)
    for c in nodes:
        if c[0] <= 0:
            out.append((0, 0, 0, 0))
            continue
        p = parent(c)
        out.extend(child(p, k) for k in range(8))
    return remove_duplicates(out)


def grid_from_points(pts, max_depth, box_min=(-1.0, -1.0, -1.0), box_max=(1.0, 1.0, 1.0)):
    p = np.asarray(pts, np.float32)
    bmin = np.asarray(box_min, np.float32)
    diag = (np.asarray(box_max, np.float32) - bmin).astype(np.float32)
    w = np.float32(1.0) / np.float32(1 << max_depth)
    t = ((p - bmin).astype(np.float32) / diag).astype(np.float32) / w
    c = np.floor(t.astype(np.float32)).astype(np.int64)
    nodes = remove_duplicates([(max_depth, int(a), int(b), int(d)) for a, b, d in c])
    nodes = grade(nodes)
    nodes = regularize_up(nodes)
    nodes = regularize_siblings(nodes)
    return np.array(nodes, np.int32).reshape(-1, 4)


# ---- projection-driven grid (OctreeGenerator::generate + uniformize) ----------

def expand(nodes, depth=-1):
    """upsample.cpp:404-414: add the 26 neighbours of the cells at `depth`
    (all cells when depth < 0), sorted and unique."""
    out = list(nodes)
    for c in nodes:
        if depth >= 0 and c[0] != depth:
            continue
        out.extend(neighbor(c, k) for k in range(27) if k != 13)
    return remove_duplicates(out)


def ancestor_at(c, d):
    while c[0] > d:
        c = parent(c)
    return c


def octzone_center(cells):
    """aabb_octree over [-1, 1]^3: cell centres in float32 (octree.h:944-955)."""
    c = np.asarray(cells, np.int64).reshape(-1, 4)
    w = (np.float32(2.0) / (np.int64(1) << c[:, 0]).astype(np.float32)).astype(np.float32)
    p = c[:, 1:4].astype(np.float32)
    lo = (np.float32(-1.0) + (w[:, None] * p).astype(np.float32)).astype(np.float32)
    hi = (np.float32(-1.0) + (w[:, None] * (p + np.float32(1))).astype(np.float32)).astype(np.float32)
    return ((lo + hi).astype(np.float32) / np.float32(2.0)).astype(np.float32)


def octzone_enclosing(p, depth):
    """aabb_octree::enclosing (octree.h:957-965)."""
    w = np.float32(1.0) / np.float32(1 << depth)
    t = (((np.asarray(p, np.float32) - np.float32(-1.0)).astype(np.float32) / np.float32(2.0)).astype(np.float32)
         / w).astype(np.float32)
    return tuple(int(v) for v in np.floor(t))


def stable_nodes(nodes, project):
    """find_stable_nodesGPU (upsample.cpp:304-331); project(centres) returns
    (points, normals) of one projection step without a step limit."""
    if not nodes:
        return []
    pts, nrm = project(octzone_center(nodes))
    out = []
    for c, p, n in zip(nodes, np.asarray(pts, np.float32), np.asarray(nrm, np.float32)):
        l2 = np.float32(n[0] * n[0] + n[1] * n[1] + n[2] * n[2])
        out.append((0, 0, 0, 0) if l2 < np.float32(0.5) else (c[0],) + octzone_enclosing(p, c[0]))
    return remove_duplicates(out)


def compute_leaves(current, max_depth, total, project):
    """upsample.cpp:276-289."""
    for depth in range(max_depth + 1):
        sub = stable_nodes(current, project)
        current = [child(c, k) for c in sub for k in range(8)]
        current = expand(current, depth + 1)
        total.extend(current)
    return current


def relative_depth(nodes, mx, mn):
    """getRelativeDepth (upsample.cpp:146-160); mx/mn are updated in place."""
    if not nodes:
        return 0
    for c in nodes:
        a = ancestor_at(c, 0)
        for k in range(3):
            mn[k] = min(mn[k], a[k + 1])
            mx[k] = max(mx[k], a[k + 1])
    dd = 0
    for k in range(3):
        dd = max(dd, int(np.ceil(np.float32(np.log2(float(mx[k] - mn[k] + 1))))))
    return dd


def generate(max_depth, project):
    """OctreeGenerator::generate (upsample.cpp:228-251): the collected
    candidates (total_tree), cut to the adaptive maximum depth."""
    depth0 = [(0, 0, 0, 0)]
    old, total = [], []
    max_rel = max_depth
    mn = [2**31 - 1] * 3
    mx = [-(2**31 - 1)] * 3
    while depth0:
        total.extend(depth0)
        current = compute_leaves(depth0, max_rel, total, project)
        max_rel = max(0, max_depth - relative_depth(current, mx, mn))
        old.extend(depth0)
        depth0 = remove_duplicates([ancestor_at(c, 0) for c in current])
        depth0 = expand(depth0)
        seen = set(old)
        depth0 = [c for c in depth0 if c not in seen]
    total = [ancestor_at(c, max_rel) for c in total]
    return remove_duplicates(total)


def uniformize(nodes, max_depth, cut=False):
    """uniformize + retreiveCorrectRoot (upsample.cpp:262-273, :369-402):
    (cells, new_diag, new_origin)."""
    nodes = list(nodes) + remove_duplicates([ancestor_at(c, 0) for c in nodes])
    d0 = [c for c in nodes if c[0] == 0]
    mn = [min(c[k + 1] for c in d0) for k in range(3)]
    mx = [max(c[k + 1] for c in d0) for k in range(3)]
    dd = max(int(np.ceil(np.float32(np.log2(float(mx[k] - mn[k] + 1))))) for k in range(3))
    diag, origin = 1.0, (0.0, 0.0, 0.0)
    if dd > 0:
        nodes = [(c[0] + dd, c[1] - mn[0] * (1 << c[0]), c[2] - mn[1] * (1 << c[0]), c[3] - mn[2] * (1 << c[0]))
                 for c in nodes]
        diag, origin = float(1 << dd), tuple(float(v) for v in mn)
    nodes = grade(remove_duplicates(nodes))
    nodes = regularize_up(nodes)
    if cut:
        nodes = [c for c in nodes if c[0] <= max_depth]
    nodes = regularize_siblings(nodes)
    return np.array(nodes, np.int32).reshape(-1, 4), diag, origin
