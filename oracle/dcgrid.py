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
