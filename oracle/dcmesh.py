"""TEST INFRASTRUCTURE ONLY: pure-Python restatement of the reference's
dual-contouring mesh extraction and mesh refinement, for small inputs.

* minimal-edge enumeration: minimal_edges::traverse / traverse_node /
  traverse_face / traverse_edge (sources/dual-contouring/octree.h:400-540),
  over the sorted_octree relations (octree.h:206-275);
* triangle emission and vertex numbering: dual_contour::extract and
  on_min_edges (sources/dual-contouring/dual_contouring.h:59-87, :190-229);
* mesh::smoothMesh and mesh::subdivideMesh (sources/scene/upsample.h:55-133).

Cells are (depth, x, y, z) tuples; corner values are looked up by the integer
lattice corner at the deepest level.  The restatement enumerates the same
calls in the same order as the reference, so vertex numbering and triangle
order can be compared exactly.
"""
from __future__ import annotations

import numpy as np

X, Y, Z = 0, 1, 2


# The 4 inner edges of a face between two cells, per face direction: (edge
# direction, which half along it), in the order of the reference's
# subedges/subedgedir tables (octree.h:480-492).
FACE_EDGES = {
    X: ((Y, 0), (Y, 1), (Z, 0), (Z, 1)),
    Y: ((X, 1), (X, 0), (Z, 0), (Z, 1)),
    Z: ((Y, 0), (Y, 1), (X, 0), (X, 1)),
}


def _bit(c, axis):
    return (c >> axis) & 1


def _perp(axis):
    return [a for a in (X, Y, Z) if a != axis]


class SortedOctree:
    """sorted_octree: cells in node_comparator order, children by child id."""

    def __init__(self, cells):
        cells = [tuple(int(v) for v in c) for c in cells]
        self.cells = sorted(set(cells), key=lambda c: (c[0], c[3], c[2], c[1]))
        self.index = {c: i for i, c in enumerate(self.cells)}
        self.max_depth = max(c[0] for c in self.cells)
        self.children = [None] * len(self.cells)
        for i, (d, x, y, z) in enumerate(self.cells):
            kids = [self.index.get((d + 1, 2 * x + (k & 1), 2 * y + ((k >> 1) & 1), 2 * z + ((k >> 2) & 1)))
                    for k in range(8)]
            present = [k for k in kids if k is not None]
            if present:
                assert len(present) == 8, "every inner cell needs 8 children"
                self.children[i] = kids

    def is_leaf(self, n):
        return self.children[n] is None


def minimal_edges(tree: SortedOctree):
    """List of (n1, n2, n3, n4, dir) in the reference's traversal order."""
    out = []
    root = tree.index.get((0, 0, 0, 0))
    if root is None:
        return out

    def kid(n, k):
        return n if tree.is_leaf(n) else tree.children[n][k]

    def node(n):
        if tree.is_leaf(n):
            return
        ch = tree.children[n]
        for t in range(8):
            node(ch[t])
        for d in (X, Y, Z):
            for c in range(8):
                if not _bit(c, d):
                    face(ch[c], ch[c | (1 << d)], d)
        for e in (X, Y, Z):
            p1, p2 = _perp(e)
            for h in (0, 1):
                cells = [0] * 4
                for s1 in (0, 1):
                    for s2 in (0, 1):
                        c = (h << e) | (s1 << p1) | (s2 << p2)
                        cells[s1 + 2 * s2] = ch[c]
                edge(*cells, e)

    def face(n1, n2, d):
        if tree.is_leaf(n1) and tree.is_leaf(n2):
            return
        lo = [c for c in range(8) if _bit(c, d)]      # n1's children on the face
        hi = [c for c in range(8) if not _bit(c, d)]  # n2's children on the face
        for f in range(4):
            face(kid(n1, lo[f]), kid(n2, hi[f]), d)
        for e, h in FACE_EDGES[d]:
            (f_axis,) = [a for a in (X, Y, Z) if a not in (d, e)]
            p1, p2 = _perp(e)
            cells = [0] * 4
            for side_d in (0, 1):
                for side_f in (0, 1):
                    c = (h << e) | ((1 - side_d) << d) | (side_f << f_axis)
                    n = kid(n1, c) if side_d == 0 else kid(n2, c)
                    sides = {d: side_d, f_axis: side_f}
                    cells[sides[p1] + 2 * sides[p2]] = n
            edge(*cells, e)

    def edge(n1, n2, n3, n4, e):
        ns = (n1, n2, n3, n4)
        if all(tree.is_leaf(n) for n in ns):
            out.append((n1, n2, n3, n4, e))
            return
        p1, p2 = _perp(e)
        for h in (0, 1):
            sub = []
            for slot, n in enumerate(ns):
                s1, s2 = slot & 1, slot >> 1
                c = (h << e) | ((1 - s1) << p1) | ((1 - s2) << p2)
                sub.append(kid(n, c))
            edge(*sub, e)

    node(root)
    return out


def _corner(cell, k, max_depth):
    d, x, y, z = cell
    delta = 1 << (max_depth - d)
    return ((x + (k & 1)) * delta, (y + ((k >> 1) & 1)) * delta, (z + ((k >> 2) & 1)) * delta)


def edge_corners(e, slot):
    """The two corners (of the cell in `slot` around an edge of direction e)
    that bound the edge; in direction Y the upper end comes first, as in the
    reference's corner table (dual_contouring.h:208-213)."""
    p1, p2 = _perp(e)
    s1, s2 = slot & 1, slot >> 1
    base = ((1 - s1) << p1) | ((1 - s2) << p2)
    c_lo, c_hi = base, base | (1 << e)
    return (c_hi, c_lo) if e == Y else (c_lo, c_hi)


def extract(cells, corner_value, cell_vertex):
    """dual_contour::extract: (vertex cell indices in creation order,
    triangles as index triples).  corner_value(lattice_xyz) -> float;
    cell_vertex(cell_index) -> position (only used to fill the list)."""
    tree = SortedOctree(cells)
    md = tree.max_depth
    node_vertex = {}
    order = []
    tris = []

    def get_vertex(n):
        if n not in node_vertex:
            node_vertex[n] = len(order)
            order.append(n)
        return node_vertex[n]

    for n1, n2, n3, n4, e in minimal_edges(tree):
        nodes = (n1, n2, n3, n4)
        sel, sel_d = 0, -1
        for i in range(4):
            if tree.cells[nodes[i]][0] > sel_d:
                sel, sel_d = i, tree.cells[nodes[i]][0]
        c0, c1 = edge_corners(e, sel)
        f0 = corner_value(_corner(tree.cells[nodes[sel]], c0, md))
        f1 = corner_value(_corner(tree.cells[nodes[sel]], c1, md))
        if np.isnan(f0) or np.isnan(f1):
            continue
        m0, m1 = f0 < 0, f1 < 0
        if m0 == m1:
            continue
        for a, b, c in ((0, 1, 3), (0, 3, 2)):
            v = (get_vertex(nodes[a]), get_vertex(nodes[b]), get_vertex(nodes[c]))
            if v[0] == v[1] or v[1] == v[2] or v[2] == v[0]:
                continue
            tris.append((v[0], v[2], v[1]) if m0 else (v[0], v[1], v[2]))
    verts = [cell_vertex(tree.cells[n]) for n in order]
    return tree, order, verts, tris


def smooth(points, tris):
    """mesh::smoothMesh: every vertex moves to the mean of its triangle
    neighbours (counted once per incident triangle side), float32."""
    p = np.asarray(points, np.float32)
    new = np.zeros_like(p)
    val = np.zeros(len(p), np.float32)
    for a, b, c in tris:
        new[a] = new[a] + (p[b] + p[c])
        new[b] = new[b] + (p[a] + p[c])
        new[c] = new[c] + (p[b] + p[a])
        val[a] += 2
        val[b] += 2
        val[c] += 2
    return (new / val[:, None]).astype(np.float32)


def subdivide(points, tris):
    """mesh::subdivideMesh: 1 -> 4 split, new vertex per edge at the midpoint
    in first-seen order."""
    pts = [np.asarray(q, np.float32) for q in np.asarray(points, np.float32)]
    tris = [tuple(t) for t in tris]
    on_edge = {}

    def mid(i, j):
        k = (min(i, j), max(i, j))
        if k not in on_edge:
            pts.append(((pts[i] + pts[j]) / np.float32(2)).astype(np.float32))
            on_edge[k] = len(pts) - 1
        return on_edge[k]

    out = list(tris)
    for t, (a, b, c) in enumerate(tris):
        ab = mid(a, b)
        bc = mid(c, b)
        ca = mid(c, a)
        out[t] = (a, ab, ca)
        out.extend([(ab, b, bc), (ab, bc, ca), (ca, bc, c)])
    return np.array(pts, np.float32), out
