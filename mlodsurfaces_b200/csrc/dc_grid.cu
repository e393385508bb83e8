// dc_grid.cu -- the dual-contouring cell grid built from points (host).
//
// OctreeGenerator::generateFromPoints (upsample.cpp:128-144) then
// uniformizeFromPoints (upsample.cpp:253-260): the cells enclosing the points
// at max_depth, graded (grade, upsample.cpp:67-93), completed with all their
// ancestors (regularize_up, :40-46) and with the siblings of every non-root
// cell (regularize_siblings, :48-65), in sorted_octree order (node_comparator,
// octree.h:147-154: depth, then z, y, x).  Integer set work on a few million
// cells; the device evaluates the field on the result.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "dc.h"
#include "mlods_internal.cuh"

namespace mlods
{
namespace dcg
{
void remove_duplicates(std::vector<Cell>& v)
{
    std::sort(v.begin(), v.end(), cell_less);
    v.erase(std::unique(v.begin(), v.end()), v.end());
}

static void remove_duplicates_reverse(std::vector<Cell>& v)
{
    std::sort(v.rbegin(), v.rend(), cell_less);
    v.erase(std::unique(v.begin(), v.end()), v.end());
}

// grade, upsample.cpp:67-93
void grade(std::vector<Cell>& nodes)
{
    static const int corners[8] = {0, 2, 6, 8, 18, 20, 24, 26};
    if (nodes.empty()) return;
    std::sort(nodes.rbegin(), nodes.rend(), cell_less);
    size_t i = 0;
    int current = nodes[0].depth;
    while (i < nodes.size()) {
        if (current != nodes[i].depth) {
            remove_duplicates_reverse(nodes);
            current = nodes[i].depth;
        }
        if (nodes[i].depth > 0)
            for (int c : corners) nodes.push_back(parent(neighbor(nodes[i], c)));
        ++i;
    }
    remove_duplicates(nodes);
}

// regularize_up, upsample.cpp:40-46
void regularize_up(std::vector<Cell>& nodes)
{
    for (size_t t = 0; t < nodes.size(); ++t)
        if (nodes[t].depth != 0) nodes.push_back(parent(nodes[t]));
    remove_duplicates(nodes);
}

// regularize_siblings, upsample.cpp:48-65 (entries of depth-0 cells stay the
// default octree_id, the root)
void regularize_siblings(std::vector<Cell>& nodes)
{
    const size_t s = nodes.size();
    nodes.resize(9 * s, Cell{0, 0, 0, 0});
    for (size_t t = 0; t < s; ++t) {
        if (nodes[t].depth <= 0) continue;
        const Cell p = parent(nodes[t]);
        for (int k = 0; k < 8; ++k) nodes[s + 8 * t + k] = child(p, k);
    }
    remove_duplicates(nodes);
}

// expand, upsample.cpp:404-414
void expand(std::vector<Cell>& nodes, int depth)
{
    const size_t n = nodes.size();
    for (size_t t = 0; t < n; ++t) {
        if (depth >= 0 && nodes[t].depth != depth) continue;
        for (int k = 0; k < 27; ++k)
            if (k != 13) nodes.push_back(neighbor(nodes[t], k));
    }
    remove_duplicates(nodes);
}

void cells_to_ints(const std::vector<Cell>& nodes, std::vector<int32_t>& out, int& max_depth)
{
    max_depth = 0;
    out.resize(nodes.size() * 4);
    for (size_t i = 0; i < nodes.size(); ++i) {
        out[4 * i] = nodes[i].depth;
        out[4 * i + 1] = nodes[i].x;
        out[4 * i + 2] = nodes[i].y;
        out[4 * i + 3] = nodes[i].z;
        max_depth = std::max(max_depth, nodes[i].depth);
    }
}

}  // namespace dcg

using namespace dcg;

int dcgrid_from_points(const float* pts, int64_t n, int max_depth, const float box_min[3], const float box_max[3],
                       std::vector<int32_t>& cells_out, int& depth_out)
{
    if (n <= 0 || !pts) {
        set_last_error("dc grid: no points");
        return MLODS_ERR_INVALID;
    }
    if (max_depth < 0 || max_depth > 16) {
        set_last_error("dc grid: max_depth=%d out of range [0, 16]", max_depth);
        return MLODS_ERR_INVALID;
    }
    float diag[3];
    for (int a = 0; a < 3; ++a) {
        diag[a] = box_max[a] - box_min[a];
        if (!(diag[a] > 0.f)) {
            set_last_error("dc grid: empty box");
            return MLODS_ERR_INVALID;
        }
    }
    // aabb_octree::enclosing, octree.h:957-965: P = (pos - min) / diag / w, floored
    const float w = 1.0f / float(1 << max_depth);
    std::vector<Cell> nodes(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        int c[3];
        for (int a = 0; a < 3; ++a) {
            const float t = (pts[3 * i + a] - box_min[a]) / diag[a] / w;
            c[a] = int(std::floor(t));
        }
        nodes[size_t(i)] = Cell{max_depth, c[0], c[1], c[2]};
    }
    remove_duplicates(nodes);
    grade(nodes);
    regularize_up(nodes);
    regularize_siblings(nodes);
    cells_to_ints(nodes, cells_out, depth_out);
    return MLODS_OK;
}

}  // namespace mlods
