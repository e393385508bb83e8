// dc_adaptive.cu -- the projection-driven dual-contouring grid.
//
// OctreeGenerator::generate (upsample.cpp:228-251) refines cells level by
// level: the centre of every candidate cell is projected once onto the
// surface (no step limit, find_stable_nodesGPU, upsample.cpp:304-331), the
// cell at the same depth that encloses the projection is kept (the root when
// the projection failed), its 8 children and their 26 neighbours become the
// next level's candidates (compute_leaves, :276-289).  Depth-0 cells next to
// the ones reached are explored the same way until no new one appears, and
// every level's candidates are collected.  uniformize (:262-273) then shifts
// the collection under one root (retreiveCorrectRoot / union_nodes,
// :369-402), grades, completes ancestors and siblings and optionally cuts at
// the maximum depth.  The projections run on the device (one launch per
// level); the integer set work stays on the host, as the reference's does.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>

#include "dc.h"
#include "tree.cuh"

namespace mlods
{
namespace
{
using dcg::Cell;
// bound on the depth-0 cells explored (the [-1, 1]^3 zone is one of them; a
// surface normalised into it reaches its 26 neighbours at most)
constexpr size_t kMaxRootCells = 4096;

// aabb_octree over [-1, 1]^3 (upsample.cpp:307-310): centre of a cell,
// octree.h:944-955, float arithmetic
inline void octzone_center(const Cell& c, float out[3])
{
    const float w = 2.0f / float(1 << c.depth);
    const int p[3] = {c.x, c.y, c.z};
    for (int a = 0; a < 3; ++a) {
        const float lo = -1.0f + w * float(p[a]);
        const float hi = -1.0f + w * float(p[a] + 1);
        out[a] = (lo + hi) / 2.0f;
    }
}

// float -> int as x86 truncation does for out-of-range values (INT_MIN)
inline int floor_to_int(float v)
{
    const float f = std::floor(v);
    if (!(f >= -2147483648.0f && f < 2147483648.0f)) return INT_MIN;
    return int(f);
}

// aabb_octree::enclosing, octree.h:957-965
inline Cell octzone_enclosing(const float p[3], int depth)
{
    const float w = 1.0f / float(1 << depth);
    int c[3];
    for (int a = 0; a < 3; ++a) c[a] = floor_to_int((p[a] - -1.0f) / 2.0f / w);
    return Cell{depth, c[0], c[1], c[2]};
}

struct Projector {
    mlods_tree_s* T;
    cudaStream_t s;
    float* d_buf = nullptr;
    size_t cap = 0;
    int64_t projected = 0;
    ~Projector() { cudaFree(d_buf); }

    // One projection step of the cell centres, no step limit
    // (find_stable_nodesGPU, upsample.cpp:304-331): the enclosing cell at the
    // same depth, or the root when the projection failed; sorted, unique.
    int stable(const std::vector<Cell>& nodes, std::vector<Cell>& out)
    {
        out.clear();
        const size_t n = nodes.size();
        if (n == 0) return MLODS_OK;
        if (cap < n) {
            cudaFree(d_buf);
            d_buf = nullptr;
            cap = 0;
            MLODS_CUDA(cudaMalloc(&d_buf, n * 9 * sizeof(float)));
            cap = n;
        }
        std::vector<float> h(n * 3), hn(n * 3);
        for (size_t i = 0; i < n; ++i) octzone_center(nodes[i], &h[3 * i]);
        float* d_q = d_buf;
        float* d_p = d_buf + 3 * n;
        float* d_n = d_buf + 6 * n;
        MLODS_CUDA(cudaMemcpyAsync(d_q, h.data(), n * 12, cudaMemcpyHostToDevice, s));
        const int rc = project_buffers(T, int64_t(n), d_q, d_p, d_n, 1, FLT_MAX, s);
        if (rc != MLODS_OK) return rc;
        MLODS_CUDA(cudaMemcpyAsync(h.data(), d_p, n * 12, cudaMemcpyDeviceToHost, s));
        MLODS_CUDA(cudaMemcpyAsync(hn.data(), d_n, n * 12, cudaMemcpyDeviceToHost, s));
        MLODS_CUDA(cudaStreamSynchronize(s));
        projected += int64_t(n);
        out.resize(n);
        for (size_t i = 0; i < n; ++i) {
            const float* v = &hn[3 * i];
            const float l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            out[i] = l2 < 0.5f ? Cell{0, 0, 0, 0} : octzone_enclosing(&h[3 * i], nodes[i].depth);
        }
        dcg::remove_duplicates(out);
        return MLODS_OK;
    }
};

void append(std::vector<Cell>& v, const std::vector<Cell>& a) { v.insert(v.end(), a.begin(), a.end()); }

// compute_leaves, upsample.cpp:276-289
int compute_leaves(Projector& P, std::vector<Cell> current, int max_depth, std::vector<Cell>& total,
                   std::vector<Cell>& out)
{
    std::vector<Cell> sub;
    for (int depth = 0; depth < max_depth + 1; ++depth) {
        const int rc = P.stable(current, sub);
        if (rc != MLODS_OK) return rc;
        current.resize(sub.size() * 8);
        for (size_t i = 0; i < sub.size(); ++i)
            for (int k = 0; k < 8; ++k) current[8 * i + size_t(k)] = dcg::child(sub[i], k);
        dcg::expand(current, depth + 1);
        append(total, current);
    }
    out.swap(current);
    return MLODS_OK;
}

// getRelativeDepth, upsample.cpp:146-160 (min/max persist across calls)
int relative_depth(const std::vector<Cell>& nodes, int mx[3], int mn[3])
{
    if (nodes.empty()) return 0;
    for (const Cell& n : nodes) {
        const Cell a = dcg::ancestor_at(n, 0);
        const int p[3] = {a.x, a.y, a.z};
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], p[k]);
            mx[k] = std::max(mx[k], p[k]);
        }
    }
    int dd = 0;
    for (int k = 0; k < 3; ++k) {
        const int ext = mx[k] - mn[k] + 1;
        dd = std::max(dd, int(std::ceil(float(std::log2(double(ext))))));  // int extent: log2 in double
    }
    return dd;
}

std::vector<Cell> depth0_ancestors(std::vector<Cell> nodes)
{
    for (Cell& n : nodes) n = dcg::ancestor_at(n, 0);
    dcg::remove_duplicates(nodes);
    return nodes;
}

// onlySetDepthNodes, upsample.cpp:162-172
void only_set_depth(std::vector<Cell>& nodes, int depth)
{
    for (Cell& n : nodes)
        if (n.depth > depth) n = dcg::ancestor_at(n, depth);
    dcg::remove_duplicates(nodes);
}

// OctreeGenerator::generate, upsample.cpp:228-251; returns the collected
// candidates (the reference's total_tree) cut to the adaptive maximum depth
int generate(Projector& P, int max_depth, std::vector<Cell>& total)
{
    std::vector<Cell> depth0 = {Cell{0, 0, 0, 0}}, old_depth0, current;
    int max_rel = max_depth;
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {-INT_MAX, -INT_MAX, -INT_MAX};
    total.clear();
    while (!depth0.empty()) {
        append(total, depth0);
        const int rc = compute_leaves(P, depth0, max_rel, total, current);
        if (rc != MLODS_OK) return rc;
        max_rel = std::max(0, max_depth - relative_depth(current, mx, mn));
        append(old_depth0, depth0);
        if (old_depth0.size() > kMaxRootCells) {
            set_last_error("dc adaptive grid: the surface spans more than %zu unit cells", kMaxRootCells);
            return MLODS_ERR_CAPACITY;
        }
        depth0 = depth0_ancestors(current);
        dcg::expand(depth0, -1);
        // vector_difference_inplace, upsample.cpp:103-112
        std::vector<Cell> seen = old_depth0;
        dcg::remove_duplicates(seen);
        depth0.erase(std::remove_if(depth0.begin(), depth0.end(),
                                    [&](const Cell& c) {
                                        return std::binary_search(seen.begin(), seen.end(), c, dcg::cell_less);
                                    }),
                     depth0.end());
    }
    only_set_depth(total, max_rel);
    return MLODS_OK;
}

// union_nodes + retreiveCorrectRoot, upsample.cpp:369-402
void correct_root(std::vector<Cell>& nodes, float new_diag[3], float new_origin[3])
{
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {-INT_MAX, -INT_MAX, -INT_MAX};
    bool has0 = false;
    for (const Cell& n : nodes) {
        if (n.depth != 0) continue;
        const int p[3] = {n.x, n.y, n.z};
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], p[k]);
            mx[k] = std::max(mx[k], p[k]);
        }
        has0 = true;
    }
    int dd = 0;
    if (has0)
        for (int k = 0; k < 3; ++k) dd = std::max(dd, int(std::ceil(float(std::log2(double(mx[k] - mn[k] + 1))))));
    if (!has0 || dd == 0) {
        // the reference returns depth -1 here and then evaluates 1 << -1; a
        // single depth-0 cell needs no shift, so keep the unit frame
        for (int k = 0; k < 3; ++k) {
            new_diag[k] = 1.0f;
            new_origin[k] = 0.0f;
        }
        return;
    }
    for (Cell& n : nodes) {
        const int s = 1 << n.depth;
        n.x -= mn[0] * s;
        n.y -= mn[1] * s;
        n.z -= mn[2] * s;
        n.depth += dd;
    }
    for (int k = 0; k < 3; ++k) {
        new_origin[k] = float(mn[k]);  // unit_octree::bounds(octree_id(0, min)).min()
        new_diag[k] = float(1 << dd);
    }
}

}  // namespace

int dcgrid_adaptive(mlods_tree_s* T, int max_depth, bool cut, cudaStream_t s, std::vector<int32_t>& cells_out,
                    int& depth_out, float xform[12], int64_t* n_projected)
{
    if (max_depth < 0 || max_depth > 14) {
        set_last_error("dc adaptive grid: max_depth=%d out of range [0, 14]", max_depth);
        return MLODS_ERR_INVALID;
    }
    if (!T->kernel_set) {
        set_last_error("dc adaptive grid: no kernel set (call mlods_set_kernel first)");
        return MLODS_ERR_STATE;
    }
    // the generator projects with the APSS object's project(), the MLoD (or
    // global) projection even when the octree is in kNN / ball mode
    const int saved_mode = T->params.mode;
    if (saved_mode == MLODS_MODE_KNN || saved_mode == MLODS_MODE_BALL) T->params.mode = MLODS_MODE_MLOD;
    Projector P{T, s};
    std::vector<Cell> nodes;
    const int rc = generate(P, max_depth, nodes);
    T->params.mode = saved_mode;
    if (rc != MLODS_OK) return rc;
    if (n_projected) *n_projected = P.projected;
    // uniformize, upsample.cpp:262-273
    append(nodes, depth0_ancestors(nodes));
    float nd[3], no[3];
    correct_root(nodes, nd, no);
    dcg::grade(nodes);
    dcg::regularize_up(nodes);
    if (cut) nodes.erase(std::remove_if(nodes.begin(), nodes.end(), [&](const Cell& c) { return c.depth > max_depth; }),
                         nodes.end());
    dcg::regularize_siblings(nodes);
    dcg::cells_to_ints(nodes, cells_out, depth_out);
    // new2bbox = unit2bbox * sortedOctreeToUnit (scene.cpp:1259-1311), box [-1, 1]^3
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 4; ++c) xform[4 * r + c] = 0.f;
        xform[4 * r + r] = 2.0f * nd[r];
        xform[4 * r + 3] = 2.0f * no[r] + -1.0f;
    }
    return MLODS_OK;
}

}  // namespace mlods
