// dc_mesh.cu -- dual-contouring mesh extraction and refinement.
//
// Extraction (dual_contour::extract, dual_contouring.h:59-87, :190-229): the
// minimal edges of the cell octree are enumerated by the recursive
// node / face / edge procedure of minimal_edges::traverse (octree.h:400-540),
// in the same order; an edge whose two end values (corners of the deepest of
// its 3-4 cells) change sign gives two triangles over the cells' vertices,
// oriented by the sign of the first end.  Vertices are numbered on first use,
// as the reference's get_vertex does, so the index lists match it exactly.
// Refinement (scene.cpp:1402-1452, upsample.h:55-133): the vertices are
// projected (3 iterations), then twice smoothed, 1->4 subdivided and projected
// again.  Integer traversal and mesh edits stay on the host; projections run
// on the device.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "dc.h"
#include "tree.cuh"

// A mesh lives either in device memory (`dev`, the result of mlods_dc_mesh:
// the mesh functions then run on the device and mlods_mesh_get copies it
// out) or in the host vectors (the result of mlods_dc_extract).
struct mlods_mesh_s {
    std::vector<float> pos;  // 3 per vertex
    std::vector<float> nrm;  // 3 per vertex
    std::vector<uint32_t> tri;
    mlods::DeviceMesh* dev = nullptr;
    // host wall time of mlods_dc_mesh's stages (ms): corner field, extraction,
    // upload + transform, projections, smoothing, subdivision, download (0:
    // the mesh stays in device memory)
    double stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
    mlods_mesh_s() = default;
    mlods_mesh_s(const mlods_mesh_s&) = delete;
    mlods_mesh_s& operator=(const mlods_mesh_s&) = delete;
    ~mlods_mesh_s() { mlods::dmesh_destroy(dev); }
    int64_t nv() const { return dev ? mlods::dmesh_nv(*dev) : int64_t(pos.size() / 3); }
    int64_t nt() const { return dev ? mlods::dmesh_nt(*dev) : int64_t(tri.size() / 3); }
};

namespace mlods
{
namespace
{
using dcg::Cell;
constexpr int kX = 0, kY = 1, kZ = 2;

// (edge direction, half along it) of the 4 inner edges of a face, per face
// direction, in the order of the reference's subedges / subedgedir tables
// (octree.h:480-492)
constexpr int kFaceEdges[3][4][2] = {
    {{kY, 0}, {kY, 1}, {kZ, 0}, {kZ, 1}},
    {{kX, 1}, {kX, 0}, {kZ, 0}, {kZ, 1}},
    {{kY, 0}, {kY, 1}, {kX, 0}, {kX, 1}},
};

inline void perp(int e, int& p1, int& p2)
{
    p1 = e == kX ? kY : kX;
    p2 = e == kZ ? kY : kZ;
}

struct Grid {
    const int32_t* c;  // (depth, x, y, z) per cell, sorted
    int64_t n;
    int max_depth;
    std::vector<int64_t> begin;  // first cell of each depth, max_depth + 2 entries
    std::vector<int32_t> kids;   // 8 per cell, -1 for leaves

    Cell cell(int64_t i) const { return Cell{c[4 * i], c[4 * i + 1], c[4 * i + 2], c[4 * i + 3]}; }
    int64_t find(const Cell& q) const
    {
        if (q.depth < 0 || q.depth > max_depth) return -1;
        int64_t lo = begin[size_t(q.depth)], hi = begin[size_t(q.depth) + 1];
        while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if (dcg::cell_less(cell(mid), q)) lo = mid + 1;
            else hi = mid;
        }
        return (lo < begin[size_t(q.depth) + 1] && cell(lo) == q) ? lo : -1;
    }
};

// sorted_octree relations (octree.h:227-262): every non-root cell needs its
// parent and every inner cell exactly 8 children
int build_grid(const int32_t* cells, int64_t n, Grid& g)
{
    g.c = cells;
    g.n = n;
    g.max_depth = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (cells[4 * i] < 0 || cells[4 * i] > 30) {
            set_last_error("dc extract: cell %lld has depth %d", (long long)i, cells[4 * i]);
            return MLODS_ERR_INVALID;
        }
        g.max_depth = std::max(g.max_depth, int(cells[4 * i]));
        if (i > 0 && !dcg::cell_less(g.cell(i - 1), g.cell(i))) {
            set_last_error("dc extract: cells must be sorted (depth, z, y, x) and unique (cell %lld)", (long long)i);
            return MLODS_ERR_INVALID;
        }
    }
    g.begin.assign(size_t(g.max_depth) + 2, n);
    for (int64_t i = n - 1; i >= 0; --i) g.begin[size_t(cells[4 * i])] = i;
    for (int d = g.max_depth; d >= 0; --d)
        if (g.begin[size_t(d)] > g.begin[size_t(d) + 1]) g.begin[size_t(d)] = g.begin[size_t(d) + 1];
    if (n >= (int64_t(1) << 31)) {
        set_last_error("dc extract: %lld cells exceed 32-bit cell indices", (long long)n);
        return MLODS_ERR_CAPACITY;
    }
    g.kids.assign(size_t(n) * 8, -1);
    // parent lookups on host threads: every cell writes one distinct slot of
    // its parent, so the writes do not overlap
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::atomic<int64_t> orphan{-1};
    auto link = [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            const Cell c = g.cell(i);
            if (c.depth == 0) continue;
            const Cell p = dcg::parent(c);
            const int64_t pi = g.find(p);
            if (pi < 0) {
                orphan.store(i);
                continue;
            }
            const int k = (c.x - 2 * p.x) + 2 * (c.y - 2 * p.y) + 4 * (c.z - 2 * p.z);
            g.kids[size_t(pi) * 8 + size_t(k)] = int32_t(i);
        }
    };
    std::vector<std::thread> pool;
    const int64_t step = (n + hw - 1) / hw;
    for (unsigned t = 1; t < hw && int64_t(t) * step < n; ++t)
        pool.emplace_back(link, int64_t(t) * step, std::min(n, int64_t(t + 1) * step));
    link(0, std::min(n, step));
    for (std::thread& th : pool) th.join();
    if (orphan.load() >= 0) {
        set_last_error("dc extract: cell %lld has no parent in the grid", (long long)orphan.load());
        return MLODS_ERR_INVALID;
    }
    for (int64_t i = 0; i < n; ++i) {
        int cnt = 0;
        for (int k = 0; k < 8; ++k) cnt += g.kids[size_t(i) * 8 + size_t(k)] >= 0;
        if (cnt != 0 && cnt != 8) {
            set_last_error("dc extract: cell %lld has %d children (needs 0 or 8)", (long long)i, cnt);
            return MLODS_ERR_INVALID;
        }
    }
    return MLODS_OK;
}

// One call of the reference's recursive enumeration: traverse_node (kind 0,
// one cell), traverse_face (kind 1, two cells, direction d) or traverse_edge
// (kind 2, four cells, direction d).
struct Call {
    int kind, dir;
    int64_t n[4];
};

// A sign-changing minimal edge: its four cells (slot order) and whether its
// triangles are flipped.
struct Crossing {
    int32_t n[4];
    int32_t flip;
};

struct Walker {
    const Grid& g;
    const float* cf;  // 8 corner values per cell

    bool leaf(int64_t n) const { return g.kids[size_t(n) * 8] < 0; }
    int64_t kid(int64_t n, int c) const { return leaf(n) ? n : g.kids[size_t(n) * 8 + size_t(c)]; }
    bool minimal(const Call& c) const
    {
        return c.kind == 2 && leaf(c.n[0]) && leaf(c.n[1]) && leaf(c.n[2]) && leaf(c.n[3]);
    }

    // The calls a call makes, in the reference's order (octree.h:423-540).
    template <typename F>
    void children(const Call& c, F f) const
    {
        if (c.kind == 0) {  // traverse_node
            if (leaf(c.n[0])) return;
            const int32_t* ch = &g.kids[size_t(c.n[0]) * 8];
            for (int t = 0; t < 8; ++t) f(Call{0, 0, {ch[t], 0, 0, 0}});
            for (int d = 0; d < 3; ++d)
                for (int k = 0; k < 8; ++k)
                    if (!((k >> d) & 1)) f(Call{1, d, {ch[k], ch[k | (1 << d)], 0, 0}});
            for (int e = 0; e < 3; ++e) {
                int p1, p2;
                perp(e, p1, p2);
                for (int h = 0; h < 2; ++h) {
                    Call x{2, e, {0, 0, 0, 0}};
                    for (int s = 0; s < 4; ++s) x.n[s] = ch[(h << e) | ((s & 1) << p1) | ((s >> 1) << p2)];
                    f(x);
                }
            }
        } else if (c.kind == 1) {  // traverse_face
            const int d = c.dir;
            const int64_t n1 = c.n[0], n2 = c.n[1];
            if (leaf(n1) && leaf(n2)) return;
            int on1[4], on2[4], k1 = 0, k2 = 0;
            for (int k = 0; k < 8; ++k) {
                if ((k >> d) & 1) on1[k1++] = k;
                else on2[k2++] = k;
            }
            for (int q = 0; q < 4; ++q) f(Call{1, d, {kid(n1, on1[q]), kid(n2, on2[q]), 0, 0}});
            for (int k = 0; k < 4; ++k) {
                const int e = kFaceEdges[d][k][0], h = kFaceEdges[d][k][1];
                const int fa = 3 - d - e;  // the axis normal to both
                int p1, p2;
                perp(e, p1, p2);
                Call x{2, e, {0, 0, 0, 0}};
                for (int sd = 0; sd < 2; ++sd)
                    for (int sf = 0; sf < 2; ++sf) {
                        const int kk = (h << e) | ((1 - sd) << d) | (sf << fa);
                        const int s1 = p1 == d ? sd : sf, s2 = p2 == d ? sd : sf;
                        x.n[s1 + 2 * s2] = sd == 0 ? kid(n1, kk) : kid(n2, kk);
                    }
                f(x);
            }
        } else {  // traverse_edge
            if (minimal(c)) return;
            int p1, p2;
            perp(c.dir, p1, p2);
            for (int h = 0; h < 2; ++h) {
                Call x{2, c.dir, {0, 0, 0, 0}};
                for (int s = 0; s < 4; ++s)
                    x.n[s] = kid(c.n[s], (h << c.dir) | ((1 - (s & 1)) << p1) | ((1 - (s >> 1)) << p2));
                f(x);
            }
        }
    }

    // on_min_edges' test (dual_contouring.h:196-228): the edge's end values
    // are corners of the deepest of its cells (the first one on ties)
    void test(const Call& c, std::vector<Crossing>& out) const
    {
        int sel = 0, sel_d = -1;
        for (int i = 0; i < 4; ++i) {
            const int d = g.c[4 * c.n[i]];
            if (d > sel_d) {
                sel = i;
                sel_d = d;
            }
        }
        int p1, p2;
        perp(c.dir, p1, p2);
        const int base = ((1 - (sel & 1)) << p1) | ((1 - (sel >> 1)) << p2);
        int c0 = base, c1 = base | (1 << c.dir);
        if (c.dir == kY) std::swap(c0, c1);  // the reference lists the upper end first for Y edges
        const float f0 = cf[8 * c.n[sel] + c0], f1 = cf[8 * c.n[sel] + c1];
        if (std::isnan(f0) || std::isnan(f1)) return;
        const bool m0 = f0 < 0, m1 = f1 < 0;
        if (m0 == m1) return;
        out.push_back(Crossing{{int32_t(c.n[0]), int32_t(c.n[1]), int32_t(c.n[2]), int32_t(c.n[3])}, m0 ? 1 : 0});
    }

    void run(const Call& c, std::vector<Crossing>& out) const
    {
        if (minimal(c)) {
            test(c, out);
            return;
        }
        children(c, [&](const Call& x) { run(x, out); });
    }
};

// extract's triangle pair per crossing and first-use vertex numbering
// (dual_contouring.h:64-86), in enumeration order
struct Numbering {
    std::vector<int64_t> vertex_of;
    std::vector<int64_t> order;  // cell of each vertex, in creation order
    std::vector<uint32_t> tri;

    explicit Numbering(int64_t n_cells) : vertex_of(size_t(n_cells), -1) {}

    uint32_t vertex(int64_t n)
    {
        int64_t& v = vertex_of[size_t(n)];
        if (v < 0) {
            v = int64_t(order.size());
            order.push_back(n);
        }
        return uint32_t(v);
    }

    void add(const Crossing& x)
    {
        static const int tris[2][3] = {{0, 1, 3}, {0, 3, 2}};
        for (const auto& t : tris) {
            const uint32_t v0 = vertex(x.n[t[0]]), v1 = vertex(x.n[t[1]]), v2 = vertex(x.n[t[2]]);
            if (v0 == v1 || v1 == v2 || v2 == v0) continue;
            tri.push_back(v0);
            tri.push_back(x.flip ? v2 : v1);
            tri.push_back(x.flip ? v1 : v2);
        }
    }
};

// 4x4 float transform applied as Eigen's Matrix4f * Vector4f (columns
// accumulated left to right), rows 0-2 given as a 3x4 array
inline void apply_xform(const float* m, const float* v, float* out)
{
    for (int r = 0; r < 3; ++r) {
        float a = m[4 * r] * v[0];
        a = a + m[4 * r + 1] * v[1];
        a = a + m[4 * r + 2] * v[2];
        out[r] = a + m[4 * r + 3];
    }
}

}  // namespace

int dc_extract(const int32_t* cells, int64_t n_cells, const float* corner_f, const float* cell_vertex,
               mlods_mesh_s* m)
{
    Grid g;
    int rc = build_grid(cells, n_cells, g);
    if (rc != MLODS_OK) return rc;
    m->pos.clear();
    m->nrm.clear();
    m->tri.clear();
    const int64_t root = g.find(Cell{0, 0, 0, 0});
    if (root < 0) return MLODS_OK;  // minimal_edges::traverse starts at the root only
    if (n_cells >= (int64_t(1) << 31)) {
        set_last_error("dc extract: %lld cells exceed 32-bit cell indices", (long long)n_cells);
        return MLODS_ERR_CAPACITY;
    }
    const Walker w{g, corner_f};
    // the top of the recursion as an ordered list of independent calls
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<Call> tasks = {Call{0, 0, {root, 0, 0, 0}}};
    for (int round = 0; round < 8 && tasks.size() < size_t(16 * hw); ++round) {
        std::vector<Call> next;
        bool grew = false;
        for (const Call& c : tasks) {
            size_t before = next.size();
            if (!w.minimal(c)) w.children(c, [&](const Call& x) { next.push_back(x); });
            if (next.size() == before && w.minimal(c)) next.push_back(c);  // a minimal edge stays a task
            grew = grew || next.size() != before + 1;
        }
        tasks.swap(next);
        if (!grew) break;
    }
    // the calls run on host threads; their crossings concatenate in task order
    std::vector<std::vector<Crossing>> found(tasks.size());
    std::atomic<size_t> next_task{0};
    auto worker = [&]() {
        for (size_t t; (t = next_task.fetch_add(1)) < tasks.size();) w.run(tasks[t], found[t]);
    };
    std::vector<std::thread> pool;
    for (unsigned i = 1; i < hw && i < tasks.size(); ++i) pool.emplace_back(worker);
    worker();
    for (std::thread& th : pool) th.join();
    Numbering num(n_cells);
    for (const auto& list : found)
        for (const Crossing& x : list) num.add(x);
    m->pos.resize(num.order.size() * 3);
    m->nrm.assign(num.order.size() * 3, 0.f);
    for (size_t i = 0; i < num.order.size(); ++i)
        for (int a = 0; a < 3; ++a) m->pos[3 * i + size_t(a)] = cell_vertex[3 * num.order[i] + a];
    m->tri.swap(num.tri);
    return MLODS_OK;
}

// mesh::smoothMesh, upsample.h:55-78
void mesh_smooth(mlods_mesh_s* m)
{
    const size_t nv = m->pos.size() / 3;
    std::vector<float> acc(nv * 3, 0.f), val(nv, 0.f);
    const float* p = m->pos.data();
    for (size_t t = 0; t + 2 < m->tri.size(); t += 3) {
        const uint32_t a = m->tri[t], b = m->tri[t + 1], c = m->tri[t + 2];
        for (int k = 0; k < 3; ++k) {
            acc[3 * a + k] += p[3 * b + k] + p[3 * c + k];
            acc[3 * b + k] += p[3 * a + k] + p[3 * c + k];
            acc[3 * c + k] += p[3 * b + k] + p[3 * a + k];
        }
        val[a] += 2.f;
        val[b] += 2.f;
        val[c] += 2.f;
    }
    for (size_t v = 0; v < nv; ++v)
        for (int k = 0; k < 3; ++k) m->pos[3 * v + size_t(k)] = acc[3 * v + size_t(k)] / val[v];
}

// mesh::subdivideMesh, upsample.h:80-133
void mesh_subdivide(mlods_mesh_s* m)
{
    const size_t nt = m->tri.size() / 3;
    std::unordered_map<uint64_t, uint32_t> on_edge;
    on_edge.reserve(nt * 2);
    auto mid = [&](uint32_t i, uint32_t j) -> uint32_t {
        const uint64_t key = (uint64_t(std::min(i, j)) << 32) | uint64_t(std::max(i, j));
        auto it = on_edge.find(key);
        if (it != on_edge.end()) return it->second;
        const uint32_t id = uint32_t(m->pos.size() / 3);
        float q[3];
        for (int k = 0; k < 3; ++k) q[k] = (m->pos[3 * size_t(i) + k] + m->pos[3 * size_t(j) + k]) / 2.f;
        for (int k = 0; k < 3; ++k) m->pos.push_back(q[k]);
        on_edge.emplace(key, id);
        return id;
    };
    m->tri.reserve(nt * 12);
    for (size_t t = 0; t < nt; ++t) {
        const uint32_t a = m->tri[3 * t], b = m->tri[3 * t + 1], c = m->tri[3 * t + 2];
        const uint32_t ab = mid(a, b);
        const uint32_t bc = mid(c, b);
        const uint32_t ca = mid(c, a);
        m->tri[3 * t + 1] = ab;
        m->tri[3 * t + 2] = ca;
        const uint32_t more[9] = {ab, b, bc, ab, bc, ca, ca, bc, c};
        m->tri.insert(m->tri.end(), more, more + 9);
    }
    m->nrm.resize(m->pos.size(), 0.f);  // normals.resize: new vertices get (0, 0, 0)
}

void mesh_transform(mlods_mesh_s* m, const float* xform)
{
    for (size_t v = 0; v < m->pos.size() / 3; ++v) {
        float o[3];
        apply_xform(xform, &m->pos[3 * v], o);
        std::memcpy(&m->pos[3 * v], o, sizeof o);
    }
}

// APSS::project of the vertices in place (scene.cpp:1422-1428)
int mesh_project(mlods_tree_s* T, mlods_mesh_s* m, int iters, cudaStream_t s)
{
    const int64_t nv = int64_t(m->pos.size() / 3);
    if (nv == 0) return MLODS_OK;
    float* d = nullptr;
    MLODS_CUDA(cudaMalloc(&d, size_t(nv) * 36));
    auto done = [&](int rc) {
        cudaFree(d);
        return rc;
    };
    cudaError_t e = cudaMemcpyAsync(d, m->pos.data(), size_t(nv) * 12, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return done(cuda_fail(e, "mesh project: upload", __FILE__, __LINE__));
    int rc = project_buffers(T, nv, d, d + 3 * nv, d + 6 * nv, iters, -1.f, s);
    if (rc != MLODS_OK) return done(rc);
    m->nrm.resize(m->pos.size());
    e = cudaMemcpyAsync(m->pos.data(), d + 3 * nv, size_t(nv) * 12, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->nrm.data(), d + 6 * nv, size_t(nv) * 12, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return done(cuda_fail(e, "mesh project: download", __FILE__, __LINE__));
    return done(MLODS_OK);
}

}  // namespace mlods

using namespace mlods;

extern "C" {

int mlods_dc_extract(int64_t n_cells, const int32_t* cells, const float* corner_f, const float* cell_vertex,
                     mlods_mesh* out)
{
    if (!out || n_cells <= 0 || !cells || !corner_f || !cell_vertex) {
        set_last_error("dc extract: bad arguments");
        return MLODS_ERR_INVALID;
    }
    *out = nullptr;
    auto* m = new (std::nothrow) mlods_mesh_s();
    if (!m) {
        set_last_error("dc extract: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    const int rc = dc_extract(cells, n_cells, corner_f, cell_vertex, m);
    if (rc != MLODS_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return MLODS_OK;
}

int mlods_mesh_info(mlods_mesh m, int64_t* n_vertices, int64_t* n_triangles)
{
    if (!m) {
        set_last_error("null mesh");
        return MLODS_ERR_INVALID;
    }
    if (n_vertices) *n_vertices = m->nv();
    if (n_triangles) *n_triangles = m->nt();
    return MLODS_OK;
}

int mlods_mesh_get(mlods_mesh m, float* vertices, float* normals, uint32_t* indices)
{
    if (!m) {
        set_last_error("null mesh");
        return MLODS_ERR_INVALID;
    }
    if (m->dev) return dmesh_get(*m->dev, vertices, normals, indices, nullptr);
    if (vertices) std::memcpy(vertices, m->pos.data(), m->pos.size() * sizeof(float));
    if (normals) std::memcpy(normals, m->nrm.data(), m->nrm.size() * sizeof(float));
    if (indices) std::memcpy(indices, m->tri.data(), m->tri.size() * sizeof(uint32_t));
    return MLODS_OK;
}

int mlods_mesh_device_arrays(mlods_mesh m, const float** vertices, const float** normals, const uint32_t** indices)
{
    if (!m) {
        set_last_error("null mesh");
        return MLODS_ERR_INVALID;
    }
    if (!m->dev) {
        set_last_error("mesh device arrays: the mesh is in host memory");
        return MLODS_ERR_INVALID;
    }
    if (vertices) *vertices = dmesh_pos(*m->dev);
    if (normals) *normals = dmesh_nrm(*m->dev);
    if (indices) *indices = dmesh_tri(*m->dev);
    return MLODS_OK;
}

int mlods_mesh_stage_ms(mlods_mesh m, double* ms)
{
    if (!m || !ms) {
        set_last_error("mesh stage times: bad arguments");
        return MLODS_ERR_INVALID;
    }
    std::memcpy(ms, m->stage_ms, sizeof m->stage_ms);
    return MLODS_OK;
}

int mlods_mesh_free(mlods_mesh m)
{
    delete m;
    return MLODS_OK;
}

int mlods_mesh_transform(mlods_mesh m, const float* xform)
{
    if (!m || !xform) {
        set_last_error("mesh transform: bad arguments");
        return MLODS_ERR_INVALID;
    }
    if (m->dev) return dmesh_transform(*m->dev, xform, nullptr);
    mesh_transform(m, xform);
    return MLODS_OK;
}

int mlods_mesh_smooth(mlods_mesh m)
{
    if (!m) {
        set_last_error("null mesh");
        return MLODS_ERR_INVALID;
    }
    if (m->dev) {
        const int rc = dmesh_smooth(*m->dev, nullptr);
        if (rc != MLODS_OK) return rc;
        MLODS_CUDA(cudaStreamSynchronize(nullptr));
        return MLODS_OK;
    }
    mesh_smooth(m);
    return MLODS_OK;
}

int mlods_mesh_subdivide(mlods_mesh m)
{
    if (!m) {
        set_last_error("null mesh");
        return MLODS_ERR_INVALID;
    }
    if (uint64_t(m->nv()) + 3 * uint64_t(m->nt()) > uint64_t(UINT32_MAX)) {
        set_last_error("mesh subdivide: result would exceed 32-bit vertex indices");
        return MLODS_ERR_CAPACITY;
    }
    if (m->dev) {
        const int rc = dmesh_subdivide(*m->dev, nullptr);
        if (rc != MLODS_OK) return rc;
        MLODS_CUDA(cudaStreamSynchronize(nullptr));
        return MLODS_OK;
    }
    mesh_subdivide(m);
    return MLODS_OK;
}

int mlods_mesh_project(mlods_tree t, mlods_mesh m, int32_t n_iterations, void* stream)
{
    if (!t || !m || n_iterations < 0) {
        set_last_error("mesh project: bad arguments");
        return MLODS_ERR_INVALID;
    }
    MLODS_ON_DEVICE(t->device);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (m->dev) {
        const int rc = dmesh_project(t, *m->dev, n_iterations, s);
        if (rc != MLODS_OK) return rc;
        MLODS_CUDA(cudaStreamSynchronize(s));
        return MLODS_OK;
    }
    return mesh_project(t, m, n_iterations, s);
}

int mlods_dc_mesh(mlods_tree t, mlods_dcgrid g, int32_t use_normals, int32_t refine_rounds, void* stream,
                  mlods_mesh* out)
{
    if (!t || !g || !out || refine_rounds < 0) {
        set_last_error("dc mesh: bad arguments");
        return MLODS_ERR_INVALID;
    }
    MLODS_ON_DEVICE(t->device);
    *out = nullptr;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = int64_t(g->cells.size() / 4);
    if (n == 0) {
        set_last_error("dc mesh: empty grid");
        return MLODS_ERR_INVALID;
    }
    using clk = std::chrono::steady_clock;
    auto since = [](clk::time_point t0) { return std::chrono::duration<double, std::milli>(clk::now() - t0).count(); };
    auto* m = new (std::nothrow) mlods_mesh_s();
    DeviceMesh* dmp = dmesh_create();
    if (!m || !dmp) {
        delete m;
        dmesh_destroy(dmp);
        set_last_error("dc mesh: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    DeviceMesh& dm = *dmp;
    // corner field in device memory
    auto t0 = clk::now();
    DcField field;
    int rc = dc_field_device(t, n, g->cells.data(), false, g->max_depth, g->xform, use_normals, field, s);
    m->stage_ms[0] = since(t0);
    // extraction: on the device when the grid allows, else on the host
    t0 = clk::now();
    bool on_device = false;
    if (rc == MLODS_OK) {
        std::vector<int64_t> begin(size_t(g->max_depth) + 2, n);
        for (int64_t i = n - 1; i >= 0; --i) begin[size_t(g->cells[4 * size_t(i)])] = i;
        for (int d = g->max_depth; d >= 0; --d) begin[size_t(d)] = std::min(begin[size_t(d)], begin[size_t(d) + 1]);
        rc = dc_extract_device(field.cells, n, begin.data(), g->max_depth, field.cf, field.vert, dm, &on_device, s);
    }
    if (rc == MLODS_OK && !on_device) {
        std::vector<float> cf(size_t(n) * 8), vx(size_t(n) * 3);
        cudaError_t e = cudaMemcpyAsync(cf.data(), field.cf, cf.size() * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(vx.data(), field.vert, vx.size() * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        rc = e == cudaSuccess ? dc_extract(g->cells.data(), n, cf.data(), vx.data(), m)
                              : cuda_fail(e, "dc mesh: field download", __FILE__, __LINE__);
        if (rc == MLODS_OK)
            rc = dmesh_upload(dm, m->pos.data(), int64_t(m->pos.size() / 3), m->tri.data(),
                              int64_t(m->tri.size() / 3), s);
        if (rc == MLODS_OK && cudaStreamSynchronize(s) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "dc mesh: upload", __FILE__, __LINE__);
        std::vector<float>().swap(m->pos);  // the device copy is the mesh from here on
        std::vector<float>().swap(m->nrm);
        std::vector<uint32_t>().swap(m->tri);
    }
    dc_field_free(field);
    m->stage_ms[1] = since(t0);
    // the refinement loop stays in device memory (mesh_dev.cu); each stage
    // ends synchronised, so its host time is its device time plus launches
    auto stage = [&](int k, auto fn) {
        if (rc != MLODS_OK) return;
        const auto ts = clk::now();
        rc = fn();
        if (rc == MLODS_OK && cudaStreamSynchronize(s) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "dc mesh stage", __FILE__, __LINE__);
        m->stage_ms[k] += since(ts);
    };
    stage(2, [&] { return dmesh_transform(dm, g->xform, s); });  // scene.cpp:1400-1408
    stage(3, [&] { return dmesh_project(t, dm, 3, s); });
    for (int r = 0; rc == MLODS_OK && r < refine_rounds; ++r) {
        stage(4, [&] { return dmesh_smooth(dm, s); });
        stage(5, [&] { return dmesh_subdivide(dm, s); });
        stage(3, [&] { return dmesh_project(t, dm, 3, s); });
    }
    m->dev = dmp;  // the mesh stays in device memory; mlods_mesh_get copies it out
    if (rc != MLODS_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return MLODS_OK;
}

}  // extern "C"
