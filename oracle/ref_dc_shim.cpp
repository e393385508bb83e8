// Test-only checker: the reference's own dual-contouring and point-set code,
// compiled from its sources by oracle/Makefile (target refdc) with the Eigen
// stand-in of oracle/stubs, behind a C ABI for the tests.  Never part of the
// library.
//
// Compiled from the reference (untouched):
//   sources/scene/upsample.cpp   OctreeGenerator::generate / generateFromPoints,
//                                uniformize / uniformizeFromPoints (grade,
//                                regularize_up, regularize_siblings, cut,
//                                retreiveCorrectRoot), mesh::smoothMesh /
//                                mesh::subdivideMesh (upsample.h:55-133)
//   sources/dual-contouring/octree.h, dual_contouring.h  (sorted_octree,
//                                minimal_edges::traverse, dual_contour::extract)
//   sources/apss/Pn.cpp          Pn::load (tinyply), Pn::normalize, Pn::order
//
// Restated here (scene.cpp needs Qt and OpenGL): the glue of
// scene::computeDualContouring (scene.cpp:1252-1452) between those pieces --
// the unit-to-box maps, the corner list, the corner values from one
// projection each, and the vertex projection / smoothing / subdivision loop.
//
// Every projection the reference code asks for goes through a callback, so a
// test can feed it the projections of the library under test and compare the
// grid, corner field and mesh logic bit for bit.
#define TINYPLY_IMPLEMENTATION
#include "scene/upsample.h"

#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

extern "C" {
// Projects n points in place (pts: 3 n floats), writing unit normals (zero on
// failure), with `iters` steps and the given step limit (< 0: the tree's box
// radius).  cpu_rule = 1 for APSS::projectCPU, 0 for APSS::project.
typedef void (*refdc_project_fn)(void* ctx, int64_t n, float* pts, float* nrm, int32_t iters, float step_max,
                                 int32_t cpu_rule);
}

// The reference defines these two APSS members in GPUUtils.cu, which is not
// compiled here; the callback object below overrides both.
void APSS::copyPointsToGPU(unsigned int, glm::vec3*) {}
void APSS::erasePointsFromGPU() {}

namespace
{
// An APSS whose projections come from the callback, following the
// copyPointsToGPU / project protocol of Fastapss (Fastapss.cu:439-455): project
// runs on the uploaded buffer in place and copies back on request.
class CallbackAPSS : public APSS
{
public:
    CallbackAPSS(refdc_project_fn fn, void* ctx) : m_fn(fn), m_ctx(ctx) { m_apssOctree = nullptr; }
    ~CallbackAPSS() override {}

    void project(unsigned int n, glm::vec3* outPts, glm::vec3* outNmls, unsigned int iters, Kernel const&,
                 float stepMax = -1.f) const override
    {
        if (n == 0 || n > m_buf.size()) return;
        m_nrm.assign(n, glm::vec3(0.f));
        m_fn(m_ctx, int64_t(n), &m_buf[0].x, &m_nrm[0].x, int32_t(iters), stepMax, 0);
        ++m_calls;
        m_projected += n;
        if (outPts) std::memcpy(outPts, m_buf.data(), size_t(n) * sizeof(glm::vec3));
        if (outNmls) std::memcpy(outNmls, m_nrm.data(), size_t(n) * sizeof(glm::vec3));
    }
    void copyToGPU(const Kernel&, unsigned int) override {}
    void eraseFromGPU() override {}
    void projectCPU(glm::vec3 const& q, glm::vec3& out, glm::vec3& outN, unsigned int iters, Kernel const&,
                    float stepMax = -1.f) const override
    {
        glm::vec3 p = q, n(0.f);
        m_fn(m_ctx, 1, &p.x, &n.x, int32_t(iters), stepMax, 1);
        out = p;
        outN = n;
    }
    void copyPointsToGPU(unsigned int n, glm::vec3* pts) override { m_buf.assign(pts, pts + n); }
    void erasePointsFromGPU() override { m_buf.clear(); }

    mutable int64_t m_calls = 0, m_projected = 0;

private:
    refdc_project_fn m_fn;
    void* m_ctx;
    mutable std::vector<glm::vec3> m_buf, m_nrm;
};

struct Grid {
    std::vector<int32_t> cells;  // (depth, x, y, z) in sorted_octree order
    int max_depth = 0;
    glm::vec3 new_diag{1.f}, new_origin{0.f};
    int64_t projected = 0;        // centre projections made by the generator
    sorted_octree<char> soct;
};

void grid_from_soct(Grid& g)
{
    g.cells.clear();
    g.cells.reserve(g.soct.size() * 4);
    for (size_t i = 0; i < g.soct.size(); ++i) {
        const octree_id& n = g.soct.id(i);
        g.cells.insert(g.cells.end(), {n.depth, n.pos[0], n.pos[1], n.pos[2]});
    }
    g.max_depth = g.soct.size() ? g.soct.max_depth() : 0;
}

// new2bbox = unit2bbox * sortedOctreeToUnit (scene.cpp:1257-1311) over the
// reference's [-1, 1]^3 zone
Eigen::Matrix4f new2bbox_of(const Grid& g)
{
    const aabb_octree octzone = {
        Eigen::AlignedBox3f(Eigen::Vector3f(-1.0f, -1.0f, -1.0f), Eigen::Vector3f(1.0f, 1.0f, 1.0f))};
    const Eigen::AlignedBox3f B = octzone.bounds();
    Eigen::Matrix4f unit2bbox = Eigen::Matrix4f::Zero();
    for (int a = 0; a < 3; ++a) {
        unit2bbox(a, a) = B.diagonal()[a];
        unit2bbox(a, 3) = B.min()[a];
    }
    unit2bbox(3, 3) = 1;
    Eigen::Matrix4f toUnit = Eigen::Matrix4f::Zero();
    for (int a = 0; a < 3; ++a) {
        toUnit(a, a) = g.new_diag[a];
        toUnit(a, 3) = g.new_origin[a];
    }
    toUnit(3, 3) = 1;
    return unit2bbox * toUnit;
}

glm::vec3 apply(const Eigen::Matrix4f& m, const Eigen::Vector3f& p)
{
    const Eigen::Vector4f v = m * Eigen::Vector4f(p.x(), p.y(), p.z(), 1.f);
    return glm::vec3(v.x(), v.y(), v.z());
}

struct Mesh {
    // corner field: the lattice corners of every cell and their values, in
    // the order the reference lists them (cell-major, corner c = 0..7)
    std::vector<int32_t> corner_keys;  // 3 ints per corner slot
    std::vector<float> corner_vals;    // one per corner slot
    // extraction output, vertices in the grid's unit frame
    std::vector<float> ext_vertices;
    std::vector<uint32_t> ext_indices;
    // after the transform, the projection and the refinement rounds
    std::vector<glm::vec3> vertices, normals;
    std::vector<uint32_t> indices;
};

void project_all(CallbackAPSS& apss, std::vector<glm::vec3>& v, std::vector<glm::vec3>& n, unsigned iters,
                 const Kernel& k)
{
    n.resize(v.size());
    apss.erasePointsFromGPU();
    apss.copyPointsToGPU(unsigned(v.size()), v.data());
    apss.project(unsigned(v.size()), v.data(), n.data(), iters, k);
}
}  // namespace

extern "C" {

// ---- grids --------------------------------------------------------------------
// scene::generate_adaptive_octree + uniformize (scene.cpp:155-167, :1296-1297):
// OctreeGenerator::generate(max_depth, &total), then uniformize(max_depth,
// total, soct, new_diag, new_origin, cut).
void* refdc_grid_adaptive(refdc_project_fn fn, void* ctx, int32_t max_depth, int32_t cut)
{
    auto g = std::make_unique<Grid>();
    CallbackAPSS apss(fn, ctx);
    Kernel k;
    OctreeGenerator gen(&apss, k);
    std::vector<octree_id> total;
    gen.generate(unsigned(max_depth), &total);
    uniformize(unsigned(max_depth), total, g->soct, g->new_diag, g->new_origin, cut != 0);
    g->projected = apss.m_projected;
    grid_from_soct(*g);
    return g.release();
}

// scene::generate_usual_octree + uniformizeFromPoints (scene.cpp:169-178,
// :1299): generateFromPoints(max_depth, Pn(points)) over [-1, 1]^3.
void* refdc_grid_points(const float* pts, int64_t n, int32_t max_depth)
{
    auto g = std::make_unique<Grid>();
    std::vector<glm::vec3> p(static_cast<size_t>(n));
    std::memcpy(p.data(), pts, size_t(n) * sizeof(glm::vec3));
    Pn pn(p);
    Kernel k;
    OctreeGenerator gen(nullptr, k);
    std::vector<octree_id> nodes = gen.generateFromPoints(unsigned(max_depth), pn);
    uniformizeFromPoints(nodes, g->soct, g->new_diag, g->new_origin);
    grid_from_soct(*g);
    return g.release();
}

int64_t refdc_grid_size(void* h) { return int64_t(static_cast<Grid*>(h)->cells.size() / 4); }
int32_t refdc_grid_max_depth(void* h) { return static_cast<Grid*>(h)->max_depth; }
int64_t refdc_grid_projected(void* h) { return static_cast<Grid*>(h)->projected; }
void refdc_grid_cells(void* h, int32_t* out)
{
    const Grid* g = static_cast<Grid*>(h);
    std::memcpy(out, g->cells.data(), g->cells.size() * sizeof(int32_t));
}
// rows 0-2 of new2bbox (12 floats, row-major)
void refdc_grid_xform(void* h, float* out)
{
    const Eigen::Matrix4f m = new2bbox_of(*static_cast<Grid*>(h));
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) out[4 * r + c] = m(r, c);
}
void refdc_grid_free(void* h) { delete static_cast<Grid*>(h); }

// ---- corner field, extraction and refinement ------------------------------------
// scene::computeDualContouring after the grid (scene.cpp:1311-1452).
void* refdc_mesh(void* grid, refdc_project_fn fn, void* ctx, int32_t refine_rounds)
{
    Grid& g = *static_cast<Grid*>(grid);
    auto m = std::make_unique<Mesh>();
    CallbackAPSS apss(fn, ctx);
    Kernel kern;
    const Eigen::Matrix4f new2bbox = new2bbox_of(g);
    const sorted_octree<char>& tree = g.soct;
    const size_t octSize = tree.size();

    // corners: 8 per cell on the deepest level's lattice, mapped to the tree
    // frame and projected once each, one iteration (scene.cpp:1361-1385)
    std::vector<glm::vec3> listOfCorners(octSize * 8), listOfNormals(octSize * 8), listOfProjected(octSize * 8);
    std::vector<Eigen::Vector3i> allCorners(octSize * 8);
    for (size_t i = 0; i < octSize; ++i) {
        const octree_id n = tree.id(i);
        for (unsigned c = 0; c < 8; ++c) {
            const float w = 1.0f / (1 << tree.max_depth());
            const int delta = 1 << (tree.max_depth() - n.depth);
            const Eigen::Vector3i p = delta * n.corner(c);
            allCorners[i * 8 + c] = p;
            const Eigen::Vector3f pf = p.cast<float>() * w;
            listOfCorners[i * 8 + c] = apply(new2bbox, pf);
        }
    }
    apss.erasePointsFromGPU();
    apss.copyPointsToGPU(unsigned(listOfCorners.size()), listOfCorners.data());
    apss.project(unsigned(listOfCorners.size()), listOfProjected.data(), listOfNormals.data(), 1, kern);

    std::unordered_map<Eigen::Vector3i, float, vec3i_hash> corners;
    for (size_t i = 0; i < listOfCorners.size(); ++i) {
        if (glm::length2(listOfNormals[i]) < 0.5f)  // failed projection: zero normal
            corners[allCorners[i]] = std::nanf("");
        else
            corners[allCorners[i]] = glm::dot((glm::vec3(listOfCorners[i]) - listOfProjected[i]), listOfNormals[i]);
    }
    m->corner_keys.reserve(allCorners.size() * 3);
    m->corner_vals.reserve(allCorners.size());
    for (size_t i = 0; i < allCorners.size(); ++i) {
        m->corner_keys.insert(m->corner_keys.end(), {allCorners[i][0], allCorners[i][1], allCorners[i][2]});
        m->corner_vals.push_back(corners[allCorners[i]]);
    }

    // the surface callback is only reached for a corner missing from the
    // map, which cannot happen here; the normal field is the zero field
    auto surface = [&](const Eigen::Vector3f& p) -> float {
        glm::vec3 pproj, nproj;
        const glm::vec3 originPt = apply(new2bbox, p);
        apss.projectCPU(originPt, pproj, nproj, 1, kern);
        return glm::dot((originPt - pproj), nproj);
    };
    auto computeNormals = [](const Eigen::Vector3f&) -> Eigen::Vector3f { return Eigen::Vector3f(0, 0, 0); };

    std::vector<oriented_point> verticesAndNormals;
    std::vector<uint32_t> indices;
    dual_contouring(tree, surface, computeNormals, corners).extract(verticesAndNormals, indices);
    m->ext_vertices.reserve(verticesAndNormals.size() * 3);
    for (const oriented_point& v : verticesAndNormals)
        m->ext_vertices.insert(m->ext_vertices.end(), {v.position.x(), v.position.y(), v.position.z()});
    m->ext_indices = indices;

    // to the tree frame, project 3 iterations, then refine (scene.cpp:1396-1452)
    std::vector<glm::vec3> vertices(verticesAndNormals.size()), normals(verticesAndNormals.size());
    for (size_t i = 0; i < verticesAndNormals.size(); ++i) {
        vertices[i] = apply(new2bbox, verticesAndNormals[i].position);
        normals[i] = glm::vec3(verticesAndNormals[i].normal.x(), verticesAndNormals[i].normal.y(),
                               verticesAndNormals[i].normal.z());
    }
    project_all(apss, vertices, normals, 3, kern);
    for (int r = 0; r < refine_rounds; ++r) {
        mesh::smoothMesh(vertices, indices);
        mesh::subdivideMesh(vertices, indices);
        normals.resize(vertices.size());
        project_all(apss, vertices, normals, 3, kern);
    }
    m->vertices = std::move(vertices);
    m->normals = std::move(normals);
    m->indices = std::move(indices);
    return m.release();
}

void refdc_mesh_sizes(void* h, int64_t* n_corner_slots, int64_t* n_ext_vertices, int64_t* n_ext_indices,
                      int64_t* n_vertices, int64_t* n_indices)
{
    const Mesh* m = static_cast<Mesh*>(h);
    *n_corner_slots = int64_t(m->corner_vals.size());
    *n_ext_vertices = int64_t(m->ext_vertices.size() / 3);
    *n_ext_indices = int64_t(m->ext_indices.size());
    *n_vertices = int64_t(m->vertices.size());
    *n_indices = int64_t(m->indices.size());
}
void refdc_mesh_get(void* h, int32_t* corner_keys, float* corner_vals, float* ext_vertices, uint32_t* ext_indices,
                    float* vertices, float* normals, uint32_t* indices)
{
    const Mesh* m = static_cast<Mesh*>(h);
    if (corner_keys) std::memcpy(corner_keys, m->corner_keys.data(), m->corner_keys.size() * sizeof(int32_t));
    if (corner_vals) std::memcpy(corner_vals, m->corner_vals.data(), m->corner_vals.size() * sizeof(float));
    if (ext_vertices) std::memcpy(ext_vertices, m->ext_vertices.data(), m->ext_vertices.size() * sizeof(float));
    if (ext_indices) std::memcpy(ext_indices, m->ext_indices.data(), m->ext_indices.size() * sizeof(uint32_t));
    if (vertices) std::memcpy(vertices, m->vertices.data(), m->vertices.size() * sizeof(glm::vec3));
    if (normals) std::memcpy(normals, m->normals.data(), m->normals.size() * sizeof(glm::vec3));
    if (indices) std::memcpy(indices, m->indices.data(), m->indices.size() * sizeof(uint32_t));
}
void refdc_mesh_free(void* h) { delete static_cast<Mesh*>(h); }

// ---- point sets (Pn.cpp) -------------------------------------------------------------
// Pn::load(path, factor, do_normalize): PLY through tinyply or the raw PN
// format, then Pn::normalize.  Returns the point count (0 on failure) and a
// handle for refpn_get.
void* refpn_load(const char* path, int32_t do_normalize, int64_t* n)
{
    auto p = std::make_unique<Pn>();
    p->load(path, 1.0f, do_normalize != 0);
    *n = int64_t(p->size());
    return p.release();
}
// positions, normals (may be empty: n_normals), offset (3) and norme (1)
void refpn_get(void* h, float* pts, float* nrm, int64_t* n_normals, float* offset, float* norme)
{
    Pn* p = static_cast<Pn*>(h);
    const auto& P = p->getPositions();
    const auto& N = p->getNormals();
    if (pts) std::memcpy(pts, P.data(), P.size() * sizeof(glm::vec3));
    if (nrm) std::memcpy(nrm, N.data(), N.size() * sizeof(glm::vec3));
    if (n_normals) *n_normals = int64_t(N.size());
    const glm::vec3 o = p->getOffset();
    if (offset) {
        offset[0] = o.x;
        offset[1] = o.y;
        offset[2] = o.z;
    }
    if (norme) *norme = p->getNorme();
}
void refpn_free(void* h) { delete static_cast<Pn*>(h); }

// Pn::order(grid) on a point set made from pts (Pn::initialize): the
// positions after the Morton reordering (Pn.cpp:388-445).
void refpn_order(const float* pts, int64_t n, int32_t grid, float* out)
{
    std::vector<glm::vec3> p(static_cast<size_t>(n));
    std::memcpy(p.data(), pts, size_t(n) * sizeof(glm::vec3));
    Pn pn(p);
    pn.order(unsigned(grid));
    std::memcpy(out, pn.getPositions().data(), size_t(n) * sizeof(glm::vec3));
}

}  // extern "C"
