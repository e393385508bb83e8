// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C ABI over the reference's own CPU implementation, compiled from the
// reference sources where they lie (sources/apss/CPUUtils.cpp, Kernel.cpp and
// sources/dual-contouring/kdTreeNN/kdTreeNN.h) by oracle/Makefile into
// oracle/_ref/libmlods_ref.so.  Tests use it to pin the oracle restatement
// against the reference's own results; the benchmark's reference arm times it.
//
// APSSOctree::projectCPU is protected and befriends a class named Fastapss
// (sources/apss/CPUUtils.h:163-168).  The GPU Fastapss lives in a CUDA file, so
// this shim declares its own Fastapss with one static member that forwards to
// projectCPU; nothing of the reference is modified.
#include "apss/CPUUtils.h"

#include <omp.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

class Fastapss
{
public:
    static void project(const APSSOctree* t, glm::vec3 const& q, glm::vec3& x, glm::vec3& n, unsigned iters,
                        bool fast, Kernel const& k, float step_max)
    {
        t->projectCPU(q, x, n, iters, fast, k, step_max);
    }
};

namespace
{
struct RefTree {
    APSSOctree tree;
    std::vector<const octreeNode*> bfs;  // breadth-first order
    int64_t n_pts = 0;
};

Kernel make_kernel(int type, float sigma, float exponent, float shift, const float* sigmas, int nsig)
{
    Kernel k;
    k.type = type == 0 ? Kernel::GAUSSIAN : (type == 1 ? Kernel::SINGULAR : Kernel::GAUSSIAN_MULTIPLE);
    k.sigma = sigma;
    k.exponent = exponent;
    k.constant_shift = shift;
    k.sigmas.assign(sigmas, sigmas + nsig);
    return k;
}
}  // namespace

extern "C" {

// Builds APSSOctree::build(points, normals, true, max_depth, 1) (CPUUtils.cpp:540-569).
// srand(seed) is called first: the reference breaks exact split ties with rand().
void* ref_tree_build(const float* pts, const float* nrm, int64_t n, int max_depth, unsigned seed)
{
    srand(seed);
    auto* rt = new RefTree();
    std::vector<glm::vec3> p(n), nn(n);
    for (int64_t i = 0; i < n; ++i) {
        p[i] = glm::vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        nn[i] = glm::vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
    }
    rt->tree.build(p, nn, true, unsigned(max_depth), 1);
    rt->n_pts = n;
    const octreeNode* root = rt->tree.get_root();
    rt->bfs.assign(root->nbOfNodes(), nullptr);
    std::vector<const octreeNode*> all = root->all_nodes();
    for (const octreeNode* nd : all) rt->bfs[nd->breadth_first_index] = nd;
    return rt;
}

void ref_tree_free(void* h) { delete static_cast<RefTree*>(h); }

int64_t ref_tree_num_nodes(void* h) { return int64_t(static_cast<RefTree*>(h)->bfs.size()); }

int ref_tree_depth(void* h) { return int(static_cast<RefTree*>(h)->tree.get_root()->computeDepth()); }

// Exports the tree in breadth-first order.  Relations follow getRelations
// (CPUUtils.cpp:213-234); stats are the float moments nodeapssNodeStats
// {s_ai, s_ai_ni[3], s_ai_pi[3], s_ai_pi_ni, s_ai_pi_pi}; perm lists each
// leaf's indices, leaves in breadth-first order.
void ref_tree_export(void* h, int32_t* depth, int32_t* parent, int32_t* first_child, int32_t* n_children,
                     int32_t* next_brother, int32_t* leaf_off, int32_t* leaf_cnt, int32_t* perm, float* bmin,
                     float* bmax, float* stats, float* area)
{
    auto* rt = static_cast<RefTree*>(h);
    const size_t nn = rt->bfs.size();
    std::vector<const octreeNode*> nodes(nn, nullptr);
    std::vector<relations> rel(nn);
    rt->tree.get_root()->getRelations(nodes, rel);
    int32_t pos = 0;
    for (size_t b = 0; b < nn; ++b) {
        const octreeNode* nd = nodes[b];
        depth[b] = int32_t(nd->depth);
        parent[b] = rel[b].father;
        first_child[b] = rel[b].firstChild;
        next_brother[b] = rel[b].nextBrother;
        n_children[b] = int32_t(nd->numberOfChildren);
        for (int a = 0; a < 3; ++a) {
            bmin[3 * b + a] = nd->boundingBox.bb[a];
            bmax[3 * b + a] = nd->boundingBox.BB[a];
        }
        const apssNodeStats& s = nd->nodeapssNodeStats;
        float* st = stats + 9 * b;
        st[0] = s.s_ai;
        st[1] = s.s_ai_ni.x; st[2] = s.s_ai_ni.y; st[3] = s.s_ai_ni.z;
        st[4] = s.s_ai_pi.x; st[5] = s.s_ai_pi.y; st[6] = s.s_ai_pi.z;
        st[7] = s.s_ai_pi_ni;
        st[8] = s.s_ai_pi_pi;
        if (nd->isLeaf()) {
            leaf_off[b] = pos;
            leaf_cnt[b] = int32_t(nd->indices.size());
            for (unsigned idx : nd->indices) perm[pos++] = int32_t(idx);
        } else {
            leaf_off[b] = -1;
            leaf_cnt[b] = 0;
        }
    }
    const auto& ps = rt->tree.getPointsApssNodeStats();
    for (int64_t i = 0; i < rt->n_pts; ++i) area[i] = ps[i].s_ai;
}

// Projects nq queries with the reference CPU path, an OpenMP loop shaped as
// scene::projectPointsOnCPU (scene.cpp:982-986), each query calling
// APSSOctree::projectCPU(q, x, n, n_iter, fast, kernel, step_max).
//   mode 0: MLoD (fast=true)   mode 1: global APSS (fast=false)
//   mode 2: kNN APSS (knnMode(true, k))   mode 3: ball APSS (ballMode(true, ball_r))
// Returns the wall time in seconds of the projection loop.
double ref_project(void* h, const float* q, float* out_p, float* out_n, int64_t nq, int n_iter, int ktype,
                   float sigma, float exponent, float shift, const float* sigmas, int nsig, float cutoff,
                   int min_depth, float step_max, int mode, int k, float ball_r, int nthreads)
{
    auto* rt = static_cast<RefTree*>(h);
    APSSOctree& t = rt->tree;
    t.setScalingProtectionSphere(cutoff);
    t.setMinDepth(unsigned(min_depth));
    t.knnMode(mode == 2, unsigned(k));
    t.ballMode(mode == 3, ball_r);
    if (mode != 2 && mode != 3) {
        t.knnMode(false, unsigned(k));
        t.ballMode(false, ball_r);
    }
    const Kernel kern = make_kernel(ktype, sigma, exponent, shift, sigmas, nsig);
    const bool fast = mode != 1;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < nq; ++i) {
        glm::vec3 qi(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
        glm::vec3 x = qi, n(0.f);
        Fastapss::project(&t, qi, x, n, unsigned(n_iter), fast, kern, step_max);
        out_p[3 * i] = x.x; out_p[3 * i + 1] = x.y; out_p[3 * i + 2] = x.z;
        out_n[3 * i] = n.x; out_n[3 * i + 1] = n.y; out_n[3 * i + 2] = n.z;
    }
    return omp_get_wtime() - t0;
}

// APSSOctree::cpuSphere (CPUUtils.cpp:638-663) at nq queries with the k
// nearest points: out = (u0, u123.x, u123.y, u123.z, u4) per query.
void ref_cpu_sphere(void* h, const float* q, int64_t nq, int k, int ktype, float sigma, float exponent, float shift,
                    const float* sigmas, int nsig, float* out)
{
    auto* rt = static_cast<RefTree*>(h);
    APSSOctree& t = rt->tree;
    t.knnMode(true, unsigned(k));
    const Kernel kern = make_kernel(ktype, sigma, exponent, shift, sigmas, nsig);
    for (int64_t i = 0; i < nq; ++i) {
        float u0 = 0.f, u4 = 0.f;
        glm::vec3 u123(0.f);
        t.cpuSphere(glm::vec3(q[3 * i], q[3 * i + 1], q[3 * i + 2]), u0, u123, u4, kern);
        out[5 * i] = u0;
        out[5 * i + 1] = u123.x;
        out[5 * i + 2] = u123.y;
        out[5 * i + 3] = u123.z;
        out[5 * i + 4] = u4;
    }
    t.knnMode(false, unsigned(k));
}

// Builds a kd-tree over the points with kdTree::build defaults (depth 12,
// 1 point per leaf) and returns k nearest neighbours, sorted by distance.
void ref_kdtree_knn(const float* pts, int64_t n, const float* q, int64_t nq, int k, int32_t* out_idx,
                    double* out_d2)
{
    std::vector<glm::vec3> p(n);
    for (int64_t i = 0; i < n; ++i) p[i] = glm::vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    kdTreeNN::kdTree<glm::vec3> kd;
    kd.build(p);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < nq; ++i) {
        kdTreeNN::searchResults res;
        kd.knearest(glm::vec3(q[3 * i], q[3 * i + 1], q[3 * i + 2]), unsigned(k), res, true);
        for (int j = 0; j < k; ++j) {
            out_idx[i * k + j] = j < int(res.size()) ? int32_t(res[j].idx) : -1;
            out_d2[i * k + j] = j < int(res.size()) ? res[j].sqrDist : -1.0;
        }
    }
}

}  // extern "C"
