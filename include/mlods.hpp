// mlods.hpp -- C++ mirror of the reference's projection classes over the C ABI
// of libmlods.so (mlods.h).  Header-only; link with -lmlods.
//
// Same class names, member names, signatures and defaults as the reference:
//   Kernel       sources/apss/Kernel.h:24-60, Kernel.cpp:76-190
//   BBOX         sources/apss/CPUUtils.h:70-99
//   APSSOctree   sources/apss/CPUUtils.h:166-229 (build runs on the device)
//   APSS         sources/apss/GPUUtils.h:22-67
//   Fastapss     sources/apss/Fastapss.h:32-51
// so that the reference's scene/upsample callers compile against it with
// `using namespace mlods;` and `vec3` standing in for glm::vec3 (same layout:
// three floats; glm::vec3 pointers can be passed through reinterpret_cast).
//
// Differences (all documented at the call):
//   - errors throw mlods::Error instead of printing and exit()ing
//     (gpuErrchk, GPUUtils.cu:32-41);
//   - projectCPU evaluates the reference's CPU semantics on the device;
//   - stop() does not touch the CUDA profiler.
#pragma once

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "mlods.h"

namespace mlods
{

struct vec3 {
    float x = 0.f, y = 0.f, z = 0.f;
    vec3() = default;
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
static_assert(sizeof(vec3) == 12, "vec3 must match the layout of glm::vec3");

class Error : public std::runtime_error
{
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), code(code) {}
    int code;
};

inline void check(int rc)
{
    if (rc != MLODS_OK) throw Error(rc, std::string("mlods: ") + mlods_last_error());
}

class Kernel
{
public:
    enum KernelType { GAUSSIAN, SINGULAR, GAUSSIAN_MULTIPLE };  // Kernel.h:37

    float sigma = 2.f;  // Kernel::Kernel(), Kernel.cpp:76
    float exponent = 1.f;
    float constant_shift = 0.f;
    std::vector<float> sigmas;
    std::vector<float> fixedSigmas;
    float beginningSigma = 0.f;
    float factor = 0.f;
    unsigned nbOfComputedSigmas = 1;
    KernelType type = GAUSSIAN;

    // Kernel::updateSigmas, Kernel.cpp:172-190
    void updateSigmas(bool computedSigmas = true, float radius = 1.f)
    {
        if (computedSigmas) {
            sigmas.resize(nbOfComputedSigmas);
            sigmas[0] = beginningSigma;
            for (unsigned i = 1; i < nbOfComputedSigmas; i++) sigmas[i] = sigmas[i - 1] * factor;
        } else {
            sigmas = fixedSigmas;
        }
        sigma *= radius;
        for (float& s : sigmas) s *= radius;
    }

    // Kernel::w, Kernel.cpp:64-83 (host evaluation, double arithmetic)
    float w(vec3 const& p, vec3 const& eta) const
    {
        const float dx = p.x - eta.x, dy = p.y - eta.y, dz = p.z - eta.z;
        const float d2 = dx * dx + dy * dy + dz * dz;
        if (type == GAUSSIAN_MULTIPLE) {
            double s = 0.0;
            for (float sg : sigmas) s += std::exp(-d2 / (2.0 * sg * sg)) / (sg * sg * sg);
            return s == 0 ? constant_shift : float(s);
        }
        if (type == GAUSSIAN) return float(std::exp(-d2 / (2.0 * sigma * sigma)) + constant_shift);
        if (type == SINGULAR) {
            const float v = std::max(constant_shift, 0.0001f);
            return float(std::pow(v, exponent) / std::pow(d2 + constant_shift, exponent));
        }
        return 1.f;
    }

    mlods_kernel to_c() const
    {
        mlods_kernel k{};
        k.type = type == GAUSSIAN ? MLODS_GAUSSIAN : (type == SINGULAR ? MLODS_SINGULAR : MLODS_GAUSSIAN_MULTIPLE);
        k.sigma = sigma;
        k.exponent = exponent;
        k.constant_shift = constant_shift;
        k.n_sigmas = int32_t(sigmas.size());
        if (sigmas.size() > MLODS_INLINE_SIGMAS)
            k.sigmas_ext = sigmas.data();  // read while this Kernel is alive and unchanged
        else
            for (size_t i = 0; i < sigmas.size(); ++i) k.sigmas[i] = sigmas[i];
        return k;
    }
};

// BBOX, CPUUtils.h:70-99 (float arithmetic as the reference)
struct BBOX {
    vec3 bb, BB;
    float squareDiagonal() const
    {
        const float dx = BB.x - bb.x, dy = BB.y - bb.y, dz = BB.z - bb.z;
        return dx * dx + dy * dy + dz * dz;
    }
    float diagonal() const { return std::sqrt(squareDiagonal()); }
    float radius() const { return diagonal() / 2.f; }
    vec3 center() const { return vec3((bb.x + BB.x) / 2.f, (bb.y + BB.y) / 2.f, (bb.z + BB.z) / 2.f); }
    float squareRadius() const { return squareDiagonal() / 4.f; }
};

class APSS;

// Device-resident octree with per-node moments (CPUUtils.h:166-229).
class APSSOctree
{
    friend class APSS;

public:
    APSSOctree() = default;
    APSSOctree(const APSSOctree&) = delete;
    APSSOctree& operator=(const APSSOctree&) = delete;
    virtual ~APSSOctree() { mlods_tree_free(m_tree); }

    // APSSOctree::build, CPUUtils.cpp:540-569.  Builds on the device; only the
    // reference's settings (tight root box, one point per leaf) are accepted.
    void build(const std::vector<vec3>& i_points, std::vector<vec3> const& normals, bool updateRootBoundingBox = true,
               unsigned int maxDepth = 12, unsigned int maxNumberOfPointsPerLeaf = 1)
    {
        if (!updateRootBoundingBox || maxNumberOfPointsPerLeaf != 1)
            throw Error(MLODS_ERR_INVALID, "mlods: only updateRootBoundingBox=true, 1 point per leaf are supported");
        if (i_points.size() != normals.size() || i_points.empty())
            throw Error(MLODS_ERR_INVALID, "mlods: points and normals must be non-empty and of equal size");
        mlods_tree_free(m_tree);
        m_tree = nullptr;
        check(mlods_tree_build(&i_points[0].x, &normals[0].x, int64_t(i_points.size()), int32_t(maxDepth), nullptr,
                               &m_tree));
        m_points = i_points;  // the reference keeps the samples on the host too
        m_normals = normals;
        mlods_tree_info inf{};
        check(mlods_tree_get_info(m_tree, &inf));
        m_bbox.bb = vec3(inf.bbox_min[0], inf.bbox_min[1], inf.bbox_min[2]);
        m_bbox.BB = vec3(inf.bbox_max[0], inf.bbox_max[1], inf.bbox_max[2]);
        m_numberOfNodes = unsigned(inf.n_nodes);
        m_depth = unsigned(inf.depth);
        m_numberOfLeaves = unsigned(inf.n_points);
    }

    BBOX const& getBoundingBox() const { return m_bbox; }
    unsigned getNbOfLeaves() const { return m_numberOfLeaves; }
    unsigned nbOfNodes() const { return m_numberOfNodes; }
    unsigned computeDepth() const { return m_depth; }
    float getScalingProtectionSphere() const { return m_scalingProtectionSphere; }
    unsigned getMinDepth() { return m_minDepth; }
    void setScalingProtectionSphere(float val) { m_scalingProtectionSphere = val; }
    void setMinDepth(unsigned val) { m_minDepth = val; }

    // CPUUtils.cpp:674-688
    void knnMode(bool setMode, unsigned knn = 20)
    {
        m_knnMode = setMode;
        if (m_knnMode) m_ballMode = !setMode;
        m_knn = knn;
    }
    void ballMode(bool setMode, float ballRadius = 0.1f)
    {
        m_ballMode = setMode;
        if (m_ballMode) m_knnMode = !setMode;
        m_ballRadius = ballRadius;
    }
    bool isAPSS() { return m_knnMode || m_ballMode; }

    // CPUUtils.cpp:665-672: the k nearest samples of x (nearest first).
    void getKnn(vec3 const& x, unsigned k, std::vector<vec3>& neighbors) const
    {
        std::vector<int32_t> idx(k);
        std::vector<float> d2(k);
        check(mlods_knn_host(m_tree, 1, &x.x, int32_t(k), idx.data(), d2.data()));
        neighbors.clear();
        for (int32_t i : idx)
            if (i >= 0) neighbors.push_back(m_points[size_t(i)]);
    }

    // CPUUtils.cpp:638-663: the algebraic sphere u0 + u123.x + u4 |x|^2
    // fitted to the m_knn nearest samples of qStart, weights kernel.w, float
    // sums in world coordinates as the reference takes them.
    void cpuSphere(vec3 const& qStart, float& u0, vec3& u123, float& u4, Kernel const& kernel = Kernel()) const
    {
        std::vector<int32_t> idx(m_knn);
        std::vector<float> d2(m_knn);
        check(mlods_knn_host(m_tree, 1, &qStart.x, int32_t(m_knn), idx.data(), d2.data()));
        auto dot = [](vec3 const& a, vec3 const& b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
        float s_pn = 0.f, s_pp = 0.f, s_w = 0.f;
        vec3 s_p(0.f, 0.f, 0.f), s_n(0.f, 0.f, 0.f);
        for (int32_t i : idx) {
            if (i < 0) continue;
            const vec3& p = m_points[size_t(i)];
            const vec3& n = m_normals[size_t(i)];
            const float wi = kernel.w(p, qStart);
            s_pn += wi * dot(p, n);
            s_pp += wi * dot(p, p);
            s_p = vec3(s_p.x + wi * p.x, s_p.y + wi * p.y, s_p.z + wi * p.z);
            s_n = vec3(s_n.x + wi * n.x, s_n.y + wi * n.y, s_n.z + wi * n.z);
            s_w += wi;
        }
        const vec3 n_w(s_n.x / s_w, s_n.y / s_w, s_n.z / s_w), p_w(s_p.x / s_w, s_p.y / s_w, s_p.z / s_w);
        u4 = 0.5f * (s_pn - dot(s_p, n_w)) / (s_pp - dot(s_p, p_w));
        u123 = vec3((s_n.x - 2 * u4 * s_p.x) / s_w, (s_n.y - 2 * u4 * s_p.y) / s_w, (s_n.z - 2 * u4 * s_p.z) / s_w);
        u0 = -(dot(s_p, u123) + u4 * s_pp) / s_w;
    }

    mlods_tree handle() const { return m_tree; }

private:
    mlods_tree m_tree = nullptr;
    std::vector<vec3> m_points, m_normals;
    BBOX m_bbox;
    unsigned m_numberOfNodes = 0, m_depth = 0, m_numberOfLeaves = 0;
    float m_scalingProtectionSphere = 2.f;
    unsigned m_minDepth = 0;
    bool m_knnMode = false;
    unsigned m_knn = 20;
    bool m_ballMode = false;
    float m_ballRadius = 0.1f;
};

// Projection interface (GPUUtils.h:22-67).  Wraps an APSSOctree it does not own.
class APSS
{
public:
    APSS() { check(mlods_queries_create(&m_queries)); }
    APSS(const APSS&) = delete;
    APSS& operator=(const APSS&) = delete;
    virtual ~APSS() { mlods_queries_destroy(m_queries); }

    // Fastapss::project, Fastapss.cu:439-455: iterate n_iterations in place on
    // the device query buffer; copy back when the pointers are non-null.  As
    // in the reference, `kernel` is not used: the device kernel is the one
    // given to copyToGPU/updateKernel.
    virtual void project(unsigned int nbOfVectors, vec3* outputPoints, vec3* outputNormals, unsigned int n_iterations,
                         Kernel const& kernel, float stepMaxSize = -1.f) const
    {
        (void)kernel;
        if (nbOfVectors == 0) return;  // Fastapss.cu:441-445 prints and returns
        sync_params();
        check(mlods_project(tree(), m_queries, int64_t(nbOfVectors), int32_t(n_iterations), stepMaxSize,
                            outputPoints ? &outputPoints[0].x : nullptr, outputNormals ? &outputNormals[0].x : nullptr,
                            nullptr));
    }

    virtual void copyToGPU(const Kernel& kernel, unsigned int nbOfVectors)
    {
        (void)nbOfVectors;
        updateKernel(kernel);
    }
    virtual void eraseFromGPU() { erasePointsFromGPU(); }

    // APSSOctree::projectCPU semantics (CPU blend rule, CPUUtils.cpp:621-636),
    // evaluated on the device for one query.  Re-entrant: every call has its
    // own device buffers, work counter and statistics, and re-applying
    // unchanged options writes nothing, so host threads may call it at once
    // on one tree, as the reference's OpenMP loops do (scene.cpp:982-986).
    // Slow per call -- batch callers should use project().
    virtual void projectCPU(vec3 const& qStart, vec3& outputPoint, vec3& outputNormal, unsigned int n_iterations,
                            Kernel const& kernel = Kernel(), float stepMaxSize = -1.f) const
    {
        (void)kernel;
        sync_params();
        vec3 p, n;
        check(mlods_project_host(tree(), 1, &qStart.x, &p.x, &n.x, int32_t(n_iterations), stepMaxSize,
                                 MLODS_BLEND_CPU, nullptr));
        outputPoint = p;
        outputNormal = n;
    }

    void reorganizePoints(const std::vector<unsigned>* invalidPts, unsigned endValid)
    {
        check(mlods_queries_reorganize(m_queries, int64_t(invalidPts->size()), invalidPts->data(), endValid, nullptr));
    }

    void setScalingProtectionSphere(float val)
    {
        m_scalingProtectionSphere = val;
        m_apssOctree->setScalingProtectionSphere(val);
    }
    float getScalingProtectionSphere() { return m_scalingProtectionSphere; }
    void setMinDepth(unsigned val)
    {
        m_minDepth = val;
        m_apssOctree->setMinDepth(val);
    }
    unsigned getMinDepth() { return m_minDepth; }

    void stop() {}
    void eraseAndRestart()
    {
        eraseFromGPU();
        delete m_apssOctree;
        m_apssOctree = new APSSOctree();
    }

    virtual void copyPointsToGPU(unsigned int nbOfVectors, vec3* outputPoints)
    {
        check(mlods_queries_upload(m_queries, int64_t(nbOfVectors), &outputPoints[0].x, nullptr));
    }
    virtual void erasePointsFromGPU() { check(mlods_queries_free(m_queries)); }

    void updateKernel(Kernel const& kernel)
    {
        const mlods_kernel k = kernel.to_c();
        check(mlods_set_kernel(tree(), &k));
    }

    const APSSOctree* CPU() { return m_apssOctree; }

    int blend_rule = MLODS_BLEND_GPU;  // extension: select the CPU blend rule on the device
    // extension: the MLoD walk schedule (mlods_params.queries_per_warp): 1, 2
    // or 4 Morton-adjacent queries share one walk of the tree
    int queries_per_warp = 1;

    // extension: times the walk schedules on n sample queries (host array)
    // with n_iterations steps and keeps the fastest in queries_per_warp
    int tuneSchedule(unsigned int n, const vec3* sample, unsigned int n_iterations)
    {
        sync_params();
        int32_t chosen = queries_per_warp;
        check(mlods_tune_schedule_host(tree(), int64_t(n), &sample[0].x, int32_t(n_iterations), &chosen, nullptr));
        queries_per_warp = chosen;
        return chosen;
    }

protected:
    virtual int32_t mode() const
    {
        if (m_apssOctree->m_knnMode) return MLODS_MODE_KNN;
        if (m_apssOctree->m_ballMode) return MLODS_MODE_BALL;
        return MLODS_MODE_MLOD;
    }
    mlods_tree tree() const
    {
        if (!m_apssOctree || !m_apssOctree->m_tree) throw Error(MLODS_ERR_STATE, "mlods: octree not built");
        return m_apssOctree->m_tree;
    }
    void sync_params() const
    {
        mlods_params p;
        mlods_default_params(&p);
        p.cutoff = m_scalingProtectionSphere;
        p.min_depth = int32_t(m_minDepth);
        p.mode = mode();
        p.knn = int32_t(m_apssOctree->m_knn);
        p.ball_radius = m_apssOctree->m_ballRadius;
        p.blend_rule = blend_rule;
        p.queries_per_warp = queries_per_warp;
        check(mlods_set_params(tree(), &p));
    }

    float m_scalingProtectionSphere = 2.f;
    unsigned m_minDepth = 0;
    APSSOctree* m_apssOctree = nullptr;
    mlods_queries m_queries = nullptr;  // owned, as m_outPts/m_outNmls (GPUUtils.h:56-57)
};

// MLoD projection (Fastapss.h:32-51).
class Fastapss : public APSS
{
public:
    explicit Fastapss(APSSOctree* apssOctree) { m_apssOctree = apssOctree; }
    Fastapss(APSSOctree* apssOctree, const Kernel& kernel, unsigned int nbOfVectors) : Fastapss(apssOctree)
    {
        copyToGPU(kernel, nbOfVectors);
    }
};

// APSS over all points, no level of detail (GlobalAPSS.h:19-43); projectCPU is
// the reference's fast=false path (GlobalAPSS.cu:283-286).
class GlobalAPSS final : public APSS
{
public:
    explicit GlobalAPSS(APSSOctree* apssOctree) { m_apssOctree = apssOctree; }
    GlobalAPSS(APSSOctree* apssOctree, const Kernel& kernel, unsigned int nbOfVectors) : GlobalAPSS(apssOctree)
    {
        copyToGPU(kernel, nbOfVectors);
    }

    // GlobalAPSS.cu:288-291
    void cpuSphere(vec3 const& qStart, float& u0, vec3& u123, float& u4, Kernel const& kernel = Kernel()) const
    {
        m_apssOctree->cpuSphere(qStart, u0, u123, u4, kernel);
    }

protected:
    int32_t mode() const override
    {
        const int32_t m = APSS::mode();
        return m == MLODS_MODE_MLOD ? MLODS_MODE_GLOBAL : m;
    }
};

}  // namespace mlods
