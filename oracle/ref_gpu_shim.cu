// ref_gpu_shim.cu -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own GPU projection code (sources/apss/Fastapss.cu,
// which itself includes GPUUtils.cu and GlobalAPSS.cu, as the reference's
// CMake build does, CMakeLists.txt:15) for sm_100a and exposes a C ABI:
// the reference GPU results pin the GPU blend rule of the oracle, and its
// timing is the plain one-launch-per-call GPU baseline.  Built by
// oracle/Makefile into oracle/_ref/libmlods_refgpu.so.
//
// Safety: the reference kernel indexes depthStats[node.depth] and
// depthStats[depth + 1] in a MAX_DEPTH(12)-entry local array
// (Fastapss.cu:173-261), which is out of bounds for leaves at depth 12.  The
// shim refuses any tree whose depth is 12 or more, so every access the
// reference kernel makes stays in bounds.  It also refuses more than
// 65535 * 128 queries, beyond which computeNbBlocks folds the grid into .y
// (GPUUtils.cu:218-225).
#include "apss/Fastapss.cu"

#include <cstdint>
#include <cstdio>

namespace
{
struct RefGpu {
    APSSOctree* tree = nullptr;
    Fastapss* apss = nullptr;
    Kernel kernel;
};

struct RefGlobal {
    APSSOctree* tree = nullptr;
    GlobalAPSS* apss = nullptr;
    Kernel kernel;
};
}  // namespace

extern "C" {

void* refgpu_create(const float* pts, const float* nrm, int64_t n, int max_depth, int ktype, float sigma,
                    float exponent, float shift, const float* sigmas, int nsig, float cutoff, int min_depth,
                    char* err, int errlen)
{
    std::vector<glm::vec3> p(n), nn(n);
    for (int64_t i = 0; i < n; ++i) {
        p[i] = glm::vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        nn[i] = glm::vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
    }
    auto* r = new RefGpu();
    r->tree = new APSSOctree();
    r->tree->build(p, nn, true, unsigned(max_depth), 1);
    const unsigned depth = r->tree->get_root()->computeDepth();
    if (depth >= MAX_DEPTH) {
        std::snprintf(err, size_t(errlen), "tree depth %u: the reference kernel would index depthStats out of bounds",
                      depth);
        delete r->tree;
        delete r;
        return nullptr;
    }
    r->kernel.type = ktype == 0 ? Kernel::GAUSSIAN : (ktype == 1 ? Kernel::SINGULAR : Kernel::GAUSSIAN_MULTIPLE);
    r->kernel.sigma = sigma;
    r->kernel.exponent = exponent;
    r->kernel.constant_shift = shift;
    r->kernel.sigmas.assign(sigmas, sigmas + nsig);
    r->apss = new Fastapss(r->tree);
    r->apss->setScalingProtectionSphere(cutoff);
    r->apss->setMinDepth(unsigned(min_depth));
    r->apss->copyToGPU(r->kernel, unsigned(n));
    return r;
}

// Uploads n queries, runs `calls` Fastapss::project calls of iters_per_call
// iterations each (the app runs 10 calls of 1 iteration, scene.cpp:929-933,
// mainwindow.h:155), then copies the result back.  Returns the device time
// of the project calls in milliseconds (CUDA events on the default stream),
// or a negative value if n is out of range.
double refgpu_project(void* h, const float* q, int64_t n, int calls, int iters_per_call, float step_max,
                      float* out_p, float* out_n)
{
    if (n <= 0 || n > int64_t(65535) * 128) return -1.0;
    auto* r = static_cast<RefGpu*>(h);
    std::vector<glm::vec3> qq(n);
    for (int64_t i = 0; i < n; ++i) qq[i] = glm::vec3(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
    r->apss->copyPointsToGPU(unsigned(n), qq.data());
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    for (int c = 0; c < calls; ++c) r->apss->project(unsigned(n), nullptr, nullptr, unsigned(iters_per_call), r->kernel, step_max);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<glm::vec3> op(n), on(n);
    r->apss->project(unsigned(n), op.data(), on.data(), 0, r->kernel, step_max);
    for (int64_t i = 0; i < n; ++i) {
        out_p[3 * i] = op[i].x; out_p[3 * i + 1] = op[i].y; out_p[3 * i + 2] = op[i].z;
        out_n[3 * i] = on[i].x; out_n[3 * i + 1] = on[i].y; out_n[3 * i + 2] = on[i].z;
    }
    r->apss->erasePointsFromGPU();
    return double(ms);
}

// A new weight kernel for the same tree, through the reference's own
// APSS::updateKernel (GPUUtils.cu:466-472), as scene::setNewKernel does.
void refgpu_set_kernel(void* h, int ktype, float sigma, float exponent, float shift, const float* sigmas, int nsig)
{
    auto* r = static_cast<RefGpu*>(h);
    r->kernel.type = ktype == 0 ? Kernel::GAUSSIAN : (ktype == 1 ? Kernel::SINGULAR : Kernel::GAUSSIAN_MULTIPLE);
    r->kernel.sigma = sigma;
    r->kernel.exponent = exponent;
    r->kernel.constant_shift = shift;
    r->kernel.sigmas.assign(sigmas, sigmas + nsig);
    r->apss->updateKernel(r->kernel);
}

void refgpu_free(void* h)
{
    auto* r = static_cast<RefGpu*>(h);
    if (!r) return;
    delete r->apss;
    delete r->tree;
    delete r;
}

// The reference's GlobalAPSS (GlobalAPSS.cu:95-258): every query sums over
// all points, one projection step per project() call, and each call copies
// the points and normals back to the host (GlobalAPSS.cu:231-232).
void* refgpu_global_create(const float* pts, const float* nrm, int64_t n, int max_depth, int ktype, float sigma,
                           float exponent, float shift, const float* sigmas, int nsig)
{
    std::vector<glm::vec3> p(n), nn(n);
    for (int64_t i = 0; i < n; ++i) {
        p[i] = glm::vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        nn[i] = glm::vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
    }
    auto* r = new RefGlobal();
    r->tree = new APSSOctree();
    r->tree->build(p, nn, true, unsigned(max_depth), 1);
    r->kernel.type = ktype == 0 ? Kernel::GAUSSIAN : (ktype == 1 ? Kernel::SINGULAR : Kernel::GAUSSIAN_MULTIPLE);
    r->kernel.sigma = sigma;
    r->kernel.exponent = exponent;
    r->kernel.constant_shift = shift;
    r->kernel.sigmas.assign(sigmas, sigmas + nsig);
    r->apss = new GlobalAPSS(r->tree);
    r->apss->copyToGPU(r->kernel, unsigned(n));
    return r;
}

// Uploads n queries and runs `calls` GlobalAPSS::project calls of one step
// each (the reference's call pattern: scene.cpp:929-933).  Returns the
// device milliseconds of the calls (CUDA events on the default stream), or a
// negative value if n is out of the reference's launch range.
double refgpu_global_project(void* h, const float* q, int64_t n, int calls, float step_max, float* out_p,
                             float* out_n)
{
    if (n <= 0 || n > int64_t(65535) * 128) return -1.0;
    auto* r = static_cast<RefGlobal*>(h);
    std::vector<glm::vec3> qq(n), op(n), on(n);
    for (int64_t i = 0; i < n; ++i) qq[i] = glm::vec3(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
    r->apss->copyPointsToGPU(unsigned(n), qq.data());
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    for (int c = 0; c < calls; ++c) r->apss->project(unsigned(n), op.data(), on.data(), 1u, r->kernel, step_max);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int64_t i = 0; i < n; ++i) {
        out_p[3 * i] = op[i].x; out_p[3 * i + 1] = op[i].y; out_p[3 * i + 2] = op[i].z;
        out_n[3 * i] = on[i].x; out_n[3 * i + 1] = on[i].y; out_n[3 * i + 2] = on[i].z;
    }
    r->apss->erasePointsFromGPU();
    return double(ms);
}

void refgpu_global_free(void* h)
{
    auto* r = static_cast<RefGlobal*>(h);
    if (!r) return;
    delete r->apss;
    delete r->tree;
    delete r;
}

}  // extern "C"
