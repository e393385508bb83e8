// capi.cu -- extern "C" entry points of libmlods.so (declared in include/mlods.h).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include "dc.h"
#include "gather.cuh"
#include "project.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
thread_local char g_err[1024] = "";
std::atomic<int64_t> g_launches{0};
}  // namespace

int sm_count_for_current_device()
{
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (dev < 64 && cache[dev]) return cache[dev];
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    if (dev < 64) cache[dev] = v;
    return v;
}

// Stream-ordered scratch from a memory pool owned by the library (one per
// device), which keeps up to 8 GiB of freed scratch for reuse, so per-call
// buffers of a few GB cost neither a cudaMalloc nor a synchronising cudaFree.
namespace
{
cudaMemPool_t g_pools[64] = {};
std::mutex g_pools_mu;
}  // namespace

// The pool of device `dev`, or nullptr if none was made yet.
cudaMemPool_t scratch_pool(int dev)
{
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_pools_mu);
    return g_pools[dev];
}

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s)
{
    cudaMemPool_t* pools = g_pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64) return cudaMallocAsync(p, bytes, s);
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_pools_mu);
        if (!pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&pools[dev], &props);
            if (e != cudaSuccess) {
                pools[dev] = nullptr;
                return e;
            }
            uint64_t keep = uint64_t(8) << 30;
            e = cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) return e;
        }
        pool = pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

cudaError_t scratch_free(void* p, cudaStream_t s) { return p ? cudaFreeAsync(p, s) : cudaSuccess; }

// Unused memory of the current device's pool back to the system.
cudaError_t scratch_release()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = scratch_pool(dev);
    if (!pool) return cudaSuccess;
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return e;
    return cudaMemPoolTrimTo(pool, 0);
}

namespace
{
inline size_t al256(size_t v) { return (v + 255) / 256 * 256; }
}  // namespace

void note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

void set_last_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line)
{
    set_last_error("CUDA error %d (%s) in %s at %s:%d", int(e), cudaGetErrorString(e), what, file, line);
    // reset the runtime's last-error slot so that a later launch check does
    // not report this (non-sticky) error again
    (void)cudaGetLastError();
    return MLODS_ERR_CUDA;
}

int validate_kernel(const mlods_kernel* k)
{
    if (!k) {
        set_last_error("null kernel");
        return MLODS_ERR_INVALID;
    }
    if (k->type != MLODS_GAUSSIAN && k->type != MLODS_SINGULAR && k->type != MLODS_GAUSSIAN_MULTIPLE) {
        set_last_error("unknown kernel type %d", k->type);
        return MLODS_ERR_INVALID;
    }
    if (k->n_sigmas < 0) {
        set_last_error("n_sigmas=%d is negative", k->n_sigmas);
        return MLODS_ERR_INVALID;
    }
    if (k->n_sigmas > MLODS_INLINE_SIGMAS && !k->sigmas_ext) {
        set_last_error("n_sigmas=%d needs sigmas_ext (more than %d sigmas)", k->n_sigmas, MLODS_INLINE_SIGMAS);
        return MLODS_ERR_INVALID;
    }
    if (k->type == MLODS_GAUSSIAN_MULTIPLE && k->n_sigmas == 0) {
        set_last_error("multi-Gaussian kernel needs at least one sigma");
        return MLODS_ERR_INVALID;
    }
    if (k->type == MLODS_GAUSSIAN && !(k->sigma > 0.f)) {
        set_last_error("Gaussian kernel needs sigma > 0");
        return MLODS_ERR_INVALID;
    }
    return MLODS_OK;
}

namespace
{
// Device tables of long multi-Gaussian sigma lists, one per distinct list and
// device, kept until the process exits: trees, batches and server requests
// may share them and a captured graph may still read them, so they are never
// freed while the library is loaded.  At most kMaxSigmaTables per device.
constexpr size_t kMaxSigmaTables = 4096;
struct SigmaTable {
    int device;
    std::vector<float2> terms;
    float2* d;
};
std::vector<SigmaTable> g_sigma_tables;
std::mutex g_sigma_mu;

int intern_sigma_table(const std::vector<float2>& terms, const float2** out)
{
    int dev = 0;
    MLODS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_sigma_mu);
    size_t on_dev = 0;
    for (const SigmaTable& t : g_sigma_tables) {
        if (t.device != dev) continue;
        ++on_dev;
        if (t.terms.size() == terms.size() &&
            std::memcmp(t.terms.data(), terms.data(), terms.size() * sizeof(float2)) == 0) {
            *out = t.d;
            return MLODS_OK;
        }
    }
    if (on_dev >= kMaxSigmaTables) {
        set_last_error("more than %zu distinct long sigma lists on device %d", kMaxSigmaTables, dev);
        return MLODS_ERR_CAPACITY;
    }
    float2* d = nullptr;
    MLODS_CUDA(cudaMalloc(&d, terms.size() * sizeof(float2)));
    const cudaError_t e = cudaMemcpy(d, terms.data(), terms.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(e, "sigma table upload", __FILE__, __LINE__);
    }
    g_sigma_tables.push_back(SigmaTable{dev, terms, d});
    *out = d;
    return MLODS_OK;
}
}  // namespace

int make_kernel_consts(const mlods_kernel& k, KernelConsts* out)
{
    KernelConsts c;
    std::memset(&c, 0, sizeof c);
    const double log2e = 1.4426950408889634;
    c.type = k.type;
    c.shift = k.constant_shift;
    c.exponent = k.exponent;
    c.nsig = k.n_sigmas;
    const double sg = k.sigma;
    c.g_scale = float(-log2e / (2.0 * sg * sg));
    const double v = std::max(double(k.constant_shift), 1e-4);
    c.num = float(std::pow(v, double(k.exponent)));
    const float* sig = k.n_sigmas > MLODS_INLINE_SIGMAS ? k.sigmas_ext : k.sigmas;
    std::vector<float2> terms(static_cast<size_t>(std::max(k.n_sigmas, 0)));
    for (int i = 0; i < k.n_sigmas; ++i) {
        const double s = sig[i];
        terms[size_t(i)] = make_float2(float(-log2e / (2.0 * s * s)), float(1.0 / (s * s * s)));
    }
    if (k.n_sigmas <= MLODS_INLINE_SIGMAS) {
        for (int i = 0; i < k.n_sigmas; ++i) {
            c.ms_scale[i] = terms[size_t(i)].x;
            c.ms_w[i] = terms[size_t(i)].y;
        }
    } else if (k.type == MLODS_GAUSSIAN_MULTIPLE) {
        const int rc = intern_sigma_table(terms, &c.ms_ext);
        if (rc != MLODS_OK) return rc;
    }
    *out = c;
    return MLODS_OK;
}

// Kernel weight at squared distance d2 on the host, from the same constants
// the device uses (Kernel::w, Kernel.cpp:64-83).
static double kernel_weight_host(const KernelConsts& kc, double d2)
{
    const double ln2 = 0.6931471805599453;
    if (kc.type == MLODS_GAUSSIAN) return std::exp(d2 * kc.g_scale * ln2) + kc.shift;
    if (kc.type == MLODS_GAUSSIAN_MULTIPLE) {
        double s = 0.0;
        if (kc.nsig <= MLODS_INLINE_SIGMAS) {
            for (int i = 0; i < kc.nsig; ++i) s += std::exp(d2 * kc.ms_scale[i] * ln2) * kc.ms_w[i];
            return s;
        }
        std::vector<float2> t(static_cast<size_t>(kc.nsig));
        if (cudaMemcpy(t.data(), kc.ms_ext, t.size() * sizeof(float2), cudaMemcpyDeviceToHost) != cudaSuccess) {
            (void)cudaGetLastError();
            return 0.0;  // no pruning rather than a wrong threshold
        }
        for (const float2& v : t) s += std::exp(d2 * v.x * ln2) * v.y;
        return s;
    }
    return double(kc.num) * std::exp(-double(kc.exponent) * std::log(d2 + kc.shift));
}

// Ensures the tree's projection scratch holds `bytes` bytes (plus the stats
// block at its start).
static int ensure_scratch(mlods_tree_s* T, size_t bytes)
{
    const size_t need = al256(8 * sizeof(int64_t)) + bytes;
    if (T->d_scratch && T->scratch_bytes >= need) return MLODS_OK;
    // grow by half at least: callers with rising sizes (the grid generator's
    // levels, a refined mesh) reallocate a few times instead of every call
    const size_t grown = std::max(need, T->scratch_bytes + T->scratch_bytes / 2);
    if (T->d_scratch) cudaFree(T->d_scratch);
    T->d_scratch = nullptr;
    T->scratch_bytes = 0;
    MLODS_CUDA(cudaMalloc(&T->d_scratch, grown));
    T->scratch_bytes = grown;
    T->d_stats = static_cast<int64_t*>(T->d_scratch);
    return MLODS_OK;
}

void fill_cloud_args(const mlods_tree_s* T, CloudArgs& c, const float* d_q, float* d_out_p, float* d_out_n,
                     int iters, float step_max, int rule)
{
    c.nodes = T->nodes;
    c.o0 = T->origin[0];
    c.o1 = T->origin[1];
    c.o2 = T->origin[2];
    c.kc = T->kc;
    c.cutoff = T->params.cutoff;
    c.min_depth = T->params.min_depth;
    c.step_max = step_max < 0.f ? T->root_radius : step_max;
    c.rule = rule;
    c.n_iter = iters;
    c.conv_mode = T->params.converge;
    c.conv_tol = T->params.converge_tol;
    c.q_in = d_q;
    c.out_p = d_out_p;
    c.out_n = d_out_n;
    // in place, the buffer must stay in world coordinates for the next call
    c.local_out = (T->params.local_output != 0 && d_out_p != d_q) ? 1 : 0;
    c.qpw = T->params.queries_per_warp;
    // kernel-weight pruning: a subtree is dropped below prune_tol times the
    // weight of one average sample sitting at the query (w(0) x mean area)
    c.prune_thr = 0.f;
    if (T->params.prune_tol > 0.f && T->n_pts > 0)
        c.prune_thr = float(double(T->params.prune_tol) * kernel_weight_host(T->kc, 0.0) *
                            (double(T->root_mass) / double(T->n_pts)));
}

// Pruning margin of the neighbour searches: points may sit up to half a
// world-frame ulp outside their cell box (the reference classifies against the
// double split but stores the float one), and local coordinates are rounded.
static float gather_eps(const mlods_tree_s* T)
{
    float m = 0.f, ext = 0.f;
    for (int a = 0; a < 3; ++a) {
        m = std::max(m, std::max(std::fabs(T->bb[a]), std::fabs(T->BB[a])));
        ext = std::max(ext, T->BB[a] - T->bb[a]);
    }
    const float ulp = std::nextafter(m, INFINITY) - m;
    return 2.f * ulp + 1e-6f * ext + 1e-30f;
}

static void fill_gather_args(mlods_tree_s* T, GatherArgs& g)
{
    g.nodes = T->nodes;
    g.node_head = T->d_node_head;
    g.codes = T->d_codes;
    g.wspts = T->d_wspts;
    g.spts = T->d_spts;
    g.snrm = T->d_snrm;
    g.bounds = T->d_bounds;
    g.bounds_stride = T->bounds_stride;
    g.max_depth = T->max_depth;
    g.n_pts = T->n_pts;
    g.eps = gather_eps(T);
    g.o0 = T->origin[0];
    g.o1 = T->origin[1];
    g.o2 = T->origin[2];
    g.kc = T->kc;
    g.counter = reinterpret_cast<unsigned int*>(T->d_stats + 3);
    g.stats = T->d_stats;
    g.out_idx = nullptr;
    g.out_d2 = nullptr;
}

static int ensure_events(mlods_tree_s* T)
{
    if (!T->ev_start) {
        MLODS_CUDA(cudaEventCreate(&T->ev_start));
        MLODS_CUDA(cudaEventCreate(&T->ev_stop));
    }
    return MLODS_OK;
}

// Global, kNN and ball APSS projections (GlobalAPSS::project, GlobalAPSS.cu:203-235;
// APSSOctree::projectAPSSCPU, CPUUtils.cpp:690-737).
static int project_apss_impl(mlods_tree_s* T, int64_t n, const float* d_q, float* d_out_p, float* d_out_n, int iters,
                             float step_max, cudaStream_t s, const CallScratch* cs)
{
    int64_t* stats = nullptr;
    if (cs) {
        stats = cs->stats;
    } else {
        int rc = ensure_scratch(T, 0);
        if (rc != MLODS_OK) return rc;
        rc = ensure_events(T);
        if (rc != MLODS_OK) return rc;
        stats = T->d_stats;
    }
    cudaEvent_t ev0 = cs ? nullptr : T->ev_start, ev1 = cs ? nullptr : T->ev_stop;
    MLODS_CUDA(cudaMemsetAsync(stats, 0, 8 * sizeof(int64_t), s));
    const float sm = step_max < 0.f ? T->root_radius : step_max;
    const int mode = T->params.mode;
    if (mode == MLODS_MODE_GLOBAL) {
        GlobalArgs g;
        g.spts = T->d_spts;
        g.snrm = T->d_snrm;
        g.area = T->d_area;
        g.n_pts = T->n_pts;
        g.q_in = d_q;
        g.nq = n;
        g.out_p = d_out_p;
        g.out_n = d_out_n;
        g.n_iter = iters;
        g.step_max = sm;
        g.o0 = T->origin[0];
        g.o1 = T->origin[1];
        g.o2 = T->origin[2];
        g.kc = T->kc;
        if (ev0) MLODS_CUDA(cudaEventRecord(ev0, s));
        MLODS_CUDA(launch_global_apss(g, T->kc.type, s));
        if (ev1) {
            MLODS_CUDA(cudaEventRecord(ev1, s));
            T->timed = true;
        }
        return MLODS_OK;
    }
    GatherArgs g;
    fill_gather_args(T, g);
    g.counter = reinterpret_cast<unsigned int*>(stats + 3);
    g.stats = stats;
    g.q_in = d_q;
    g.nq = n;
    g.out_p = d_out_p;
    g.out_n = d_out_n;
    g.n_iter = iters;
    g.step_max = sm;
    g.k = T->params.knn;
    if (mode == MLODS_MODE_KNN && (g.k < 1 || g.k > MLODS_MAX_KNN)) {
        set_last_error("kNN: k=%d out of range [1, %d]", g.k, MLODS_MAX_KNN);
        return MLODS_ERR_CAPACITY;
    }
    g.ball_r = T->params.ball_radius;
    if (mode == MLODS_MODE_BALL && g.ball_r < 0.f) {
        // CPUUtils.cpp:706-707: a negative radius means 3 * sigmas[0]
        if (T->kernel.n_sigmas < 1) {
            set_last_error("ball mode: radius < 0 needs a kernel with sigmas");
            return MLODS_ERR_INVALID;
        }
        g.ball_r = T->kernel.sigmas[0] * 3;
    }
    if (ev0) MLODS_CUDA(cudaEventRecord(ev0, s));
    MLODS_CUDA(launch_gather(g, mode == MLODS_MODE_KNN ? kGatherKnnApss : kGatherBallApss, T->kc.type,
                             sm_count_for_current_device(), s));
    if (ev1) {
        MLODS_CUDA(cudaEventRecord(ev1, s));
        T->timed = true;
    }
    return MLODS_OK;
}

size_t project_call_bytes(const mlods_tree_s* T, int64_t n)
{
    if (T->params.mode != MLODS_MODE_MLOD) return 0;
    const bool reorder = T->params.reorder != 0 && n > 1;
    return reorder ? al256(size_t(n) * 4) + query_order_temp_bytes(n) : 0;
}

int project_buffers(mlods_tree_s* T, int64_t n, const float* d_q, float* d_out_p, float* d_out_n, int iters,
                    float step_max, cudaStream_t s, int rule_override, const CallScratch* cs)
{
    if (!T->kernel_set) {
        set_last_error("project: no kernel set (call mlods_set_kernel first)");
        return MLODS_ERR_STATE;
    }
    if (n <= 0 || n >= (int64_t(1) << 32)) {
        set_last_error("project: n=%lld out of range [1, 2^32)", (long long)n);
        return MLODS_ERR_INVALID;
    }
    if (iters < 0) {
        set_last_error("project: negative iteration count");
        return MLODS_ERR_INVALID;
    }
    if (T->params.mode != MLODS_MODE_MLOD)
        return project_apss_impl(T, n, d_q, d_out_p, d_out_n, iters, step_max, s, cs);
    const bool reorder = T->params.reorder != 0 && n > 1;
    const size_t order_bytes = project_call_bytes(T, n);
    char* base = nullptr;
    int64_t* stats = nullptr;
    if (cs) {
        if (cs->bytes < order_bytes) {
            set_last_error("project: call scratch of %zu bytes, %zu needed", cs->bytes, order_bytes);
            return MLODS_ERR_INVALID;
        }
        base = cs->base;
        stats = cs->stats;
    } else {
        const int rc = ensure_scratch(T, order_bytes);
        if (rc != MLODS_OK) return rc;
        base = static_cast<char*>(T->d_scratch) + al256(8 * sizeof(int64_t));
        stats = T->d_stats;
    }
    MLODS_CUDA(cudaMemsetAsync(stats, 0, 8 * sizeof(int64_t), s));
    uint32_t* d_order = nullptr;
    if (reorder) {
        d_order = reinterpret_cast<uint32_t*>(base);
        float ext = 0.f;
        for (int a = 0; a < 3; ++a) ext = std::max(ext, T->BB[a] - T->bb[a]);
        MLODS_CUDA(compute_query_order(d_q, n, T->origin, ext, d_order, base + al256(size_t(n) * 4), s));
    }
    const int rule = rule_override >= 0 ? rule_override : T->params.blend_rule;
    ProjectArgs a;
    fill_cloud_args(T, a.cloud, d_q, d_out_p, d_out_n, iters, step_max, rule);
    a.order = d_order;
    a.nq = n;
    a.counter = reinterpret_cast<unsigned int*>(stats + 3);
    a.stats = stats;
    a.queries_per_warp = T->params.queries_per_warp;
    if (cs) {
        MLODS_CUDA(launch_mlod_project(a, T->kc.type, rule, sm_count_for_current_device(), s));
        return MLODS_OK;
    }
    const int rc = ensure_events(T);
    if (rc != MLODS_OK) return rc;
    MLODS_CUDA(cudaEventRecord(T->ev_start, s));
    MLODS_CUDA(launch_mlod_project(a, T->kc.type, rule, sm_count_for_current_device(), s));
    MLODS_CUDA(cudaEventRecord(T->ev_stop, s));
    T->timed = true;
    return MLODS_OK;
}

}  // namespace mlods

using namespace mlods;

// Opens an entry point on a tree: rejects a null handle and makes the tree's
// device current until the function returns (a process may hold trees on
// several GPUs).
#define CHECK_TREE(t)                            \
    if (!(t)) {                                  \
        set_last_error("null tree handle");      \
        return MLODS_ERR_INVALID;                \
    }                                            \
    MLODS_ON_DEVICE((t)->device)

extern "C" {

const char* mlods_last_error(void) { return g_err; }

int mlods_version(void) { return 100; }

void mlods_default_params(mlods_params* p)
{
    if (!p) return;
    p->cutoff = 2.f;        // GPUUtils.h:63
    p->min_depth = 0;       // GPUUtils.h:64
    p->mode = MLODS_MODE_MLOD;
    p->knn = 20;            // CPUUtils.h:211
    p->ball_radius = 0.1f;  // CPUUtils.h:214
    p->blend_rule = MLODS_BLEND_GPU;
    p->reorder = 1;
    p->prune_tol = 0.f;
    p->converge = MLODS_CONVERGE_OFF;
    p->converge_tol = 0.f;
    p->local_output = 0;
    p->queries_per_warp = 1;
}

int mlods_tree_build_device(const float* d_pts, const float* d_nrm, int64_t n, int32_t max_depth, void* stream,
                            mlods_tree* out)
{
    if (!out || !d_pts || !d_nrm) {
        set_last_error("tree build: null argument");
        return MLODS_ERR_INVALID;
    }
    *out = nullptr;
    auto* T = new (std::nothrow) mlods_tree_s();
    if (!T) {
        set_last_error("tree build: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    mlods_default_params(&T->params);
    const int rc = build_tree(T, d_pts, d_nrm, n, max_depth, static_cast<cudaStream_t>(stream));
    if (rc != MLODS_OK) {
        free_tree_device(T);
        delete T;
        return rc;
    }
    *out = T;
    return MLODS_OK;
}

int mlods_tree_build(const float* pts, const float* nrm, int64_t n, int32_t max_depth, void* stream,
                     mlods_tree* out)
{
    if (!out || !pts || !nrm) {
        set_last_error("tree build: null argument");
        return MLODS_ERR_INVALID;
    }
    if (n <= 0) {
        set_last_error("tree build: n must be positive");
        return MLODS_ERR_INVALID;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float* d = nullptr;
    MLODS_CUDA(cudaMalloc(&d, size_t(n) * 6 * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(d, pts, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d + 3 * n, nrm, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(e, "tree build upload", __FILE__, __LINE__);
    }
    const int rc = mlods_tree_build_device(d, d + 3 * n, n, max_depth, stream, out);
    cudaStreamSynchronize(s);
    cudaFree(d);
    return rc;
}

int mlods_tree_free(mlods_tree t)
{
    if (!t) return MLODS_OK;
    MLODS_ON_DEVICE(t->device);
    free_tree_device(t);
    cudaFree(t->d_scratch);
    if (t->ev_start) cudaEventDestroy(t->ev_start);
    if (t->ev_stop) cudaEventDestroy(t->ev_stop);
    delete t;
    return MLODS_OK;
}

int mlods_tree_get_info(mlods_tree t, mlods_tree_info* info)
{
    CHECK_TREE(t);
    if (!info) {
        set_last_error("null info");
        return MLODS_ERR_INVALID;
    }
    info->n_points = t->n_pts;
    info->n_nodes = t->n_nodes;
    info->n_extra = t->n_extra;
    info->depth = t->depth;
    info->max_depth = t->max_depth;
    info->n_ties = t->n_ties;
    for (int a = 0; a < 3; ++a) {
        info->bbox_min[a] = t->bb[a];
        info->bbox_max[a] = t->BB[a];
        info->origin[a] = t->origin[a];
    }
    info->device_bytes = t->device_bytes;
    return MLODS_OK;
}

int mlods_tree_export(mlods_tree t, int32_t* depth, int32_t* parent, int32_t* first_child, int32_t* n_children,
                      int32_t* next_brother, int32_t* leaf_off, int32_t* leaf_cnt, int32_t* perm, float* bmin,
                      float* bmax, double* mom, float* area)
{
    CHECK_TREE(t);
    return export_tree(t, depth, parent, first_child, n_children, next_brother, leaf_off, leaf_cnt, perm, bmin, bmax,
                       mom, area);
}

int mlods_set_kernel(mlods_tree t, const mlods_kernel* k)
{
    CHECK_TREE(t);
    int rc = validate_kernel(k);
    if (rc != MLODS_OK) return rc;
    KernelConsts kc;
    rc = make_kernel_consts(*k, &kc);
    if (rc != MLODS_OK) return rc;
    t->kernel = *k;
    t->kernel.sigmas_ext = nullptr;  // the caller's array need not outlive this call
    if (k->n_sigmas > MLODS_INLINE_SIGMAS) {
        t->sigmas_long.assign(k->sigmas_ext, k->sigmas_ext + k->n_sigmas);
        t->kernel.sigmas[0] = k->sigmas_ext[0];
    } else {
        t->sigmas_long.clear();
    }
    t->kc = kc;
    t->kernel_set = true;
    return MLODS_OK;
}

int mlods_set_params(mlods_tree t, const mlods_params* p)
{
    CHECK_TREE(t);
    if (!p) {
        set_last_error("null params");
        return MLODS_ERR_INVALID;
    }
    if (p->mode < MLODS_MODE_MLOD || p->mode > MLODS_MODE_BALL || (p->blend_rule != MLODS_BLEND_GPU &&
                                                                   p->blend_rule != MLODS_BLEND_CPU)) {
        set_last_error("invalid mode %d or blend rule %d", p->mode, p->blend_rule);
        return MLODS_ERR_INVALID;
    }
    if (p->min_depth < 0) {
        set_last_error("min_depth must be >= 0");
        return MLODS_ERR_INVALID;
    }
    if (!(p->prune_tol >= 0.f)) {
        set_last_error("prune_tol must be >= 0");
        return MLODS_ERR_INVALID;
    }
    if (p->prune_tol > 0.f && p->queries_per_warp == 4) {
        set_last_error("prune_tol > 0 needs queries_per_warp 1 or 2");
        return MLODS_ERR_INVALID;
    }
    if (p->converge < MLODS_CONVERGE_OFF || p->converge > MLODS_CONVERGE_TOL) {
        set_last_error("unknown convergence mode %d", p->converge);
        return MLODS_ERR_INVALID;
    }
    if (p->queries_per_warp != 1 && p->queries_per_warp != 2 && p->queries_per_warp != 4) {
        set_last_error("queries_per_warp=%d: the walk takes 1, 2 or 4 queries per warp", p->queries_per_warp);
        return MLODS_ERR_INVALID;
    }
    // unchanged options are not written again, so that callers which re-apply
    // the same options before every call (the C++ mirror's projectCPU, run
    // from many host threads at once) only read them
    if (std::memcmp(&t->params, p, sizeof *p) != 0) t->params = *p;
    return MLODS_OK;
}

int mlods_queries_create(mlods_queries* out)
{
    if (!out) {
        set_last_error("queries_create: null argument");
        return MLODS_ERR_INVALID;
    }
    *out = new (std::nothrow) mlods_queries_s();
    if (!*out) {
        set_last_error("queries_create: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    return MLODS_OK;
}

int mlods_queries_free(mlods_queries q)
{
    if (!q) {
        set_last_error("null query buffer");
        return MLODS_ERR_INVALID;
    }
    cudaFree(q->d_q);
    cudaFree(q->d_qn);
    q->d_q = q->d_qn = nullptr;
    q->n = q->cap = 0;
    return MLODS_OK;
}

int mlods_queries_destroy(mlods_queries q)
{
    if (!q) return MLODS_OK;
    mlods_queries_free(q);
    delete q;
    return MLODS_OK;
}

int mlods_queries_upload(mlods_queries q, int64_t n, const float* pts, void* stream)
{
    if (!q || n <= 0 || !pts) {
        set_last_error("queries upload: null buffer, n <= 0 or null points");
        return MLODS_ERR_INVALID;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (q->cap < n) {
        mlods_queries_free(q);
        MLODS_CUDA(cudaMalloc(&q->d_q, size_t(n) * 3 * sizeof(float)));
        MLODS_CUDA(cudaMalloc(&q->d_qn, size_t(n) * 3 * sizeof(float)));
        q->cap = n;
    }
    q->n = n;
    MLODS_CUDA(cudaMemcpyAsync(q->d_q, pts, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
    MLODS_CUDA(cudaMemsetAsync(q->d_qn, 0, size_t(n) * 3 * sizeof(float), s));
    return MLODS_OK;
}

int mlods_project(mlods_tree t, mlods_queries q, int64_t n, int32_t n_iterations, float step_max, float* out_pts,
                  float* out_nrm, void* stream)
{
    CHECK_TREE(t);
    if (!q) {
        set_last_error("null query buffer");
        return MLODS_ERR_INVALID;
    }
    if (n == 0) {
        set_last_error("No points to project");  // Fastapss.cu:441-445
        return MLODS_ERR_INVALID;
    }
    if (!q->d_q || n > q->n) {
        set_last_error("project: %lld queries requested, %lld uploaded", (long long)n, (long long)q->n);
        return MLODS_ERR_STATE;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = project_buffers(t, n, q->d_q, q->d_q, q->d_qn, n_iterations, step_max, s);
    if (rc != MLODS_OK) return rc;
    if (out_pts)
        MLODS_CUDA(cudaMemcpyAsync(out_pts, q->d_q, size_t(n) * 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out_nrm)
        MLODS_CUDA(cudaMemcpyAsync(out_nrm, q->d_qn, size_t(n) * 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    return MLODS_OK;
}

int mlods_queries_reorganize(mlods_queries q, int64_t n_invalid, const uint32_t* invalid, uint32_t end_valid,
                             void* stream)
{
    if (!q) {
        set_last_error("null query buffer");
        return MLODS_ERR_INVALID;
    }
    if (n_invalid == 0) return MLODS_OK;
    if (n_invalid < 0 || !invalid || int64_t(end_valid) > q->n || n_invalid > int64_t(end_valid)) {
        set_last_error("queries_reorganize: bad arguments (n_invalid=%lld end_valid=%u uploaded=%lld)",
                       (long long)n_invalid, end_valid, (long long)q->n);
        return MLODS_ERR_INVALID;
    }
    for (int64_t i = 0; i < n_invalid; ++i)
        if (invalid[i] >= end_valid) {
            set_last_error("queries_reorganize: index %u >= end_valid %u", invalid[i], end_valid);
            return MLODS_ERR_INVALID;
        }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* d_inv = nullptr;
    MLODS_CUDA(cudaMalloc(&d_inv, size_t(n_invalid) * 4));
    cudaError_t e = cudaMemcpyAsync(d_inv, invalid, size_t(n_invalid) * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_reorganize(q->d_q, d_inv, n_invalid, end_valid, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_inv);
    if (e != cudaSuccess) return cuda_fail(e, "queries_reorganize", __FILE__, __LINE__);
    return MLODS_OK;
}

int mlods_project_host(mlods_tree t, int64_t n, const float* q, float* out_pts, float* out_nrm, int32_t n_iterations,
                       float step_max, int32_t blend_rule, void* stream)
{
    CHECK_TREE(t);
    if (n <= 0 || !q || !out_pts) {
        set_last_error("project_host: n must be positive, q and out_pts non-null");
        return MLODS_ERR_INVALID;
    }
    if (blend_rule != -1 && blend_rule != MLODS_BLEND_GPU && blend_rule != MLODS_BLEND_CPU) {
        set_last_error("project_host: unknown blend rule %d", blend_rule);
        return MLODS_ERR_INVALID;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Everything this call writes on the device -- queries, results, work
    // counter, statistics, query order -- is its own (stream-ordered memory
    // from the library's pool), so calls from several host threads on one
    // tree may overlap, as the reference's projectCPU calls do inside its
    // OpenMP loops (scene.cpp:982-986).
    const size_t io_bytes = al256(size_t(n) * 9 * sizeof(float));
    const size_t stats_bytes = al256(8 * sizeof(int64_t));
    const size_t call_bytes = project_call_bytes(t, n);
    void* mem = nullptr;
    MLODS_CUDA(scratch_alloc(&mem, io_bytes + stats_bytes + call_bytes, s));
    float* d = static_cast<float*>(mem);
    CallScratch cs;
    cs.stats = reinterpret_cast<int64_t*>(static_cast<char*>(mem) + io_bytes);
    cs.base = static_cast<char*>(mem) + io_bytes + stats_bytes;
    cs.bytes = call_bytes;
    cudaError_t e = cudaMemcpyAsync(d, q, size_t(n) * 12, cudaMemcpyHostToDevice, s);
    int rc = MLODS_OK;
    if (e == cudaSuccess)
        rc = project_buffers(t, n, d, d + 3 * n, d + 6 * n, n_iterations, step_max, s, blend_rule, &cs);
    if (e == cudaSuccess && rc == MLODS_OK) e = cudaMemcpyAsync(out_pts, d + 3 * n, size_t(n) * 12, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && rc == MLODS_OK && out_nrm)
        e = cudaMemcpyAsync(out_nrm, d + 6 * n, size_t(n) * 12, cudaMemcpyDeviceToHost, s);
    const cudaError_t ef = scratch_free(mem, s);
    if (e == cudaSuccess) e = ef;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (rc != MLODS_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "project_host", __FILE__, __LINE__);
    return MLODS_OK;
}

int mlods_project_device(mlods_tree t, int64_t n, const float* d_q, float* d_out_pts, float* d_out_nrm,
                         int32_t n_iterations, float step_max, void* stream)
{
    CHECK_TREE(t);
    if (!d_q || !d_out_pts || !d_out_nrm) {
        set_last_error("project_device: null buffer");
        return MLODS_ERR_INVALID;
    }
    return project_buffers(t, n, d_q, d_out_pts, d_out_nrm, n_iterations, step_max, static_cast<cudaStream_t>(stream));
}

int mlods_tune_schedule(mlods_tree t, int64_t n, const float* d_q, int32_t n_iterations, void* stream,
                        int32_t* chosen, float* ms)
{
    CHECK_TREE(t);
    if (!d_q || n <= 0 || n_iterations < 0) {
        set_last_error("tune schedule: bad arguments");
        return MLODS_ERR_INVALID;
    }
    if (!t->kernel_set) {
        set_last_error("tune schedule: no kernel set (call mlods_set_kernel first)");
        return MLODS_ERR_STATE;
    }
    if (t->params.mode != MLODS_MODE_MLOD) {
        set_last_error("tune schedule: only the MLoD walk has schedules");
        return MLODS_ERR_INVALID;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int cands[3] = {1, 2, 4};
    float* out = nullptr;
    MLODS_CUDA(scratch_alloc(reinterpret_cast<void**>(&out), size_t(n) * 6 * sizeof(float), s));
    const int saved = t->params.queries_per_warp;
    int best = saved;
    float best_ms = INFINITY;
    int rc = MLODS_OK;
    for (int i = 0; i < 3 && rc == MLODS_OK; ++i) {
        float this_ms = -1.f;
        if (!(cands[i] == 4 && t->params.prune_tol > 0.f)) {
            t->params.queries_per_warp = cands[i];
            // one run to load the kernel and settle the caches, one timed
            for (int rep = 0; rep < 2 && rc == MLODS_OK; ++rep)
                rc = project_buffers(t, n, d_q, out, out + 3 * n, n_iterations, -1.f, s);
            if (rc == MLODS_OK) {
                cudaError_t e = cudaEventSynchronize(t->ev_stop);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&this_ms, t->ev_start, t->ev_stop);
                if (e != cudaSuccess) rc = cuda_fail(e, "tune schedule: timing", __FILE__, __LINE__);
            }
            if (rc == MLODS_OK && this_ms < best_ms) {
                best_ms = this_ms;
                best = cands[i];
            }
        }
        if (ms) ms[i] = this_ms;
    }
    t->params.queries_per_warp = rc == MLODS_OK ? best : saved;
    const cudaError_t ef = scratch_free(out, s);
    if (rc != MLODS_OK) return rc;
    if (ef != cudaSuccess) return cuda_fail(ef, "tune schedule: free", __FILE__, __LINE__);
    if (chosen) *chosen = best;
    return MLODS_OK;
}

int mlods_tune_schedule_host(mlods_tree t, int64_t n, const float* q, int32_t n_iterations, int32_t* chosen,
                             float* ms)
{
    CHECK_TREE(t);
    if (!q || n <= 0) {
        set_last_error("tune schedule: bad arguments");
        return MLODS_ERR_INVALID;
    }
    // the sample staged in scratch memory on the legacy stream, then tuned there
    float* d = nullptr;
    MLODS_CUDA(scratch_alloc(reinterpret_cast<void**>(&d), size_t(n) * 12, nullptr));
    cudaError_t e = cudaMemcpyAsync(d, q, size_t(n) * 12, cudaMemcpyHostToDevice, nullptr);
    const int rc = e == cudaSuccess ? mlods_tune_schedule(t, n, d, n_iterations, nullptr, chosen, ms) : MLODS_OK;
    const cudaError_t ef = scratch_free(d, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "tune schedule: upload", __FILE__, __LINE__);
    if (rc != MLODS_OK) return rc;
    if (ef != cudaSuccess) return cuda_fail(ef, "tune schedule: free", __FILE__, __LINE__);
    return MLODS_OK;
}

int mlods_knn(mlods_tree t, int64_t n, const float* d_q, int32_t k, int32_t* d_idx, float* d_d2, void* stream)
{
    CHECK_TREE(t);
    if (n <= 0 || n >= (int64_t(1) << 32) || !d_q || !d_idx || !d_d2) {
        set_last_error("knn: bad arguments");
        return MLODS_ERR_INVALID;
    }
    if (k < 1 || k > MLODS_MAX_KNN) {
        set_last_error("knn: k=%d out of range [1, %d]", k, MLODS_MAX_KNN);
        return MLODS_ERR_CAPACITY;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = ensure_scratch(t, 0);
    if (rc != MLODS_OK) return rc;
    MLODS_CUDA(cudaMemsetAsync(t->d_stats, 0, 8 * sizeof(int64_t), s));
    GatherArgs g;
    fill_gather_args(t, g);
    g.q_in = d_q;
    g.nq = n;
    g.out_p = nullptr;
    g.out_n = nullptr;
    g.out_idx = d_idx;
    g.out_d2 = d_d2;
    g.k = k;
    g.ball_r = 0.f;
    g.n_iter = 1;
    g.step_max = 0.f;
    MLODS_CUDA(launch_gather(g, kGatherKnnOnly, t->kernel_set ? t->kc.type : MLODS_GAUSSIAN,
                             sm_count_for_current_device(), s));
    return MLODS_OK;
}

int mlods_knn_host(mlods_tree t, int64_t n, const float* q, int32_t k, int32_t* idx, float* d2)
{
    CHECK_TREE(t);
    if (n <= 0 || n >= (int64_t(1) << 32) || !q || !idx || !d2 || k < 1 || k > MLODS_MAX_KNN) {
        set_last_error("knn host: bad arguments");
        return MLODS_ERR_INVALID;
    }
    char* d = nullptr;
    const size_t qb = size_t(n) * 12, ib = size_t(n) * size_t(k) * 4;
    MLODS_CUDA(cudaMalloc(&d, qb + 2 * ib));
    float* d_q = reinterpret_cast<float*>(d);
    int32_t* d_idx = reinterpret_cast<int32_t*>(d + qb);
    float* d_d2 = reinterpret_cast<float*>(d + qb + ib);
    int rc = MLODS_OK;
    cudaError_t e = cudaMemcpy(d_q, q, qb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) rc = mlods_knn(t, n, d_q, k, d_idx, d_d2, nullptr);
    if (e == cudaSuccess && rc == MLODS_OK) e = cudaMemcpy(idx, d_idx, ib, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && rc == MLODS_OK) e = cudaMemcpy(d2, d_d2, ib, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (rc != MLODS_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "knn host", __FILE__, __LINE__);
    return MLODS_OK;
}

static int dcgrid_points(const float* pts, int64_t n, int32_t max_depth, const float* box_min, const float* box_max,
                         bool device, cudaStream_t s, mlods_dcgrid* out)
{
    if (!out || !box_min || !box_max) {
        set_last_error("dcgrid: null argument");
        return MLODS_ERR_INVALID;
    }
    *out = nullptr;
    auto* g = new (std::nothrow) mlods_dcgrid_s();
    if (!g) {
        set_last_error("dcgrid: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    bool handled = false;
    int rc = MLODS_OK;
    if (device) rc = dcgrid_from_points_device(pts, n, max_depth, box_min, box_max, s, g->cells, g->max_depth, &handled);
    if (rc == MLODS_OK && !handled) {
        if (device && pts && n > 0) {  // the host version reads host memory
            std::vector<float> h(size_t(n) * 3);
            cudaError_t e = cudaMemcpy(h.data(), pts, h.size() * sizeof(float), cudaMemcpyDefault);
            rc = e == cudaSuccess ? dcgrid_from_points(h.data(), n, max_depth, box_min, box_max, g->cells, g->max_depth)
                                  : cuda_fail(e, "dcgrid: points download", __FILE__, __LINE__);
        } else {
            rc = dcgrid_from_points(pts, n, max_depth, box_min, box_max, g->cells, g->max_depth);
        }
    }
    if (rc != MLODS_OK) {
        delete g;
        return rc;
    }
    // unit2bbox of the box (scene.cpp:1259-1269); the grid is not shifted
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 4; ++c) g->xform[4 * r + c] = 0.f;
        g->xform[4 * r + r] = box_max[r] - box_min[r];
        g->xform[4 * r + 3] = box_min[r];
    }
    *out = g;
    return MLODS_OK;
}

int mlods_dcgrid_from_points(const float* pts, int64_t n, int32_t max_depth, const float* box_min,
                             const float* box_max, mlods_dcgrid* out)
{
    return dcgrid_points(pts, n, max_depth, box_min, box_max, false, nullptr, out);
}

int mlods_dcgrid_from_points_device(const float* pts, int64_t n, int32_t max_depth, const float* box_min,
                                    const float* box_max, void* stream, mlods_dcgrid* out)
{
    return dcgrid_points(pts, n, max_depth, box_min, box_max, true, static_cast<cudaStream_t>(stream), out);
}

int mlods_dcgrid_adaptive(mlods_tree t, int32_t max_depth, int32_t cut, void* stream, mlods_dcgrid* out)
{
    CHECK_TREE(t);
    if (!out) {
        set_last_error("dcgrid adaptive: null output");
        return MLODS_ERR_INVALID;
    }
    *out = nullptr;
    auto* g = new (std::nothrow) mlods_dcgrid_s();
    if (!g) {
        set_last_error("dcgrid: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    const int rc = dcgrid_adaptive(t, max_depth, cut != 0, static_cast<cudaStream_t>(stream), g->cells,
                                   g->max_depth, g->xform, &g->n_projected);
    if (rc != MLODS_OK) {
        delete g;
        return rc;
    }
    *out = g;
    return MLODS_OK;
}

int mlods_dcgrid_xform(mlods_dcgrid g, float* xform, int64_t* n_projected)
{
    if (!g) {
        set_last_error("null dc grid");
        return MLODS_ERR_INVALID;
    }
    if (xform) std::memcpy(xform, g->xform, sizeof g->xform);
    if (n_projected) *n_projected = g->n_projected;
    return MLODS_OK;
}

int mlods_dcgrid_info(mlods_dcgrid g, int64_t* n_cells, int32_t* max_depth)
{
    if (!g) {
        set_last_error("null dc grid");
        return MLODS_ERR_INVALID;
    }
    if (n_cells) *n_cells = int64_t(g->cells.size() / 4);
    if (max_depth) *max_depth = g->max_depth;
    return MLODS_OK;
}

int mlods_dcgrid_cells(mlods_dcgrid g, int32_t* cells)
{
    if (!g || !cells) {
        set_last_error("null dc grid or output");
        return MLODS_ERR_INVALID;
    }
    std::memcpy(cells, g->cells.data(), g->cells.size() * sizeof(int32_t));
    return MLODS_OK;
}

int mlods_dcgrid_free(mlods_dcgrid g)
{
    delete g;
    return MLODS_OK;
}

int mlods_dc_evaluate(mlods_tree t, int64_t n_cells, const int32_t* cells, int32_t max_depth, const float* xform,
                      int32_t use_normals, float* corner_f, float* vertex, int32_t* n_cross,
                      int64_t* n_unique_corners, void* stream)
{
    CHECK_TREE(t);
    if (!t->kernel_set) {
        set_last_error("dc evaluate: no kernel set (call mlods_set_kernel first)");
        return MLODS_ERR_STATE;
    }
    return dc_evaluate(t, n_cells, cells, false, max_depth, xform, use_normals, corner_f, vertex, n_cross,
                       n_unique_corners, static_cast<cudaStream_t>(stream));
}

int mlods_dc_evaluate_device(mlods_tree t, int64_t n_cells, const int32_t* d_cells, int32_t max_depth,
                             const float* xform, int32_t use_normals, float* d_corner_f, float* d_vertex,
                             int32_t* d_n_cross, int64_t* n_unique_corners, void* stream)
{
    CHECK_TREE(t);
    if (!t->kernel_set) {
        set_last_error("dc evaluate: no kernel set (call mlods_set_kernel first)");
        return MLODS_ERR_STATE;
    }
    return dc_evaluate(t, n_cells, d_cells, true, max_depth, xform, use_normals, d_corner_f, d_vertex, d_n_cross,
                       n_unique_corners, static_cast<cudaStream_t>(stream));
}

int mlods_last_stats(mlods_tree t, int64_t* node_visits, int64_t* rounds, int32_t* max_stack, int64_t* overflows,
                     float* kernel_ms)
{
    CHECK_TREE(t);
    int64_t h[5] = {0, 0, 0, 0, 0};
    float ms = 0.f;
    if (t->timed) {
        MLODS_CUDA(cudaEventSynchronize(t->ev_stop));
        MLODS_CUDA(cudaEventElapsedTime(&ms, t->ev_start, t->ev_stop));
    }
    if (t->d_stats) MLODS_CUDA(cudaMemcpy(h, t->d_stats, sizeof h, cudaMemcpyDeviceToHost));
    if (node_visits) *node_visits = h[0];
    if (rounds) *rounds = h[4];
    if (max_stack) *max_stack = int32_t(h[1]);
    if (overflows) *overflows = h[2];
    if (kernel_ms) *kernel_ms = ms;
    return MLODS_OK;
}

int mlods_last_iterations(mlods_tree t, int64_t* iterations)
{
    CHECK_TREE(t);
    if (!iterations) {
        set_last_error("last iterations: null output");
        return MLODS_ERR_INVALID;
    }
    int64_t h[6] = {0, 0, 0, 0, 0, 0};
    if (t->d_stats) MLODS_CUDA(cudaMemcpy(h, t->d_stats, sizeof h, cudaMemcpyDeviceToHost));
    *iterations = h[5];
    return MLODS_OK;
}

int mlods_last_walk_counts(mlods_tree t, int64_t* lane_visits, int64_t* pruned)
{
    CHECK_TREE(t);
    int64_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (t->d_stats) MLODS_CUDA(cudaMemcpy(h, t->d_stats, sizeof h, cudaMemcpyDeviceToHost));
    if (lane_visits) *lane_visits = h[6];
    if (pruned) *pruned = h[7];
    return MLODS_OK;
}

int64_t mlods_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int mlods_release_scratch(void)
{
    MLODS_CUDA(scratch_release());
    return MLODS_OK;
}

}  // extern "C"
