// noalloc.cu -- MLoD projection that allocates no device memory.
//
// mlods_project_device keeps its per-call scratch (the query processing
// order, the radix-sort buffers that compute it, the work counter and the
// statistics block) in a buffer owned by the tree, allocated with cudaMalloc
// on the first call and grown whenever a larger batch arrives.  Some callers
// cannot allow that: a frame loop with a fixed device-memory budget, code
// that runs while a caching allocator owns all free memory, a process that
// must reach its final footprint at start-up.  mlods_project_device_noalloc
// runs the same kernel with all of that scratch in one fixed array in device
// memory that belongs to the module (g_noalloc_scratch below), so a call
// allocates nothing; the price is an upper bound on the queries per call.
//
// Setup happens once per device on the first call (cudaGetSymbolAddress of
// the array, with the tree's device current); make that first call outside
// any stream capture.  The address belongs to the device's context: if the
// context is destroyed and recreated (cudaDeviceReset), the next call sees a
// new context identifier and repeats the setup, which allocates nothing.
// Every call reuses the same array: calls that overlap in time on one device
// (two streams, two host threads) race on it and must be serialised by the
// caller.
#include <algorithm>
#include <mutex>

#include "project.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
constexpr int64_t kNoAllocMaxQueries = MLODS_NOALLOC_MAX_QUERIES;
constexpr size_t kStatsBytes = 256;  // 8 int64 statistics, the work counter is [3]
// stats + order (4 B per query) + order temp (keys 2 x 8 B, values 4 B per
// query, sort histograms); checked against the exact need at setup
constexpr size_t kNoAllocScratchBytes = size_t(13) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
struct ScratchSetup {
    void* ptr = nullptr;           // device address of the array in that context
    unsigned long long ctx = 0;    // identifier of the context it was taken in (0: unknown)
};
ScratchSetup g_scratch[kMaxDevices];

inline size_t al256(size_t v) { return (v + 255) / 256 * 256; }

// Identifier of the calling thread's current context (the driver's
// cuCtxGetCurrent + cuCtxGetId, reached through the runtime so that the
// library does not link the driver library), or 0 when there is none or the
// driver cannot tell.
unsigned long long current_context_id()
{
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        (void)cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    void* ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx) return 0;
    unsigned long long id = 0;
    return get_id(ctx, &id) == 0 ? id : 0;
}

// Device address of this device's copy of the scratch array.
int scratch_for_current_device(char** out)
{
    int dev = 0;
    MLODS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("project_device_noalloc: device %d out of range", dev);
        return MLODS_ERR_CAPACITY;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    ScratchSetup& su = g_scratch[dev];
    if (!su.ptr || current_context_id() != su.ctx) {
        const size_t need = kStatsBytes + al256(size_t(kNoAllocMaxQueries) * 4) +
                            query_order_temp_bytes(kNoAllocMaxQueries);
        if (need > kNoAllocScratchBytes) {
            set_last_error("project_device_noalloc: scratch array (%zu bytes) smaller than the %zu bytes "
                           "%lld queries need", kNoAllocScratchBytes, need, (long long)kNoAllocMaxQueries);
            return MLODS_ERR_CAPACITY;
        }
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            su.ptr = nullptr;
            return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        }
        su.ptr = p;
        su.ctx = current_context_id();  // the context now exists
    }
    *out = static_cast<char*>(su.ptr);
    return MLODS_OK;
}

}  // namespace
}  // namespace mlods

using namespace mlods;

extern "C" int mlods_project_device_noalloc(mlods_tree t, int64_t n, const float* d_q, float* d_out_pts,
                                            float* d_out_nrm, int32_t n_iterations, float step_max, void* stream)
{
    if (!t) {
        set_last_error("null tree handle");
        return MLODS_ERR_INVALID;
    }
    MLODS_ON_DEVICE(t->device);
    if (!d_q || !d_out_pts || !d_out_nrm) {
        set_last_error("project_device_noalloc: null buffer");
        return MLODS_ERR_INVALID;
    }
    if (!t->kernel_set) {
        set_last_error("project_device_noalloc: no kernel set (call mlods_set_kernel first)");
        return MLODS_ERR_STATE;
    }
    if (t->params.mode != MLODS_MODE_MLOD) {
        set_last_error("project_device_noalloc: only the MLoD mode is supported");
        return MLODS_ERR_INVALID;
    }
    if (n_iterations < 0) {
        set_last_error("project_device_noalloc: negative iteration count");
        return MLODS_ERR_INVALID;
    }
    if (n <= 0) {
        set_last_error("project_device_noalloc: n=%lld must be positive", (long long)n);
        return MLODS_ERR_INVALID;
    }
    if (n > kNoAllocMaxQueries) {
        set_last_error("project_device_noalloc: n=%lld exceeds the fixed scratch capacity of %lld queries per "
                       "call (split the batch, or use mlods_project_device)",
                       (long long)n, (long long)kNoAllocMaxQueries);
        return MLODS_ERR_CAPACITY;
    }
    char* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc != MLODS_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t* stats = reinterpret_cast<int64_t*>(base);
    // the statistics and the work counter must start at zero
    MLODS_CUDA(cudaMemsetAsync(stats, 0, kStatsBytes, s));
    uint32_t* d_order = nullptr;
    if (t->params.reorder != 0 && n > 1) {
        d_order = reinterpret_cast<uint32_t*>(base + kStatsBytes);
        char* tmp = base + kStatsBytes + al256(size_t(n) * 4);
        float ext = 0.f;
        for (int a = 0; a < 3; ++a) ext = std::max(ext, t->BB[a] - t->bb[a]);
        MLODS_CUDA(compute_query_order(d_q, n, t->origin, ext, d_order, tmp, s));
    }
    const int rule = t->params.blend_rule;
    ProjectArgs a;
    fill_cloud_args(t, a.cloud, d_q, d_out_pts, d_out_nrm, n_iterations, step_max, rule);
    a.order = d_order;
    a.nq = n;
    a.counter = reinterpret_cast<unsigned int*>(stats + 3);
    a.stats = stats;
    a.queries_per_warp = t->params.queries_per_warp;
    MLODS_CUDA(launch_mlod_project(a, t->kc.type, rule, sm_count_for_current_device(), s));
    return MLODS_OK;
}
