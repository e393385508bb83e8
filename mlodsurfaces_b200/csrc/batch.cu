// batch.cu -- many resident trees projected by a few persistent launches.
//
// No counterpart in the reference (one tree, one launch per call).  The batch
// keeps per-tree launch arguments on the device, orders all queries by
// (tree, Morton code) with one radix sort, and runs, per kernel
// specialisation, mlod_batch_kernel over the smaller trees, whose warps pull
// queries from a shared counter across trees so that trees of very different
// sizes load-balance inside one launch; each large tree runs the single-tree
// kernel over its own slot range.  With use_graph the
// memset/order/kernel sequence is captured once in a CUDA graph and replayed
// while the buffers and sizes stay the same.  A small autotuner picks the
// query order (Morton or input order) and the grid size by timing.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "project.cuh"
#include "tree.cuh"

struct mlods_batch_s {
    std::vector<mlods_tree_s*> trees;
    int device = 0;
    // device state
    mlods::CloudArgs* d_clouds = nullptr;
    int64_t* d_offsets = nullptr;
    mlods::BatchFrame* d_frames = nullptr;
    int64_t* d_rank_slot = nullptr;
    int32_t* d_rank_cloud = nullptr;
    int64_t* d_stats = nullptr;  // stats block (8 int64) then one work counter per group
    std::vector<mlods::BatchGroup> groups;
    void* d_order_buf = nullptr;
    size_t order_bytes = 0;
    std::vector<mlods::CloudArgs> h_clouds;  // last uploaded
    std::vector<int64_t> h_offsets;
    // tuned launch shape
    int reorder = 1;
    int grid_pct = 100;
    // graph cache
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* g_q = nullptr;
    void* g_p = nullptr;
    void* g_n = nullptr;
    int64_t g_total = -1;
    int g_iters = -1;
    int g_reorder = -1;
    int g_pct = -1;
    int g_kernels = 0;  // kernels one replay runs
    bool ran = false;   // the events hold a launch
    // graphs are captured on this private stream (the legacy default stream
    // cannot be captured) and launched on the caller's stream
    cudaStream_t cap_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace mlods
{
namespace
{
inline size_t up256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kStatsBytes = 8 * sizeof(int64_t) + kMaxBatchGroups * sizeof(unsigned int);

void drop_graph(mlods_batch_s* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->g_total = -1;
}

// Enqueues the whole batch on s (capturable: no host synchronisation).
// timed: bracket the kernel with the batch's events.
int enqueue(mlods_batch_s* b, const float* d_q, int64_t total, bool timed, cudaStream_t s)
{
    const int n = int(b->trees.size());
    MLODS_CUDA(cudaMemsetAsync(b->d_stats, 0, kStatsBytes, s));
    // the order groups the clouds by kernel specialisation (always needed),
    // with Morton order inside each cloud when reorder is on
    uint32_t* order = static_cast<uint32_t*>(b->d_order_buf);
    void* tmp = static_cast<char*>(b->d_order_buf) + up256(size_t(total) * 4);
    MLODS_CUDA(compute_batch_order(d_q, total, b->d_offsets, n, b->d_frames, b->reorder != 0, order, tmp, s));
    BatchArgs a;
    a.clouds = b->d_clouds;
    a.q_offsets = b->d_offsets;
    a.n_clouds = n;
    a.total = total;
    a.order = order;
    a.rank_slot = b->d_rank_slot;
    a.rank_cloud = b->d_rank_cloud;
    a.counters = reinterpret_cast<unsigned int*>(b->d_stats + 8);
    a.stats = b->d_stats;
    if (timed) MLODS_CUDA(cudaEventRecord(b->ev0, s));
    MLODS_CUDA(launch_mlod_batch(a, b->groups, sm_count_for_current_device(), b->grid_pct, s));
    if (timed) MLODS_CUDA(cudaEventRecord(b->ev1, s));
    if (timed) b->ran = true;
    return MLODS_OK;
}

}  // namespace

int batch_prepare(mlods_batch_s* b, const int64_t* offsets, const float* d_q, float* d_p, float* d_n, int iters,
                  cudaStream_t s, int64_t* total_out)
{
    const int n = int(b->trees.size());
    if (offsets[0] != 0) {
        set_last_error("batch: offsets[0] must be 0");
        return MLODS_ERR_INVALID;
    }
    for (int i = 0; i < n; ++i)
        if (offsets[i + 1] < offsets[i]) {
            set_last_error("batch: offsets must be non-decreasing");
            return MLODS_ERR_INVALID;
        }
    const int64_t total = offsets[n];
    if (total <= 0 || total >= (int64_t(1) << 32)) {
        set_last_error("batch: %lld queries out of range [1, 2^32)", (long long)total);
        return MLODS_ERR_INVALID;
    }
    std::vector<CloudArgs> clouds(static_cast<size_t>(n));
    std::vector<BatchFrame> frames(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        mlods_tree_s* T = b->trees[size_t(i)];
        if (!T->kernel_set) {
            set_last_error("batch: tree %d has no kernel", i);
            return MLODS_ERR_STATE;
        }
        if (T->params.mode != MLODS_MODE_MLOD) {
            set_last_error("batch: tree %d is not in MLoD mode", i);
            return MLODS_ERR_INVALID;
        }
        fill_cloud_args(T, clouds[size_t(i)], d_q + 3 * offsets[i], d_p + 3 * offsets[i], d_n + 3 * offsets[i], iters,
                        -1.f, T->params.blend_rule);
        float ext = 0.f;
        for (int a = 0; a < 3; ++a) ext = std::max(ext, T->BB[a] - T->bb[a]);
        frames[size_t(i)] = BatchFrame{T->origin[0], T->origin[1], T->origin[2], ext > 0.f ? 1.f / ext : 1.f, 0u};
    }
    std::vector<BatchGroup> groups;
    std::vector<int64_t> rank_slot(static_cast<size_t>(n) + 1);
    std::vector<int32_t> rank_cloud(static_cast<size_t>(n));
    plan_batch_groups(clouds.data(), offsets, n, frames.data(), rank_slot.data(), rank_cloud.data(), groups,
                      batch_solo_min_queries(sm_count_for_current_device()));
    if (int(groups.size()) > kMaxBatchGroups) {
        set_last_error("batch: %zu kernel specialisations exceed the %d supported", groups.size(), kMaxBatchGroups);
        return MLODS_ERR_CAPACITY;
    }
    const bool same = b->h_clouds.size() == clouds.size() && b->h_offsets.size() == size_t(n + 1) &&
                      std::memcmp(b->h_clouds.data(), clouds.data(), clouds.size() * sizeof(CloudArgs)) == 0 &&
                      std::memcmp(b->h_offsets.data(), offsets, size_t(n + 1) * sizeof(int64_t)) == 0;
    if (!same) {
        drop_graph(b);
        MLODS_CUDA(cudaMemcpyAsync(b->d_clouds, clouds.data(), clouds.size() * sizeof(CloudArgs),
                                   cudaMemcpyHostToDevice, s));
        MLODS_CUDA(cudaMemcpyAsync(b->d_offsets, offsets, size_t(n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        MLODS_CUDA(cudaMemcpyAsync(b->d_frames, frames.data(), frames.size() * sizeof(BatchFrame),
                                   cudaMemcpyHostToDevice, s));
        MLODS_CUDA(cudaMemcpyAsync(b->d_rank_slot, rank_slot.data(), rank_slot.size() * sizeof(int64_t),
                                   cudaMemcpyHostToDevice, s));
        MLODS_CUDA(cudaMemcpyAsync(b->d_rank_cloud, rank_cloud.data(), rank_cloud.size() * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, s));
        MLODS_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
        b->h_clouds = clouds;
        b->h_offsets.assign(offsets, offsets + n + 1);
        b->groups = groups;
    }
    const size_t need = up256(size_t(total) * 4) + query_order_temp_bytes(total);
    if (b->order_bytes < need) {
        drop_graph(b);
        cudaFree(b->d_order_buf);
        b->d_order_buf = nullptr;
        b->order_bytes = 0;
        MLODS_CUDA(cudaMalloc(&b->d_order_buf, need));
        b->order_bytes = need;
    }
    *total_out = total;
    return MLODS_OK;
}

int batch_run(mlods_batch_s* b, const float* d_q, float* d_p, float* d_n, int64_t total, int iters, int use_graph,
              cudaStream_t s)
{
    if (!use_graph) return enqueue(b, d_q, total, true, s);
    const bool hit = b->exec && b->g_q == d_q && b->g_p == d_p && b->g_n == d_n && b->g_total == total &&
                     b->g_iters == iters && b->g_reorder == b->reorder && b->g_pct == b->grid_pct;
    if (!hit) {
        drop_graph(b);
        if (!b->cap_stream) MLODS_CUDA(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
        cudaStream_t cs = b->cap_stream;
        MLODS_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        const int64_t before = launches_so_far();
        const int rc = enqueue(b, d_q, total, false, cs);
        const int kernels = int(launches_so_far() - before);
        note_launch(-kernels);  // captured, not run; each replay counts them
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(cs, &g);
        if (rc != MLODS_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        MLODS_CUDA(ce);
        b->graph = g;
        MLODS_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
        b->g_q = d_q;
        b->g_p = d_p;
        b->g_n = d_n;
        b->g_total = total;
        b->g_iters = iters;
        b->g_reorder = b->reorder;
        b->g_pct = b->grid_pct;
        b->g_kernels = kernels;
    }
    MLODS_CUDA(cudaEventRecord(b->ev0, s));
    MLODS_CUDA(cudaGraphLaunch(b->exec, s));
    MLODS_CUDA(cudaEventRecord(b->ev1, s));
    b->ran = true;
    note_launch(b->g_kernels);
    return MLODS_OK;
}

}  // namespace mlods

using namespace mlods;

extern "C" {

int mlods_batch_create(const mlods_tree* trees, int32_t n_trees, mlods_batch* out)
{
    if (!out || !trees || n_trees <= 0 || n_trees > (1 << 16)) {
        set_last_error("batch_create: need 1..65536 trees");
        return MLODS_ERR_INVALID;
    }
    *out = nullptr;
    auto* b = new (std::nothrow) mlods_batch_s();
    if (!b) {
        set_last_error("batch_create: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    for (int i = 0; i < n_trees; ++i) {
        if (!trees[i]) {
            delete b;
            set_last_error("batch_create: tree %d is null", i);
            return MLODS_ERR_INVALID;
        }
        if (trees[i]->device != trees[0]->device) {
            delete b;
            set_last_error("batch_create: tree %d is on device %d, tree 0 on device %d", i, trees[i]->device,
                           trees[0]->device);
            return MLODS_ERR_INVALID;
        }
        b->trees.push_back(trees[i]);
    }
    b->device = trees[0]->device;
    DeviceGuard guard(b->device);
    if (guard.err != cudaSuccess) {
        delete b;
        return cuda_fail(guard.err, "batch_create: select device", __FILE__, __LINE__);
    }
    cudaError_t e = cudaMalloc(&b->d_clouds, size_t(n_trees) * sizeof(CloudArgs));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_offsets, size_t(n_trees + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_frames, size_t(n_trees) * sizeof(BatchFrame));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_rank_slot, size_t(n_trees + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_rank_cloud, size_t(n_trees) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_stats, kStatsBytes);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) {
        mlods_batch_free(b);
        return cuda_fail(e, "batch_create", __FILE__, __LINE__);
    }
    *out = b;
    return MLODS_OK;
}

int mlods_batch_free(mlods_batch b)
{
    if (!b) return MLODS_OK;
    DeviceGuard guard(b->device);
    drop_graph(b);
    cudaFree(b->d_clouds);
    cudaFree(b->d_offsets);
    cudaFree(b->d_frames);
    cudaFree(b->d_rank_slot);
    cudaFree(b->d_rank_cloud);
    cudaFree(b->d_stats);
    cudaFree(b->d_order_buf);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    delete b;
    return MLODS_OK;
}

int mlods_batch_project(mlods_batch b, const int64_t* offsets, const float* d_q, float* d_out_pts, float* d_out_nrm,
                        int32_t n_iterations, int32_t use_graph, void* stream)
{
    if (!b || !offsets || !d_q || !d_out_pts || !d_out_nrm || n_iterations < 0) {
        set_last_error("batch_project: bad arguments");
        return MLODS_ERR_INVALID;
    }
    MLODS_ON_DEVICE(b->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t total = 0;
    int rc = batch_prepare(b, offsets, d_q, d_out_pts, d_out_nrm, n_iterations, s, &total);
    if (rc != MLODS_OK) return rc;
    return batch_run(b, d_q, d_out_pts, d_out_nrm, total, n_iterations, use_graph, s);
}

int mlods_batch_tune(mlods_batch b, const int64_t* offsets, const float* d_q, float* d_out_pts, float* d_out_nrm,
                     int32_t n_iterations, void* stream)
{
    if (!b || !offsets || !d_q || !d_out_pts || !d_out_nrm) {
        set_last_error("batch_tune: bad arguments");
        return MLODS_ERR_INVALID;
    }
    MLODS_ON_DEVICE(b->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t total = 0;
    int rc = batch_prepare(b, offsets, d_q, d_out_pts, d_out_nrm, n_iterations, s, &total);
    if (rc != MLODS_OK) return rc;
    struct Cand {
        int reorder, pct;
    };
    const Cand cands[] = {{1, 100}, {0, 100}, {1, 85}, {1, 70}};
    float best = INFINITY;
    Cand pick = cands[0];
    for (const Cand& c : cands) {
        b->reorder = c.reorder;
        b->grid_pct = c.pct;
        cudaEvent_t t0, t1;
        MLODS_CUDA(cudaEventCreate(&t0));
        MLODS_CUDA(cudaEventCreate(&t1));
        MLODS_CUDA(cudaEventRecord(t0, s));
        rc = batch_run(b, d_q, d_out_pts, d_out_nrm, total, n_iterations, 0, s);
        MLODS_CUDA(cudaEventRecord(t1, s));
        MLODS_CUDA(cudaEventSynchronize(t1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (rc != MLODS_OK) return rc;
        if (ms < best) {
            best = ms;
            pick = c;
        }
    }
    b->reorder = pick.reorder;
    b->grid_pct = pick.pct;
    drop_graph(b);
    return MLODS_OK;
}

int mlods_batch_stats(mlods_batch b, int64_t* node_visits, int64_t* rounds, int64_t* overflows, float* kernel_ms,
                      int32_t* reorder, int32_t* grid_pct)
{
    if (!b) {
        set_last_error("null batch");
        return MLODS_ERR_INVALID;
    }
    if (!b->ran) {
        set_last_error("batch_stats: no batch has run yet");
        return MLODS_ERR_STATE;
    }
    MLODS_ON_DEVICE(b->device);
    int64_t h[6] = {0, 0, 0, 0, 0, 0};
    float ms = 0.f;
    MLODS_CUDA(cudaEventSynchronize(b->ev1));
    MLODS_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    MLODS_CUDA(cudaMemcpy(h, b->d_stats, sizeof h, cudaMemcpyDeviceToHost));
    if (node_visits) *node_visits = h[0];
    if (rounds) *rounds = h[4];
    if (overflows) *overflows = h[2];
    if (kernel_ms) *kernel_ms = ms;
    if (reorder) *reorder = b->reorder;
    if (grid_pct) *grid_pct = b->grid_pct;
    return MLODS_OK;
}

}  // extern "C"
