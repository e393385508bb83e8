// batch.cu -- many resident trees projected by ONE persistent launch.
//
// No counterpart in the reference (one tree, one launch per call).  The batch
// orders each tree's queries in Morton order (one radix sort over all of
// them, the tree index as the key prefix, so every tree keeps its own query
// range) and runs the queue kernel (project.cu): its warps take a tree's
// queries two (or one) at a time from a device counter -- the trees with the
// most work first -- and walk them with the tree's own specialisation of the
// walk, so trees of very different sizes and kernels load-balance inside a
// single launch.  A schedule may instead run the largest trees in launches of
// their own (the single-tree kernel, whose arguments sit in the constant bank)
// before the shared launch of the rest.  With use_graph the memset / order /
// kernel sequence is captured once in a CUDA graph and replayed while the
// buffers, sizes and schedule stay the same.  The autotuner
// (mlods_batch_tune) times a set of schedules and keeps the fastest.
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
    int64_t* d_offsets = nullptr;
    mlods::BatchFrame* d_frames = nullptr;
    int64_t* d_stats = nullptr;  // statistics block (8 int64), one 64-bit slot counter per launch group of the
                                 // shared launch, then one 32-bit work counter per tree for launches of their own
    size_t stats_bytes = 0;
    void* d_order_buf = nullptr;
    size_t order_bytes = 0;
    // what the launches use (re-uploaded when it changes)
    std::vector<mlods::CloudArgs> h_clouds;
    std::vector<int64_t> h_offsets;
    // launch shape (the tuner's pick, or set by the caller)
    mlods_batch_schedule sched{0, 1, 100, mlods::kQueueMostWorkFirst, 0};
    int run_qpw = 1;                  // the walk schedule the launches use
    std::vector<int> h_solo;          // trees with a launch of their own
    std::vector<mlods::CloudArgs> h_qclouds;  // the other trees: the shared launch's arguments
    std::vector<int64_t> h_qbase, h_qlen;
    int walk_launches = 0;            // launches of the walk per call
    // the autotuner's last run: candidates and their device ms
    std::vector<mlods_batch_schedule> tune_cands;
    std::vector<float> tune_ms;
    // graph cache
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* g_q = nullptr;
    void* g_p = nullptr;
    void* g_n = nullptr;
    int64_t g_total = -1;
    int g_iters = -1;
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

void drop_graph(mlods_batch_s* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->g_total = -1;
}

// Enqueues the whole batch on s (capturable: no host synchronisation).
// timed: bracket the kernels with the batch's events.
int enqueue(mlods_batch_s* b, const float* d_q, int64_t total, bool timed, cudaStream_t s)
{
    const int n = int(b->trees.size());
    MLODS_CUDA(cudaMemsetAsync(b->d_stats, 0, b->stats_bytes, s));
    uint32_t* order = nullptr;
    if (b->sched.reorder) {
        order = static_cast<uint32_t*>(b->d_order_buf);
        void* tmp = static_cast<char*>(b->d_order_buf) + up256(size_t(total) * 4);
        MLODS_CUDA(compute_batch_order(d_q, total, b->d_offsets, n, b->d_frames, true, order, tmp, s));
    }
    const int sm = sm_count_for_current_device();
    if (timed) MLODS_CUDA(cudaEventRecord(b->ev0, s));
    // the largest trees first, each in a launch of its own: its slice of the
    // batch order, rebased to the tree's own query indices
    unsigned int* solo_counters =
        reinterpret_cast<unsigned int*>(b->d_stats + 8 + queue_groups(int(b->h_qclouds.size())));
    for (size_t k = 0; k < b->h_solo.size(); ++k) {
        const int i = b->h_solo[k];
        ProjectArgs pa;
        pa.cloud = b->h_clouds[size_t(i)];
        pa.order = order ? order + b->h_offsets[size_t(i)] : nullptr;
        pa.order_base = order ? uint32_t(b->h_offsets[size_t(i)]) : 0u;
        pa.nq = b->h_offsets[size_t(i) + 1] - b->h_offsets[size_t(i)];
        pa.counter = solo_counters + k;
        pa.stats = b->d_stats;
        pa.queries_per_warp = b->run_qpw;
        MLODS_CUDA(launch_mlod_project(pa, pa.cloud.kc.type, pa.cloud.rule, sm, s));
    }
    if (!b->h_qclouds.empty()) {
        QueueArgs a;
        a.clouds = b->h_qclouds.data();
        a.base = b->h_qbase.data();
        a.len = b->h_qlen.data();
        a.n_clouds = int(b->h_qclouds.size());
        a.order = order;
        a.counters = reinterpret_cast<unsigned long long*>(b->d_stats + 8);
        a.stats = b->d_stats;
        a.line_order = b->sched.line_order;
        MLODS_CUDA(launch_mlod_queue(a, b->run_qpw, sm, b->sched.grid_pct, s));
    }
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
        // each cloud's arguments address its own slice of the buffers
        fill_cloud_args(T, clouds[size_t(i)], d_q + 3 * offsets[i], d_p + 3 * offsets[i], d_n + 3 * offsets[i], iters,
                        -1.f, T->params.blend_rule);
        CloudArgs& c = clouds[size_t(i)];
        c.prune_thr = 0.f;  // the queue kernel walks without pruning
        float ext = 0.f;
        for (int a = 0; a < 3; ++a) ext = std::max(ext, T->BB[a] - T->bb[a]);
        frames[size_t(i)] = BatchFrame{T->origin[0], T->origin[1], T->origin[2], ext > 0.f ? 1.f / ext : 1.f,
                                       uint32_t(i)};
    }
    // one walk schedule for the whole batch: the schedule's, else the largest
    // the trees ask for (the queue kernel walks one or two queries per warp)
    int q = b->sched.queries_per_warp;
    if (!q)
        for (const CloudArgs& c : clouds) q = std::max(q, c.qpw);
    q = q >= 2 ? 2 : 1;
    if (q != b->run_qpw) drop_graph(b);
    b->run_qpw = q;
    for (CloudArgs& c : clouds) c.qpw = q;
    const bool same = b->h_clouds.size() == clouds.size() && b->h_offsets.size() == size_t(n + 1) &&
                      std::memcmp(b->h_clouds.data(), clouds.data(), clouds.size() * sizeof(CloudArgs)) == 0 &&
                      std::memcmp(b->h_offsets.data(), offsets, size_t(n + 1) * sizeof(int64_t)) == 0;
    if (!same) {
        drop_graph(b);
        MLODS_CUDA(cudaMemcpyAsync(b->d_offsets, offsets, size_t(n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        MLODS_CUDA(cudaMemcpyAsync(b->d_frames, frames.data(), frames.size() * sizeof(BatchFrame),
                                   cudaMemcpyHostToDevice, s));
        MLODS_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
        b->h_clouds = clouds;
        b->h_offsets.assign(offsets, offsets + n + 1);
    }
    // the trees with a launch of their own (the largest first) and the rest
    std::vector<int> solo;
    std::vector<CloudArgs> qclouds;
    std::vector<int64_t> qbase, qlen;
    for (int i = 0; i < n; ++i) {
        const int64_t len = offsets[i + 1] - offsets[i];
        if (len == 0) continue;
        if (b->sched.solo_min_queries > 0 && len >= b->sched.solo_min_queries) {
            solo.push_back(i);
        } else {
            qclouds.push_back(clouds[size_t(i)]);
            qbase.push_back(offsets[i]);
            qlen.push_back(len);
        }
    }
    std::stable_sort(solo.begin(), solo.end(), [&](int x, int y) {
        return (offsets[x + 1] - offsets[x]) * std::max(clouds[size_t(x)].n_iter, 1) >
               (offsets[y + 1] - offsets[y]) * std::max(clouds[size_t(y)].n_iter, 1);
    });
    if (solo != b->h_solo || qbase != b->h_qbase || qlen != b->h_qlen) drop_graph(b);
    b->h_solo = solo;
    b->h_qclouds = qclouds;
    b->h_qbase = qbase;
    b->h_qlen = qlen;
    b->walk_launches = int(solo.size()) + (qclouds.empty() ? 0 : queue_groups(int(qclouds.size())));
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
    // (a change of schedule, trees or offsets drops the graph where it is made)
    const bool hit = b->exec && b->g_q == d_q && b->g_p == d_p && b->g_n == d_n && b->g_total == total &&
                     b->g_iters == iters;
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
    // statistics, a 64-bit slot counter for each launch group of
    // kQueueMaxClouds trees, a 32-bit work counter for each tree
    const size_t n_groups = size_t(queue_groups(n_trees));
    b->stats_bytes = (8 * sizeof(int64_t) + n_groups * sizeof(uint64_t) + size_t(n_trees) * sizeof(unsigned int) +
                      255) / 256 * 256;
    cudaError_t e = cudaMalloc(&b->d_offsets, size_t(n_trees + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_frames, size_t(n_trees) * sizeof(BatchFrame));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_stats, b->stats_bytes);
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
    cudaFree(b->d_offsets);
    cudaFree(b->d_frames);
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
    if (!b || !offsets || !d_q || !d_out_pts || !d_out_nrm || n_iterations < 0) {
        set_last_error("batch_tune: bad arguments");
        return MLODS_ERR_INVALID;
    }
    MLODS_ON_DEVICE(b->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // walk schedule, query order, grid size, order of the trees, and launches
    // of their own for the trees that fill the GPU 4 or 16 times over
    const int64_t fill = project_resident_queries(2, sm_count_for_current_device());
    const mlods_batch_schedule cands[] = {
        {1, 1, 100, kQueueMostWorkFirst, 0},        {2, 1, 100, kQueueMostWorkFirst, 0},
        {2, 1, 100, kQueueBySpecialisation, 0},     {2, 0, 100, kQueueMostWorkFirst, 0},
        {2, 1, 85, kQueueMostWorkFirst, 0},         {2, 1, 100, kQueueBySpecialisation, 16 * fill},
        {2, 1, 100, kQueueBySpecialisation, 4 * fill}};
    float best = INFINITY;
    mlods_batch_schedule pick = cands[1];
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    MLODS_CUDA(cudaEventCreate(&t0));
    cudaError_t ce = cudaEventCreate(&t1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(t0);
        return cuda_fail(ce, "batch_tune: events", __FILE__, __LINE__);
    }
    int rc = MLODS_OK;
    b->tune_cands.clear();
    b->tune_ms.clear();
    for (const mlods_batch_schedule& c : cands) {
        b->sched = c;
        drop_graph(b);
        int64_t total = 0;
        rc = batch_prepare(b, offsets, d_q, d_out_pts, d_out_nrm, n_iterations, s, &total);
        if (rc != MLODS_OK) break;
        // one run to load the kernels and settle the caches, one timed
        rc = batch_run(b, d_q, d_out_pts, d_out_nrm, total, n_iterations, 0, s);
        if (rc != MLODS_OK) break;
        ce = cudaEventRecord(t0, s);
        if (ce == cudaSuccess) rc = batch_run(b, d_q, d_out_pts, d_out_nrm, total, n_iterations, 0, s);
        if (ce == cudaSuccess && rc == MLODS_OK) ce = cudaEventRecord(t1, s);
        if (ce == cudaSuccess && rc == MLODS_OK) ce = cudaEventSynchronize(t1);
        float ms = 0.f;
        if (ce == cudaSuccess && rc == MLODS_OK) ce = cudaEventElapsedTime(&ms, t0, t1);
        if (ce != cudaSuccess) rc = cuda_fail(ce, "batch_tune: timing", __FILE__, __LINE__);
        if (rc != MLODS_OK) break;
        b->tune_cands.push_back(c);
        b->tune_ms.push_back(ms);
        if (ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    b->sched = pick;
    drop_graph(b);
    return rc;
}

int mlods_batch_stats(mlods_batch b, int64_t* node_visits, int64_t* rounds, int64_t* overflows, float* kernel_ms,
                      int64_t* lane_visits, int32_t* walk_launches)
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
    int64_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float ms = 0.f;
    MLODS_CUDA(cudaEventSynchronize(b->ev1));
    MLODS_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    MLODS_CUDA(cudaMemcpy(h, b->d_stats, sizeof h, cudaMemcpyDeviceToHost));
    if (node_visits) *node_visits = h[0];
    if (rounds) *rounds = h[4];
    if (overflows) *overflows = h[2];
    if (kernel_ms) *kernel_ms = ms;
    if (lane_visits) *lane_visits = h[6];
    if (walk_launches) *walk_launches = b->walk_launches;
    return MLODS_OK;
}

int mlods_batch_get_schedule(mlods_batch b, mlods_batch_schedule* out)
{
    if (!b || !out) {
        set_last_error("batch_get_schedule: bad arguments");
        return MLODS_ERR_INVALID;
    }
    *out = b->sched;
    out->queries_per_warp = b->sched.queries_per_warp ? b->sched.queries_per_warp : b->run_qpw;
    return MLODS_OK;
}

int mlods_batch_set_schedule(mlods_batch b, const mlods_batch_schedule* sched)
{
    if (!b || !sched) {
        set_last_error("batch_set_schedule: bad arguments");
        return MLODS_ERR_INVALID;
    }
    const mlods_batch_schedule& c = *sched;
    if (c.queries_per_warp < 0 || c.queries_per_warp > 2 || (c.reorder != 0 && c.reorder != 1) ||
        c.grid_pct < 1 || c.grid_pct > 100 ||
        (c.line_order != kQueueMostWorkFirst && c.line_order != kQueueBySpecialisation) || c.solo_min_queries < 0) {
        set_last_error("batch_set_schedule: queries_per_warp in {0, 1, 2}, reorder in {0, 1}, grid_pct in [1, 100], "
                       "line_order in {0, 1}, solo_min_queries >= 0");
        return MLODS_ERR_INVALID;
    }
    b->sched = c;
    drop_graph(b);
    return MLODS_OK;
}

int mlods_batch_tune_results(mlods_batch b, int32_t max_candidates, mlods_batch_schedule* cands, float* ms,
                             int32_t* n_candidates)
{
    if (!b || max_candidates < 0 || !n_candidates) {
        set_last_error("batch_tune_results: bad arguments");
        return MLODS_ERR_INVALID;
    }
    const int n = int(b->tune_ms.size());
    *n_candidates = n;
    for (int i = 0; i < n && i < max_candidates; ++i) {
        if (cands) cands[i] = b->tune_cands[size_t(i)];
        if (ms) ms[i] = b->tune_ms[size_t(i)];
    }
    return MLODS_OK;
}

}  // extern "C"
