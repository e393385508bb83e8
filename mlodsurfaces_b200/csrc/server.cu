// server.cu -- a projection server over resident trees.
//
// No counterpart in the reference, which projects one request at a time on
// the legacy stream.  Requests (a tree, n host query points, an iteration
// count, optionally their own weight kernel) are queued by any host thread
// and answered asynchronously.  Worker threads, one per CUDA stream, take
// what is queued (up to a batch size; large requests in pieces, small ones
// passing over those that do not fit) whenever they are free, stage it in
// pinned memory, and project the batch with the batched launches (each
// request or piece is one "cloud", with its own tree, kernel and iteration
// count), so copies of one batch overlap the projection of another.  Admission is bounded: a submit that would queue
// more than max_pending queries is refused (MLODS_ERR_CAPACITY) instead of
// growing host or device memory without limit.  Every wait has a timeout.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "project.cuh"
#include "tree.cuh"

namespace
{
using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    int tree = 0;
    int64_t n = 0;
    const float* q = nullptr;
    float* out_p = nullptr;
    float* out_n = nullptr;
    int iters = 0;
    bool own_kernel = false;
    mlods::KernelConsts kc{};
    Clock::time_point t_submit, t_done;
    int status = -1;  // -1 pending, else an MLODS_* code
    char error[256] = "";
    int64_t taken = 0;     // queries handed to batches
    int64_t finished = 0;  // queries whose batch has returned
    int piece_status = 0;  // first failing piece's status (MLODS_OK = 0 so far)
    bool cancelled = false;  // no further pieces will be handed out
};

// A contiguous range of one request's queries: requests larger than a batch
// run as several pieces, possibly in different batches on different streams.
struct Piece {
    Request* r;
    int64_t off, n;
};

struct Worker {
    cudaStream_t s = nullptr;
    float* h_stage = nullptr;  // pinned: 9 floats per query (q, p, n)
    size_t h_cap = 0;
    float* d_buf = nullptr;  // 9 floats per query
    mlods::CloudArgs* h_clouds = nullptr;  // pinned
    int64_t* h_offsets = nullptr;
    mlods::BatchFrame* h_frames = nullptr;
    mlods::CloudArgs* d_clouds = nullptr;
    int64_t* d_offsets = nullptr;
    mlods::BatchFrame* d_frames = nullptr;
    size_t cloud_cap = 0;
    mlods::QueueChunk* h_chunks = nullptr;  // pinned
    mlods::QueueChunk* d_chunks = nullptr;
    size_t chunk_cap = 0;
    int64_t* d_stats = nullptr;
    void* d_order = nullptr;  // query order and its sort buffers
    std::thread thread;
};

}  // namespace

struct mlods_server_s {
    std::vector<mlods_tree_s*> trees;
    mlods_server_config cfg{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, Request*> live;
    int64_t queued = 0;
    uint64_t next_ticket = 1;
    bool stopping = false;
    std::vector<Worker*> workers;
    // statistics
    int64_t completed = 0, batches = 0, queries = 0;
    double busy_ms = 0.0;
};

namespace mlods
{
namespace
{
inline size_t al256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kStatsBytes = 8 * sizeof(int64_t) + 256;  // statistics, then the chunk counter
constexpr int kServeChunk = 64;  // queries per work-queue chunk

int grow_pinned(void** p, size_t bytes)
{
    cudaFreeHost(*p);
    *p = nullptr;
    MLODS_CUDA(cudaMallocHost(p, bytes));
    return MLODS_OK;
}

int grow_device(void** p, size_t bytes)
{
    cudaFree(*p);
    *p = nullptr;
    MLODS_CUDA(cudaMalloc(p, bytes));
    return MLODS_OK;
}

int ensure_capacity(Worker& w, int64_t total, size_t n_req)
{
    if (w.h_cap < size_t(total)) {
        int rc = grow_pinned(reinterpret_cast<void**>(&w.h_stage), size_t(total) * 36);
        if (rc != MLODS_OK) return rc;
        rc = grow_device(reinterpret_cast<void**>(&w.d_buf), size_t(total) * 36);
        if (rc != MLODS_OK) return rc;
        const size_t ob = al256(size_t(total) * 4) + query_order_temp_bytes(total);
        rc = grow_device(&w.d_order, ob);
        if (rc != MLODS_OK) return rc;
        w.h_cap = size_t(total);
    }
    if (w.cloud_cap < n_req) {
        const size_t cap = std::max<size_t>(n_req, 64);
        int rc = grow_pinned(reinterpret_cast<void**>(&w.h_clouds), cap * sizeof(CloudArgs));
        if (rc == MLODS_OK) rc = grow_pinned(reinterpret_cast<void**>(&w.h_offsets), (cap + 1) * sizeof(int64_t));
        if (rc == MLODS_OK) rc = grow_pinned(reinterpret_cast<void**>(&w.h_frames), cap * sizeof(BatchFrame));
        if (rc == MLODS_OK) rc = grow_device(reinterpret_cast<void**>(&w.d_clouds), cap * sizeof(CloudArgs));
        if (rc == MLODS_OK) rc = grow_device(reinterpret_cast<void**>(&w.d_offsets), (cap + 1) * sizeof(int64_t));
        if (rc == MLODS_OK) rc = grow_device(reinterpret_cast<void**>(&w.d_frames), cap * sizeof(BatchFrame));
        if (rc != MLODS_OK) return rc;
        w.cloud_cap = cap;
    }
    return MLODS_OK;
}

// Projects one batch of requests on the worker's stream; host outputs are
// written before it returns.
int run_batch(mlods_server_s* S, Worker& w, const std::vector<Piece>& batch)
{
    int64_t total = 0;
    for (const Piece& pc : batch) total += pc.n;
    int rc = ensure_capacity(w, total, batch.size());
    if (rc != MLODS_OK) return rc;
    float* hq = w.h_stage;
    float* hp = w.h_stage + 3 * total;
    float* hn = w.h_stage + 6 * total;
    float* dq = w.d_buf;
    float* dp = w.d_buf + 3 * total;
    float* dn = w.d_buf + 6 * total;
    int64_t off = 0;
    for (size_t i = 0; i < batch.size(); ++i) {
        const Request* r = batch[i].r;
        mlods_tree_s* T = S->trees[size_t(r->tree)];
        std::memcpy(hq + 3 * off, r->q + 3 * batch[i].off, size_t(batch[i].n) * 12);
        CloudArgs& c = w.h_clouds[i];
        fill_cloud_args(T, c, dq + 3 * off, dp + 3 * off, dn + 3 * off, r->iters, -1.f, T->params.blend_rule);
        if (r->own_kernel) c.kc = r->kc;
        float ext = 0.f;
        for (int a = 0; a < 3; ++a) ext = std::max(ext, T->BB[a] - T->bb[a]);
        c.prune_thr = 0.f;  // the queue kernel walks without pruning
        if (c.qpw == 4) c.qpw = 2;
        w.h_frames[i] = BatchFrame{T->origin[0], T->origin[1], T->origin[2], ext > 0.f ? 1.f / ext : 1.f,
                                   uint32_t(i)};
        w.h_offsets[i] = off;
        off += batch[i].n;
    }
    w.h_offsets[batch.size()] = total;
    const size_t nc = batch.size();
    std::vector<QueueChunk> chunks;
    rc = build_queue_chunks(w.h_clouds, w.h_offsets, int(nc), kServeChunk, chunks);
    if (rc != MLODS_OK) return rc;
    if (w.chunk_cap < chunks.size()) {
        const size_t cap = std::max(chunks.size(), w.chunk_cap + w.chunk_cap / 2);
        rc = grow_pinned(reinterpret_cast<void**>(&w.h_chunks), cap * sizeof(QueueChunk));
        if (rc == MLODS_OK) rc = grow_device(reinterpret_cast<void**>(&w.d_chunks), cap * sizeof(QueueChunk));
        if (rc != MLODS_OK) return rc;
        w.chunk_cap = cap;
    }
    std::memcpy(w.h_chunks, chunks.data(), chunks.size() * sizeof(QueueChunk));
    MLODS_CUDA(cudaMemcpyAsync(dq, hq, size_t(total) * 12, cudaMemcpyHostToDevice, w.s));
    MLODS_CUDA(cudaMemcpyAsync(w.d_clouds, w.h_clouds, nc * sizeof(CloudArgs), cudaMemcpyHostToDevice, w.s));
    MLODS_CUDA(cudaMemcpyAsync(w.d_offsets, w.h_offsets, (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, w.s));
    MLODS_CUDA(cudaMemcpyAsync(w.d_frames, w.h_frames, nc * sizeof(BatchFrame), cudaMemcpyHostToDevice, w.s));
    MLODS_CUDA(cudaMemcpyAsync(w.d_chunks, w.h_chunks, chunks.size() * sizeof(QueueChunk), cudaMemcpyHostToDevice,
                               w.s));
    MLODS_CUDA(cudaMemsetAsync(w.d_stats, 0, kStatsBytes, w.s));
    uint32_t* order = static_cast<uint32_t*>(w.d_order);
    char* tmp = static_cast<char*>(w.d_order) + al256(size_t(total) * 4);
    MLODS_CUDA(compute_batch_order(dq, total, w.d_offsets, int(nc), w.d_frames, true, order, tmp, w.s));
    QueueArgs a;
    a.clouds = w.d_clouds;
    a.q_offsets = w.d_offsets;
    a.chunks = w.d_chunks;
    a.n_chunks = int64_t(chunks.size());
    a.order = order;
    a.counter = reinterpret_cast<unsigned int*>(w.d_stats + 8);
    a.stats = w.d_stats;
    MLODS_CUDA(launch_mlod_queue(a, sm_count_for_current_device(), 100, w.s));
    MLODS_CUDA(cudaMemcpyAsync(hp, dp, size_t(total) * 12, cudaMemcpyDeviceToHost, w.s));
    MLODS_CUDA(cudaMemcpyAsync(hn, dn, size_t(total) * 12, cudaMemcpyDeviceToHost, w.s));
    MLODS_CUDA(cudaStreamSynchronize(w.s));
    off = 0;
    for (const Piece& pc : batch) {
        if (pc.r->out_p) std::memcpy(pc.r->out_p + 3 * pc.off, hp + 3 * off, size_t(pc.n) * 12);
        if (pc.r->out_n) std::memcpy(pc.r->out_n + 3 * pc.off, hn + 3 * off, size_t(pc.n) * 12);
        off += pc.n;
    }
    return MLODS_OK;
}

// The next batch, under the server lock: queued requests in arrival order,
// each taken whole while it fits the batch; one larger than a whole batch is
// cut into batch-sized pieces (it keeps its place until its last piece is
// handed out); a request that fits only a later batch is passed over, so
// small requests do not wait behind large ones.  A request that was passed
// over heads the queue, so the next batch starts with it.
void form_batch(mlods_server_s* S, std::vector<Piece>& batch)
{
    const int64_t cap = std::max<int64_t>(S->cfg.max_batch_queries, 1);
    int64_t budget = cap;
    for (auto it = S->queue.begin(); it != S->queue.end() && budget > 0;) {
        if (int64_t(batch.size()) >= S->cfg.max_batch_requests) break;
        Request* r = *it;
        const int64_t rest = r->n - r->taken;
        if (rest <= budget) {
            batch.push_back(Piece{r, r->taken, rest});
            r->taken += rest;
            budget -= rest;
            S->queued -= rest;
            it = S->queue.erase(it);
        } else if (budget == cap) {
            batch.push_back(Piece{r, r->taken, cap});
            r->taken += cap;
            budget = 0;
            S->queued -= cap;
        } else {
            ++it;
        }
    }
}

void worker_main(mlods_server_s* S, Worker* w)
{
    cudaSetDevice(S->device);
    std::vector<Piece> batch;
    for (;;) {
        batch.clear();
        {
            std::unique_lock<std::mutex> lock(S->mu);
            while (!S->stopping && S->queue.empty()) S->cv_work.wait_for(lock, std::chrono::milliseconds(50));
            if (S->stopping) return;
            if (S->cfg.max_wait_us > 0 && S->queued < S->cfg.max_batch_queries)
                S->cv_work.wait_for(lock, std::chrono::microseconds(S->cfg.max_wait_us),
                                    [&] { return S->stopping || S->queued >= S->cfg.max_batch_queries; });
            if (S->stopping) return;
            form_batch(S, batch);
        }
        if (batch.empty()) continue;
        const auto t0 = Clock::now();
        const int rc = run_batch(S, *w, batch);
        const auto t1 = Clock::now();
        const char* msg = mlods_last_error();
        std::lock_guard<std::mutex> lock(S->mu);
        for (const Piece& pc : batch) {
            Request* r = pc.r;
            if (rc != MLODS_OK && r->piece_status == MLODS_OK) {
                r->piece_status = rc;
                std::snprintf(r->error, sizeof r->error, "%s", msg);
            }
            r->finished += pc.n;
            S->queries += pc.n;
            // the request's last piece, or the last one in flight of a cancelled request
            if (r->finished == r->n || (r->cancelled && r->finished == r->taken)) {
                r->status = r->piece_status;
                r->t_done = t1;
                ++S->completed;
            }
        }
        ++S->batches;
        S->busy_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
        S->cv_done.notify_all();
    }
}

void destroy_worker(Worker* w)
{
    if (!w) return;
    if (w->s) cudaStreamSynchronize(w->s);
    cudaFreeHost(w->h_stage);
    cudaFreeHost(w->h_clouds);
    cudaFreeHost(w->h_offsets);
    cudaFreeHost(w->h_frames);
    cudaFreeHost(w->h_chunks);
    cudaFree(w->d_chunks);
    cudaFree(w->d_buf);
    cudaFree(w->d_clouds);
    cudaFree(w->d_offsets);
    cudaFree(w->d_frames);
    cudaFree(w->d_stats);
    cudaFree(w->d_order);
    if (w->s) cudaStreamDestroy(w->s);
    delete w;
}

void stop_server(mlods_server_s* S)
{
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->stopping = true;
        // queued requests are cancelled; batches in flight finish, and a
        // request with pieces in flight is answered when its last one returns
        for (Request* r : S->queue) {
            r->cancelled = true;
            if (r->piece_status == MLODS_OK) {
                r->piece_status = MLODS_ERR_STATE;
                std::snprintf(r->error, sizeof r->error, "server stopped before the request ran");
            }
            if (r->finished == r->taken) {
                r->status = r->piece_status;
                r->t_done = Clock::now();
                ++S->completed;
            }
        }
        S->queue.clear();
        S->queued = 0;
    }
    S->cv_work.notify_all();
    for (Worker* w : S->workers)
        if (w->thread.joinable()) w->thread.join();
    S->cv_done.notify_all();
    for (Worker* w : S->workers) destroy_worker(w);
    S->workers.clear();
    for (auto& kv : S->live) delete kv.second;
    S->live.clear();
}

}  // namespace
}  // namespace mlods

using namespace mlods;

extern "C" {

void mlods_server_default_config(mlods_server_config* c)
{
    if (!c) return;
    c->n_streams = 2;
    c->max_batch_queries = int64_t(1) << 21;
    c->max_batch_requests = 4096;
    c->max_pending_queries = int64_t(1) << 26;
    c->max_wait_us = 0;
}

int mlods_server_create(const mlods_tree* trees, int32_t n_trees, const mlods_server_config* cfg, mlods_server* out)
{
    if (!trees || n_trees <= 0 || !out) {
        set_last_error("server create: need at least one tree");
        return MLODS_ERR_INVALID;
    }
    *out = nullptr;
    mlods_server_config c;
    mlods_server_default_config(&c);
    if (cfg) c = *cfg;
    if (c.n_streams < 1 || c.n_streams > 16 || c.max_batch_queries < 1 || c.max_batch_requests < 1 ||
        c.max_pending_queries < 1 || c.max_wait_us < 0) {
        set_last_error("server create: bad configuration");
        return MLODS_ERR_INVALID;
    }
    for (int i = 0; i < n_trees; ++i) {
        if (!trees[i] || !trees[i]->kernel_set) {
            set_last_error("server create: tree %d is null or has no kernel", i);
            return MLODS_ERR_STATE;
        }
        if (trees[i]->params.mode != MLODS_MODE_MLOD) {
            set_last_error("server create: tree %d is not in MLoD mode", i);
            return MLODS_ERR_INVALID;
        }
        if (trees[i]->device != trees[0]->device) {
            set_last_error("server create: tree %d is on device %d, tree 0 on device %d", i, trees[i]->device,
                           trees[0]->device);
            return MLODS_ERR_INVALID;
        }
    }
    MLODS_ON_DEVICE(trees[0]->device);
    auto* S = new (std::nothrow) mlods_server_s();
    if (!S) {
        set_last_error("server create: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    S->trees.assign(trees, trees + n_trees);
    S->cfg = c;
    S->device = trees[0]->device;
    for (int i = 0; i < c.n_streams; ++i) {
        auto* w = new (std::nothrow) Worker();
        cudaError_t e = w ? cudaStreamCreateWithFlags(&w->s, cudaStreamNonBlocking) : cudaErrorMemoryAllocation;
        if (e == cudaSuccess) e = cudaMalloc(&w->d_stats, kStatsBytes);
        if (e != cudaSuccess) {
            destroy_worker(w);
            stop_server(S);
            delete S;
            return cuda_fail(e, "server create", __FILE__, __LINE__);
        }
        S->workers.push_back(w);
    }
    for (Worker* w : S->workers) w->thread = std::thread(worker_main, S, w);
    *out = S;
    return MLODS_OK;
}

int mlods_server_submit(mlods_server s, int32_t tree, int64_t n, const float* q, float* out_pts, float* out_nrm,
                        int32_t n_iterations, const mlods_kernel* kernel, uint64_t* ticket)
{
    if (!s || !q || !ticket || n <= 0 || n_iterations < 0 || tree < 0 || tree >= int32_t(s->trees.size())) {
        set_last_error("server submit: bad arguments");
        return MLODS_ERR_INVALID;
    }
    if (n >= (int64_t(1) << 31)) {
        set_last_error("server submit: request of %lld queries is too large", (long long)n);
        return MLODS_ERR_CAPACITY;
    }
    auto* r = new (std::nothrow) Request();
    if (!r) {
        set_last_error("server submit: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    r->tree = tree;
    r->n = n;
    r->q = q;
    r->out_p = out_pts;
    r->out_n = out_nrm;
    r->iters = n_iterations;
    if (kernel) {
        const int rc = validate_kernel(kernel);
        if (rc != MLODS_OK) {
            delete r;
            return rc;
        }
        r->own_kernel = true;
        int krc = MLODS_OK;
        {
            DeviceGuard guard(s->device);
            krc = guard.err != cudaSuccess ? cuda_fail(guard.err, "server submit: select device", __FILE__, __LINE__)
                                           : make_kernel_consts(*kernel, &r->kc);
        }
        if (krc != MLODS_OK) {
            delete r;
            return krc;
        }
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) {
        delete r;
        set_last_error("server submit: server is stopping");
        return MLODS_ERR_STATE;
    }
    if (s->queued + n > s->cfg.max_pending_queries) {
        delete r;
        set_last_error("server submit: %lld queries queued, admitting %lld more would exceed max_pending_queries=%lld",
                       (long long)s->queued, (long long)n, (long long)s->cfg.max_pending_queries);
        return MLODS_ERR_CAPACITY;
    }
    r->ticket = s->next_ticket++;
    r->t_submit = Clock::now();
    s->queue.push_back(r);
    s->queued += n;
    s->live[r->ticket] = r;
    *ticket = r->ticket;
    s->cv_work.notify_one();
    return MLODS_OK;
}

int mlods_server_wait(mlods_server s, uint64_t ticket, int32_t timeout_ms, double* latency_ms)
{
    if (!s || timeout_ms < 0) {
        set_last_error("server wait: bad arguments");
        return MLODS_ERR_INVALID;
    }
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) {
        set_last_error("server wait: unknown ticket %llu", (unsigned long long)ticket);
        return MLODS_ERR_INVALID;
    }
    Request* r = it->second;
    const bool done = s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return r->status >= 0; });
    if (!done) {
        set_last_error("server wait: ticket %llu not finished after %d ms", (unsigned long long)ticket, timeout_ms);
        return MLODS_ERR_TIMEOUT;
    }
    const int st = r->status;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    if (st != MLODS_OK) set_last_error("%s", r->error);
    s->live.erase(it);
    delete r;
    return st;
}

int mlods_server_stats(mlods_server s, int64_t* completed, int64_t* batches, int64_t* queries, int64_t* queued,
                       double* busy_ms)
{
    if (!s) {
        set_last_error("null server");
        return MLODS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (completed) *completed = s->completed;
    if (batches) *batches = s->batches;
    if (queries) *queries = s->queries;
    if (queued) *queued = s->queued;
    if (busy_ms) *busy_ms = s->busy_ms;
    return MLODS_OK;
}

int mlods_server_free(mlods_server s)
{
    if (!s) return MLODS_OK;
    stop_server(s);
    delete s;
    return MLODS_OK;
}

}  // extern "C"
