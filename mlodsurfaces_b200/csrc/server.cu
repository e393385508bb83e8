// server.cu -- a projection server over resident trees.
//
// No counterpart in the reference, which projects one request at a time on
// the legacy stream.  Requests (a tree, n host query points, an iteration
// count, optionally their own weight kernel) are queued by any host thread
// and answered asynchronously.  Worker threads, one per CUDA stream, take
// what is queued whenever they are free (up to a batch size; large requests
// in pieces, small ones passing over those that do not fit), stage it in
// pinned memory, and project the batch with one launch of the queue kernel
// (each request or piece is one "cloud", with its own tree, kernel and
// iteration count), so copies of one batch overlap the projection of another.
//
// Admission follows the device memory: a batch's device buffers (queries,
// results, ordering scratch, launch arguments) come from the library's
// stream-ordered pool, sized for that batch, and go back when it finishes; a
// worker forms a batch only from what fits the device budget minus the
// batches in flight, so queued requests are taken up as batches finish and
// memory frees up.  A submit whose footprint would take the queued work
// beyond its own bound is refused (MLODS_ERR_CAPACITY) instead of growing
// host or device memory without limit.  Every wait has a timeout.
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

// Host-side staging of one worker (pinned, grown on demand); the device
// buffers of a batch come from the stream-ordered pool per batch.
struct Worker {
    cudaStream_t s = nullptr;
    float* h_stage = nullptr;  // 9 floats per query (q, p, n)
    size_t h_cap = 0;
    mlods::CloudArgs* h_clouds = nullptr;
    int64_t* h_offsets = nullptr;
    mlods::BatchFrame* h_frames = nullptr;
    size_t cloud_cap = 0;
    int64_t* d_stats = nullptr;
    std::thread thread;
};

}  // namespace

struct mlods_server_s {
    std::vector<mlods_tree_s*> trees;
    mlods_server_config cfg{};  // budgets resolved at creation
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, Request*> live;
    int64_t queued = 0;          // queries waiting for a batch
    int64_t pending_bytes = 0;   // footprint of the queued queries
    int64_t in_flight = 0;       // device bytes held by the batches in flight
    int64_t peak_in_flight = 0;
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
// statistics, a 64-bit slot counter for each launch group of
// kQueueMaxClouds pieces (max_batch_requests is at most kMaxServeGroups
// groups), then a 32-bit work counter for each piece that runs in a launch
// of its own
constexpr int kMaxServeGroups = 64;
constexpr size_t kStatsBytes = 8 * sizeof(int64_t) + kMaxServeGroups * sizeof(uint64_t) +
                               size_t(kMaxServeGroups) * kQueueMaxClouds * sizeof(unsigned int);
// A piece of at least this many times the queries the walk holds in flight
// on the whole GPU runs in a launch of its own (the single-tree kernel, whose
// arguments sit in the constant bank) before the shared launch of the rest.
constexpr int64_t kSoloFill = 16;

// Device layout of one batch of n queries from r requests or pieces.
struct BatchLayout {
    size_t qpn, order, temp, offsets, frames, total;
};

BatchLayout batch_layout(int64_t n, int64_t r)
{
    BatchLayout L;
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t here = at;
        at += al256(bytes);
        return here;
    };
    // (the launch arguments travel in the kernel's parameters)
    L.qpn = take(size_t(n) * 36);
    L.order = take(size_t(n) * 4);
    L.temp = take(query_order_temp_bytes(n));
    L.offsets = take(size_t(r + 1) * sizeof(int64_t));
    L.frames = take(size_t(r) * sizeof(BatchFrame));
    L.total = at;
    return L;
}

int64_t batch_bytes(int64_t n, int64_t r) { return n > 0 ? int64_t(batch_layout(n, r).total) : 0; }

// Footprint of a queued request's n remaining queries: its device bytes when
// it runs alone, plus its pinned staging.
int64_t request_bytes(int64_t n) { return n > 0 ? batch_bytes(n, 1) + n * 36 : 0; }

// The most queries a batch of r requests can hold within `bytes` of device
// memory (0 if not even one).
int64_t queries_within(int64_t bytes, int64_t r)
{
    if (batch_bytes(1, r) > bytes) return 0;
    int64_t lo = 1, hi = std::max<int64_t>(1, bytes / 36);
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo + 1) / 2;
        if (batch_bytes(mid, r) <= bytes) lo = mid; else hi = mid - 1;
    }
    return lo;
}

int grow_pinned(void** p, size_t bytes)
{
    cudaFreeHost(*p);
    *p = nullptr;
    MLODS_CUDA(cudaMallocHost(p, bytes));
    return MLODS_OK;
}

int ensure_capacity(Worker& w, int64_t total, size_t n_req)
{
    if (w.h_cap < size_t(total)) {
        const int rc = grow_pinned(reinterpret_cast<void**>(&w.h_stage), size_t(total) * 36);
        if (rc != MLODS_OK) return rc;
        w.h_cap = size_t(total);
    }
    if (w.cloud_cap < n_req) {
        const size_t cap = std::max<size_t>(n_req, 64);
        int rc = grow_pinned(reinterpret_cast<void**>(&w.h_clouds), cap * sizeof(CloudArgs));
        if (rc == MLODS_OK) rc = grow_pinned(reinterpret_cast<void**>(&w.h_offsets), (cap + 1) * sizeof(int64_t));
        if (rc == MLODS_OK) rc = grow_pinned(reinterpret_cast<void**>(&w.h_frames), cap * sizeof(BatchFrame));
        if (rc != MLODS_OK) return rc;
        w.cloud_cap = cap;
    }
    return MLODS_OK;
}

// Projects one batch of requests on the worker's stream with device buffers
// from the stream-ordered pool (returned before this returns); host outputs
// are written before it returns.
int run_batch(mlods_server_s* S, Worker& w, const std::vector<Piece>& batch)
{
    int64_t total = 0;
    for (const Piece& pc : batch) total += pc.n;
    const size_t nc = batch.size();
    const BatchLayout L = batch_layout(total, int64_t(nc));
    int rc = ensure_capacity(w, total, nc);
    if (rc != MLODS_OK) return rc;
    char* mem = nullptr;
    MLODS_CUDA(scratch_alloc(reinterpret_cast<void**>(&mem), L.total, w.s));
    float* dq = reinterpret_cast<float*>(mem + L.qpn);
    float* dp = dq + 3 * total;
    float* dn = dq + 6 * total;
    uint32_t* order = reinterpret_cast<uint32_t*>(mem + L.order);
    int64_t* d_offsets = reinterpret_cast<int64_t*>(mem + L.offsets);
    BatchFrame* d_frames = reinterpret_cast<BatchFrame*>(mem + L.frames);
    float* hq = w.h_stage;
    float* hp = w.h_stage + 3 * total;
    float* hn = w.h_stage + 6 * total;
    int64_t off = 0;
    int qpw = 1;  // one schedule per launch: the largest the batch's trees ask for
    for (size_t i = 0; i < nc; ++i) {
        const Request* r = batch[i].r;
        mlods_tree_s* T = S->trees[size_t(r->tree)];
        std::memcpy(hq + 3 * off, r->q + 3 * batch[i].off, size_t(batch[i].n) * 12);
        CloudArgs& c = w.h_clouds[i];
        fill_cloud_args(T, c, dq + 3 * off, dp + 3 * off, dn + 3 * off, r->iters, -1.f, T->params.blend_rule);
        if (r->own_kernel) c.kc = r->kc;
        c.prune_thr = 0.f;  // the queue kernel walks without pruning
        qpw = std::max(qpw, std::min(c.qpw, 2));
        float ext = 0.f;
        for (int a = 0; a < 3; ++a) ext = std::max(ext, T->BB[a] - T->bb[a]);
        w.h_frames[i] = BatchFrame{T->origin[0], T->origin[1], T->origin[2], ext > 0.f ? 1.f / ext : 1.f,
                                   uint32_t(i)};
        w.h_offsets[i] = off;
        off += batch[i].n;
    }
    w.h_offsets[nc] = total;
    cudaError_t e = cudaMemcpyAsync(dq, hq, size_t(total) * 12, cudaMemcpyHostToDevice, w.s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_offsets, w.h_offsets, (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, w.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_frames, w.h_frames, nc * sizeof(BatchFrame), cudaMemcpyHostToDevice, w.s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.d_stats, 0, kStatsBytes, w.s);
    if (e == cudaSuccess)
        e = compute_batch_order(dq, total, d_offsets, int(nc), d_frames, true, order, mem + L.temp, w.s);
    if (e == cudaSuccess) {
        const int sm = sm_count_for_current_device();
        const int64_t solo_min = kSoloFill * project_resident_queries(qpw, sm);
        std::vector<CloudArgs> qclouds;
        std::vector<int64_t> qbase, qlen;
        unsigned int* solo_counters = reinterpret_cast<unsigned int*>(w.d_stats + 8 + kMaxServeGroups);
        int n_solo = 0;
        for (size_t i = 0; i < nc && e == cudaSuccess; ++i) {
            const int64_t len = w.h_offsets[i + 1] - w.h_offsets[i];
            if (len >= solo_min) {
                // a large piece: the single-tree kernel on its slice of the order
                ProjectArgs pa;
                pa.cloud = w.h_clouds[i];
                pa.order = order + w.h_offsets[i];
                pa.order_base = uint32_t(w.h_offsets[i]);
                pa.nq = len;
                pa.counter = solo_counters + n_solo++;
                pa.stats = w.d_stats;
                pa.queries_per_warp = qpw;
                e = launch_mlod_project(pa, pa.cloud.kc.type, pa.cloud.rule, sm, w.s);
            } else {
                qclouds.push_back(w.h_clouds[i]);
                qbase.push_back(w.h_offsets[i]);
                qlen.push_back(len);
            }
        }
        if (e == cudaSuccess && !qclouds.empty()) {
            QueueArgs a;
            a.clouds = qclouds.data();
            a.base = qbase.data();
            a.len = qlen.data();
            a.n_clouds = int(qclouds.size());
            a.order = order;
            a.counters = reinterpret_cast<unsigned long long*>(w.d_stats + 8);
            a.stats = w.d_stats;
            e = launch_mlod_queue(a, qpw, sm, 100, w.s);
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hp, dp, size_t(total) * 12, cudaMemcpyDeviceToHost, w.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hn, dn, size_t(total) * 12, cudaMemcpyDeviceToHost, w.s);
    const cudaError_t ef = scratch_free(mem, w.s);  // stream-ordered: after the copies
    if (e == cudaSuccess) e = ef;
    const cudaError_t es = cudaStreamSynchronize(w.s);
    if (e == cudaSuccess) e = es;
    if (rc != MLODS_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "server batch", __FILE__, __LINE__);
    off = 0;
    for (const Piece& pc : batch) {
        if (pc.r->out_p) std::memcpy(pc.r->out_p + 3 * pc.off, hp + 3 * off, size_t(pc.n) * 12);
        if (pc.r->out_n) std::memcpy(pc.r->out_n + 3 * pc.off, hn + 3 * off, size_t(pc.n) * 12);
        off += pc.n;
    }
    return MLODS_OK;
}

// The next batch, under the server lock: queued requests in arrival order,
// each taken whole while it fits the batch -- at most max_batch_queries and
// max_batch_requests, and no more device memory than the budget leaves beside
// the batches in flight; one larger than what a batch can hold is cut into
// pieces (it keeps its place until its last piece is handed out); a request
// that fits only a later batch is passed over, so small requests do not wait
// behind large ones.  A request that was passed over heads the queue, so the
// next batch starts with it.  Returns the batch's device bytes (0: nothing
// fits until memory frees up).
int64_t form_batch(mlods_server_s* S, std::vector<Piece>& batch)
{
    const int64_t avail = S->cfg.max_device_bytes - S->in_flight;
    int64_t total = 0;
    for (auto it = S->queue.begin(); it != S->queue.end();) {
        if (int64_t(batch.size()) >= S->cfg.max_batch_requests) break;
        const int64_t nr = int64_t(batch.size()) + 1;
        const int64_t cap = std::min(S->cfg.max_batch_queries, queries_within(avail, nr));
        const int64_t room = cap - total;
        if (room <= 0) break;
        Request* r = *it;
        const int64_t rest = r->n - r->taken;
        int64_t take = 0;
        if (rest <= room) {
            take = rest;
        } else if (batch.empty()) {
            take = room;  // a piece as large as the batch can hold
        } else {
            ++it;         // fits a later batch only: pass over it
            continue;
        }
        batch.push_back(Piece{r, r->taken, take});
        S->pending_bytes -= request_bytes(rest) - request_bytes(rest - take);
        r->taken += take;
        total += take;
        S->queued -= take;
        if (r->taken == r->n) it = S->queue.erase(it);
        else break;  // the batch is full
    }
    return batch.empty() ? 0 : batch_bytes(total, int64_t(batch.size()));
}

void worker_main(mlods_server_s* S, Worker* w)
{
    cudaSetDevice(S->device);
    std::vector<Piece> batch;
    for (;;) {
        batch.clear();
        int64_t bytes = 0;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            for (;;) {
                while (!S->stopping && S->queue.empty()) S->cv_work.wait_for(lock, std::chrono::milliseconds(50));
                if (S->stopping) return;
                if (S->cfg.max_wait_us > 0 && S->queued < S->cfg.max_batch_queries)
                    S->cv_work.wait_for(lock, std::chrono::microseconds(S->cfg.max_wait_us),
                                        [&] { return S->stopping || S->queued >= S->cfg.max_batch_queries; });
                if (S->stopping) return;
                bytes = form_batch(S, batch);
                if (!batch.empty()) break;
                // nothing fits beside the batches in flight: wait for one to return
                S->cv_work.wait_for(lock, std::chrono::milliseconds(50));
            }
            S->in_flight += bytes;
            S->peak_in_flight = std::max(S->peak_in_flight, S->in_flight);
        }
        const auto t0 = Clock::now();
        const int rc = run_batch(S, *w, batch);
        const auto t1 = Clock::now();
        const char* msg = mlods_last_error();
        std::lock_guard<std::mutex> lock(S->mu);
        S->in_flight -= bytes;
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
        S->cv_work.notify_all();  // memory came back: a waiting worker may form its batch
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
    cudaFree(w->d_stats);
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
        S->pending_bytes = 0;
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
    c->max_batch_requests = 4096;
    c->max_batch_queries = int64_t(1) << 18;
    c->max_device_bytes = 0;
    c->max_pending_bytes = 0;
    c->max_wait_us = 0;
    c->reserved = 0;
}

int64_t mlods_server_batch_bytes(int64_t n_queries, int64_t n_requests)
{
    if (n_queries <= 0 || n_requests <= 0) return 0;
    return batch_bytes(n_queries, n_requests);
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
        c.max_batch_requests > kMaxServeGroups * kQueueMaxClouds ||
        c.max_device_bytes < 0 || c.max_pending_bytes < 0 || c.max_wait_us < 0) {
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
    if (c.max_device_bytes == 0) {
        size_t free_b = 0, total_b = 0;
        MLODS_CUDA(cudaMemGetInfo(&free_b, &total_b));
        c.max_device_bytes = int64_t(free_b / 2);
    }
    // a batch must be able to make progress on its own
    const int64_t floor_bytes = batch_bytes(4096, 1);
    if (c.max_device_bytes < floor_bytes) {
        set_last_error("server create: max_device_bytes=%lld is below one batch of 4096 queries (%lld bytes)",
                       (long long)c.max_device_bytes, (long long)floor_bytes);
        return MLODS_ERR_CAPACITY;
    }
    if (c.max_pending_bytes == 0) c.max_pending_bytes = 8 * c.max_device_bytes;
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
    const int64_t bytes = request_bytes(n);
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) {
        delete r;
        set_last_error("server submit: server is stopping");
        return MLODS_ERR_STATE;
    }
    if (s->pending_bytes + bytes > s->cfg.max_pending_bytes) {
        delete r;
        set_last_error("server submit: queued work holds %lld bytes; admitting %lld queries (%lld bytes) would "
                       "exceed max_pending_bytes=%lld (capacity)",
                       (long long)s->pending_bytes, (long long)n, (long long)bytes,
                       (long long)s->cfg.max_pending_bytes);
        return MLODS_ERR_CAPACITY;
    }
    r->ticket = s->next_ticket++;
    r->t_submit = Clock::now();
    s->queue.push_back(r);
    s->queued += n;
    s->pending_bytes += bytes;
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

int mlods_server_memory(mlods_server s, int64_t* in_flight_bytes, int64_t* peak_in_flight_bytes,
                        int64_t* pending_bytes, int64_t* max_device_bytes, int64_t* max_pending_bytes)
{
    if (!s) {
        set_last_error("null server");
        return MLODS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (in_flight_bytes) *in_flight_bytes = s->in_flight;
    if (peak_in_flight_bytes) *peak_in_flight_bytes = s->peak_in_flight;
    if (pending_bytes) *pending_bytes = s->pending_bytes;
    if (max_device_bytes) *max_device_bytes = s->cfg.max_device_bytes;
    if (max_pending_bytes) *max_pending_bytes = s->cfg.max_pending_bytes;
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
