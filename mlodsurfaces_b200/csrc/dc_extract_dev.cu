// dc_extract_dev.cu -- dual-contouring extraction on the device, in the
// reference's order.
//
// minimal_edges::traverse (octree.h:400-540) is a depth-first recursion of
// node, face and edge calls; dual_contour::extract (dual_contouring.h:59-87)
// numbers the vertices in the order the traversal first uses them.  Every
// call has a path from the root call: the sequence of its ancestors' branch
// choices (a node call makes 26 calls, a face call 8, an edge call 2).
// Written most significant first into a 64-bit key (5, 3 or 1 bits per
// level, after the parent's kind), the keys of the emitted edges sort in the
// depth-first order.  So the recursion runs level by level over all calls at
// once: each level's calls write their children (and the sign-changing
// minimal edges they reach) with a count / scan / write pass, the crossings
// are sorted by key, and the vertex numbering is the order of first use
// (the (cell, use) pairs stably sorted by cell, the first use of each cell
// flagged, a scan of the flags).  The result equals the host extraction
// exactly; grids deeper than 12 levels (paths longer than 64 bits) use the
// host version.
#include <algorithm>
#include <vector>

#include "dc.h"
#include "primitives.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
constexpr unsigned kThreads = 256;
inline unsigned blocks_for(int64_t n) { return unsigned((n + kThreads - 1) / kThreads); }
constexpr int kX = 0, kY = 1, kZ = 2;

// the order of a face's inner edges (edge direction, half), as on the host
__constant__ int c_face_edges[3][4][2] = {
    {{kY, 0}, {kY, 1}, {kZ, 0}, {kZ, 1}},
    {{kX, 1}, {kX, 0}, {kZ, 0}, {kZ, 1}},
    {{kY, 0}, {kY, 1}, {kX, 0}, {kX, 1}},
};

__device__ __forceinline__ void perp_d(int e, int& p1, int& p2)
{
    p1 = e == kX ? kY : kX;
    p2 = e == kZ ? kY : kZ;
}

struct Grid {
    const int4* cells;
    const int32_t* kids;  // 8 per cell, -1 for leaves
    const float* cf;      // 8 corner values per cell
};

__device__ __forceinline__ bool leaf(const Grid& g, int32_t n) { return g.kids[8 * int64_t(n)] < 0; }
__device__ __forceinline__ int32_t kid(const Grid& g, int32_t n, int c)
{
    return leaf(g, n) ? n : g.kids[8 * int64_t(n) + c];
}

// call kinds and their branch widths
constexpr int kNode = 0, kFace = 1, kEdge = 2;
__device__ __forceinline__ int width_of(int kind) { return kind == kNode ? 5 : (kind == kFace ? 3 : 1); }

struct Call {
    int4 n;        // cells (node: n.x; face: n.x, n.y; edge: all four, slot order)
    uint64_t key;  // path, most significant first
    uint32_t meta; // kind | dir << 2 | bits << 8
};

__device__ __forceinline__ int kind_of(uint32_t m) { return int(m & 3u); }
__device__ __forceinline__ int dir_of(uint32_t m) { return int((m >> 2) & 3u); }
__device__ __forceinline__ int bits_of(uint32_t m) { return int(m >> 8); }

__device__ __forceinline__ bool minimal(const Grid& g, const Call& c)
{
    return kind_of(c.meta) == kEdge && leaf(g, c.n.x) && leaf(g, c.n.y) && leaf(g, c.n.z) && leaf(g, c.n.w);
}

// Visits the calls a call makes, in the reference's order, as f(branch, call).
template <typename F>
__device__ __forceinline__ void children(const Grid& g, const Call& c, F f)
{
    const int kind = kind_of(c.meta);
    const int w = width_of(kind), bits = bits_of(c.meta) + w;
    auto child = [&](int branch, int k, int d, int4 n) {
        Call x;
        x.n = n;
        x.key = c.key | (uint64_t(branch) << (64 - bits));
        x.meta = uint32_t(k) | (uint32_t(d) << 2) | (uint32_t(bits) << 8);
        f(x);
    };
    if (kind == kNode) {
        if (leaf(g, c.n.x)) return;
        const int32_t* ch = g.kids + 8 * int64_t(c.n.x);
        int b = 0;
        for (int t = 0; t < 8; ++t) child(b++, kNode, 0, make_int4(ch[t], 0, 0, 0));
        for (int d = 0; d < 3; ++d)
            for (int k = 0; k < 8; ++k)
                if (!((k >> d) & 1)) child(b++, kFace, d, make_int4(ch[k], ch[k | (1 << d)], 0, 0));
        for (int e = 0; e < 3; ++e) {
            int p1, p2;
            perp_d(e, p1, p2);
            for (int h = 0; h < 2; ++h) {
                int32_t nd[4];
                for (int s = 0; s < 4; ++s) nd[s] = ch[(h << e) | ((s & 1) << p1) | ((s >> 1) << p2)];
                child(b++, kEdge, e, make_int4(nd[0], nd[1], nd[2], nd[3]));
            }
        }
    } else if (kind == kFace) {
        const int d = dir_of(c.meta);
        const int32_t n1 = c.n.x, n2 = c.n.y;
        if (leaf(g, n1) && leaf(g, n2)) return;
        int on1[4], on2[4], k1 = 0, k2 = 0;
        for (int k = 0; k < 8; ++k) {
            if ((k >> d) & 1) on1[k1++] = k;
            else on2[k2++] = k;
        }
        int b = 0;
        for (int q = 0; q < 4; ++q) child(b++, kFace, d, make_int4(kid(g, n1, on1[q]), kid(g, n2, on2[q]), 0, 0));
        for (int k = 0; k < 4; ++k) {
            const int e = c_face_edges[d][k][0], h = c_face_edges[d][k][1];
            const int fa = 3 - d - e;
            int p1, p2;
            perp_d(e, p1, p2);
            int32_t nd[4];
            for (int sd = 0; sd < 2; ++sd)
                for (int sf = 0; sf < 2; ++sf) {
                    const int kk = (h << e) | ((1 - sd) << d) | (sf << fa);
                    const int s1 = p1 == d ? sd : sf, s2 = p2 == d ? sd : sf;
                    nd[s1 + 2 * s2] = sd == 0 ? kid(g, n1, kk) : kid(g, n2, kk);
                }
            child(b++, kEdge, e, make_int4(nd[0], nd[1], nd[2], nd[3]));
        }
    } else {
        if (minimal(g, c)) return;
        const int e = dir_of(c.meta);
        int p1, p2;
        perp_d(e, p1, p2);
        const int32_t ns[4] = {c.n.x, c.n.y, c.n.z, c.n.w};
        for (int h = 0; h < 2; ++h) {
            int32_t nd[4];
            for (int s = 0; s < 4; ++s) nd[s] = kid(g, ns[s], (h << e) | ((1 - (s & 1)) << p1) | ((1 - (s >> 1)) << p2));
            child(h, kEdge, e, make_int4(nd[0], nd[1], nd[2], nd[3]));
        }
    }
}

// on_min_edges' sign test; returns -1 (no crossing), 0 or 1 (flip)
__device__ __forceinline__ int crossing(const Grid& g, const Call& c)
{
    const int32_t ns[4] = {c.n.x, c.n.y, c.n.z, c.n.w};
    int sel = 0, sel_d = -1;
    for (int i = 0; i < 4; ++i) {
        const int d = g.cells[ns[i]].x;
        if (d > sel_d) {
            sel = i;
            sel_d = d;
        }
    }
    const int e = dir_of(c.meta);
    int p1, p2;
    perp_d(e, p1, p2);
    const int base = ((1 - (sel & 1)) << p1) | ((1 - (sel >> 1)) << p2);
    int c0 = base, c1 = base | (1 << e);
    if (e == kY) {
        const int t = c0;
        c0 = c1;
        c1 = t;
    }
    const float f0 = g.cf[8 * int64_t(ns[sel]) + c0], f1 = g.cf[8 * int64_t(ns[sel]) + c1];
    if (isnan(f0) || isnan(f1)) return -1;
    const bool m0 = f0 < 0, m1 = f1 < 0;
    if (m0 == m1) return -1;
    return m0 ? 1 : 0;
}

__global__ void count_kernel(Grid g, const Call* __restrict__ calls, int64_t n, uint32_t* __restrict__ n_child,
                             uint32_t* __restrict__ n_cross)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Call c = calls[i];
    uint32_t k = 0, x = 0;
    if (minimal(g, c)) {
        x = crossing(g, c) >= 0 ? 1u : 0u;
    } else {
        children(g, c, [&](const Call&) { ++k; });
    }
    n_child[i] = k;
    n_cross[i] = x;
}

struct Crossing {
    int4 n;
    uint32_t flip;
};

__global__ void write_kernel(Grid g, const Call* __restrict__ calls, int64_t n, const uint32_t* __restrict__ child_at,
                             const uint32_t* __restrict__ cross_at, Call* __restrict__ next,
                             uint64_t* __restrict__ cross_key, Crossing* __restrict__ cross)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Call c = calls[i];
    if (minimal(g, c)) {
        const int f = crossing(g, c);
        if (f >= 0) {
            const uint32_t o = cross_at[i];
            cross_key[o] = c.key;
            cross[o] = Crossing{c.n, uint32_t(f)};
        }
        return;
    }
    uint32_t o = child_at[i];
    children(g, c, [&](const Call& x) { next[o++] = x; });
}

// ---- vertex numbering and triangles over the ordered crossings

// use j (0..5) of crossing r: the cells of triangles (0, 1, 3) and (0, 3, 2)
__device__ __forceinline__ int32_t use_cell(const Crossing& x, int j)
{
    const int32_t ns[4] = {x.n.x, x.n.y, x.n.z, x.n.w};
    const int slot[6] = {0, 1, 3, 0, 3, 2};
    return ns[slot[j]];
}

__global__ void uses_kernel(const Crossing* __restrict__ cross, const uint32_t* __restrict__ order, int64_t nc,
                            uint64_t* __restrict__ key, uint32_t* __restrict__ pos)
{
    const int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (u >= 6 * nc) return;
    const int64_t r = u / 6;
    key[u] = uint64_t(uint32_t(use_cell(cross[order[r]], int(u - 6 * r))));
    pos[u] = uint32_t(u);
}

__global__ void first_use_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ pos, int64_t n,
                                 uint32_t* __restrict__ first)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) first[pos[i]] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

// vertex of every use: the number of its cell's first use
__global__ void use_vertex_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ pos, int64_t n,
                                  const uint32_t* __restrict__ rank, uint32_t* __restrict__ vert_at,
                                  int32_t* __restrict__ cell_of_vertex, const uint32_t* __restrict__ first)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t h = i;
    while (h > 0 && key[h - 1] == key[i]) --h;
    const uint32_t v = rank[pos[h]];
    vert_at[pos[i]] = v;
    if (first[pos[i]]) cell_of_vertex[v] = int32_t(key[i]);
}

__global__ void tri_count_kernel(const uint32_t* __restrict__ vert_at, int64_t nc, uint32_t* __restrict__ cnt)
{
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= nc) return;
    const uint32_t* v = vert_at + 6 * r;
    uint32_t k = 0;
    for (int t = 0; t < 2; ++t) {
        const uint32_t a = v[3 * t], b = v[3 * t + 1], c = v[3 * t + 2];
        k += (a != b && b != c && c != a) ? 1u : 0u;
    }
    cnt[r] = k;
}

__global__ void tri_write_kernel(const Crossing* __restrict__ cross, const uint32_t* __restrict__ order,
                                 const uint32_t* __restrict__ vert_at, const uint32_t* __restrict__ at, int64_t nc,
                                 uint32_t* __restrict__ tri)
{
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= nc) return;
    const bool flip = cross[order[r]].flip != 0;
    const uint32_t* v = vert_at + 6 * r;
    uint32_t o = at[r];
    for (int t = 0; t < 2; ++t) {
        const uint32_t a = v[3 * t], b = v[3 * t + 1], c = v[3 * t + 2];
        if (a == b || b == c || c == a) continue;
        tri[3 * o] = a;
        tri[3 * o + 1] = flip ? c : b;
        tri[3 * o + 2] = flip ? b : c;
        ++o;
    }
}

__global__ void gather_vertices_kernel(const int32_t* __restrict__ cell_of_vertex, int64_t nv,
                                       const float* __restrict__ cell_vertex, float* __restrict__ pos)
{
    const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const int64_t c = cell_of_vertex[v];
    for (int a = 0; a < 3; ++a) pos[3 * v + a] = cell_vertex[3 * c + a];
}

// parent links of a sorted grid: the slot of every non-root cell in its
// parent's child table (binary search in the parent's depth range)
__global__ void link_kernel(const int4* __restrict__ cells, int64_t n, const int64_t* __restrict__ begin, int maxd,
                            int32_t* __restrict__ kids, int* __restrict__ bad)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 c = cells[i];
    if (c.x == 0) return;
    auto fh = [](int v) { return (v < 0 && (v % 2) != 0) ? v / 2 - 1 : v / 2; };
    const int4 p = make_int4(c.x - 1, fh(c.y), fh(c.z), fh(c.w));
    if (p.x > maxd) return;
    int64_t lo = begin[p.x], hi = begin[p.x + 1];
    auto less = [](const int4& a, const int4& b) {
        if (a.x != b.x) return a.x < b.x;
        if (a.w != b.w) return a.w < b.w;
        if (a.z != b.z) return a.z < b.z;
        return a.y < b.y;
    };
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if (less(cells[m], p)) lo = m + 1;
        else hi = m;
    }
    if (lo >= begin[p.x + 1] || cells[lo].x != p.x || cells[lo].y != p.y || cells[lo].z != p.z || cells[lo].w != p.w) {
        atomicExch(bad, 1);
        return;
    }
    const int k = (c.y - 2 * p.y) + 2 * (c.z - 2 * p.z) + 4 * (c.w - 2 * p.w);
    kids[8 * lo + k] = int32_t(i);
}

__global__ void child_count_check_kernel(const int32_t* __restrict__ kids, int64_t n, int* __restrict__ bad)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cnt = 0;
    for (int k = 0; k < 8; ++k) cnt += kids[8 * i + k] >= 0;
    if (cnt != 0 && cnt != 8) atomicExch(bad, 2);
}

// The stream of the extraction running on this host thread: its buffers come
// from the library's stream-ordered pool on that stream.
thread_local cudaStream_t tl_stream = nullptr;

struct StreamScope {
    explicit StreamScope(cudaStream_t s) { tl_stream = s; }
    ~StreamScope() { tl_stream = nullptr; }
};

struct Buf {
    void* p = nullptr;
    size_t cap = 0;
    cudaStream_t s = tl_stream;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() { scratch_free(p, s); }
    int need(size_t bytes)
    {
        if (bytes <= cap) return MLODS_OK;
        scratch_free(p, s);  // stream-ordered: after the work queued on it
        p = nullptr;
        cap = 0;
        MLODS_CUDA(scratch_alloc(&p, std::max<size_t>(bytes, 256), s));
        cap = std::max<size_t>(bytes, 256);
        return MLODS_OK;
    }
    template <typename T>
    T* as() const
    {
        return static_cast<T*>(p);
    }
};

int scan_total(uint32_t* d, int64_t n, Buf& tmp, Buf& total, uint32_t* out_total, cudaStream_t s)
{
    int rc = tmp.need(scan_temp_bytes(n));
    if (rc == MLODS_OK) rc = total.need(256);
    if (rc != MLODS_OK) return rc;
    MLODS_CUDA(exclusive_scan_u32(d, d, n, total.as<uint32_t>(), tmp.p, s));
    MLODS_CUDA(cudaMemcpyAsync(out_total, total.p, 4, cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    return MLODS_OK;
}

}  // namespace

int dc_extract_device(const int4* d_cells, int64_t n_cells, const int64_t* h_depth_begin, int max_depth,
                      const float* d_cf, const float* d_cell_vertex, DeviceMesh& out, bool* used_device, cudaStream_t s)
{
    const StreamScope scope(s);
    *used_device = false;
    if (max_depth > 12 || n_cells >= (int64_t(1) << 31)) return MLODS_OK;  // the host version takes it
    Buf kids, bad, begin, tmp, total;
    int rc = kids.need(size_t(n_cells) * 32);
    if (rc == MLODS_OK) rc = bad.need(16);
    if (rc == MLODS_OK) rc = begin.need(size_t(max_depth + 2) * 8);
    if (rc != MLODS_OK) return rc;
    MLODS_CUDA(cudaMemsetAsync(kids.p, 0xff, size_t(n_cells) * 32, s));
    MLODS_CUDA(cudaMemsetAsync(bad.p, 0, 16, s));
    MLODS_CUDA(cudaMemcpyAsync(begin.p, h_depth_begin, size_t(max_depth + 2) * 8, cudaMemcpyHostToDevice, s));
    link_kernel<<<blocks_for(n_cells), kThreads, 0, s>>>(d_cells, n_cells, begin.as<int64_t>(), max_depth,
                                                         kids.as<int32_t>(), bad.as<int>());
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    child_count_check_kernel<<<blocks_for(n_cells), kThreads, 0, s>>>(kids.as<int32_t>(), n_cells, bad.as<int>());
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    int h_bad = 0;
    MLODS_CUDA(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    if (h_bad) {
        set_last_error(h_bad == 1 ? "dc extract: a cell has no parent in the grid"
                                  : "dc extract: a cell has a number of children other than 0 or 8");
        return MLODS_ERR_INVALID;
    }
    *used_device = true;
    // the root call; no root, no edges (minimal_edges::traverse starts there)
    int64_t root = -1;
    if (h_depth_begin[1] > h_depth_begin[0]) {
        // depth-0 cells are the first ones; the root is (0, 0, 0, 0) among them
        std::vector<int4> d0(size_t(h_depth_begin[1] - h_depth_begin[0]));
        MLODS_CUDA(cudaMemcpyAsync(d0.data(), d_cells, d0.size() * sizeof(int4), cudaMemcpyDeviceToHost, s));
        MLODS_CUDA(cudaStreamSynchronize(s));
        for (size_t i = 0; i < d0.size(); ++i)
            if (d0[i].y == 0 && d0[i].z == 0 && d0[i].w == 0) root = int64_t(i);
    }
    Grid g{d_cells, kids.as<int32_t>(), d_cf};
    Buf calls_a, calls_b, n_child, n_cross, ckey, cross, ckey_all, cross_all;
    int64_t n_calls = 0, n_found = 0;
    if (root >= 0) {
        rc = calls_a.need(sizeof(Call));
        if (rc != MLODS_OK) return rc;
        Call c0;
        c0.n = make_int4(int32_t(root), 0, 0, 0);
        c0.key = 0;
        c0.meta = uint32_t(kNode);
        MLODS_CUDA(cudaMemcpyAsync(calls_a.p, &c0, sizeof c0, cudaMemcpyHostToDevice, s));
        n_calls = 1;
    }
    // crossings of all levels, appended
    for (int level = 0; n_calls > 0; ++level) {
        if (level > 14) {
            set_last_error("dc extract: recursion deeper than expected");
            return MLODS_ERR_CAPACITY;
        }
        rc = n_child.need(size_t(n_calls + 1) * 4);
        if (rc == MLODS_OK) rc = n_cross.need(size_t(n_calls + 1) * 4);
        if (rc != MLODS_OK) return rc;
        count_kernel<<<blocks_for(n_calls), kThreads, 0, s>>>(g, calls_a.as<Call>(), n_calls, n_child.as<uint32_t>(),
                                                             n_cross.as<uint32_t>());
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        uint32_t kids_total = 0, cross_total = 0;
        rc = scan_total(n_child.as<uint32_t>(), n_calls, tmp, total, &kids_total, s);
        if (rc == MLODS_OK) rc = scan_total(n_cross.as<uint32_t>(), n_calls, tmp, total, &cross_total, s);
        if (rc == MLODS_OK) rc = calls_b.need(size_t(kids_total) * sizeof(Call));
        if (rc == MLODS_OK) rc = ckey.need(size_t(cross_total) * 8);
        if (rc == MLODS_OK) rc = cross.need(size_t(cross_total) * sizeof(Crossing));
        if (rc != MLODS_OK) return rc;
        write_kernel<<<blocks_for(n_calls), kThreads, 0, s>>>(g, calls_a.as<Call>(), n_calls, n_child.as<uint32_t>(),
                                                             n_cross.as<uint32_t>(), calls_b.as<Call>(),
                                                             ckey.as<uint64_t>(), cross.as<Crossing>());
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        if (cross_total) {
            Buf k2, x2;
            rc = k2.need(size_t(n_found + cross_total) * 8);
            if (rc == MLODS_OK) rc = x2.need(size_t(n_found + cross_total) * sizeof(Crossing));
            if (rc != MLODS_OK) return rc;
            if (n_found) {
                MLODS_CUDA(cudaMemcpyAsync(k2.p, ckey_all.p, size_t(n_found) * 8, cudaMemcpyDeviceToDevice, s));
                MLODS_CUDA(cudaMemcpyAsync(x2.p, cross_all.p, size_t(n_found) * sizeof(Crossing),
                                           cudaMemcpyDeviceToDevice, s));
            }
            MLODS_CUDA(cudaMemcpyAsync(k2.as<uint64_t>() + n_found, ckey.p, size_t(cross_total) * 8,
                                       cudaMemcpyDeviceToDevice, s));
            MLODS_CUDA(cudaMemcpyAsync(x2.as<Crossing>() + n_found, cross.p, size_t(cross_total) * sizeof(Crossing),
                                       cudaMemcpyDeviceToDevice, s));
            MLODS_CUDA(cudaStreamSynchronize(s));
            std::swap(ckey_all.p, k2.p);
            std::swap(ckey_all.cap, k2.cap);
            std::swap(cross_all.p, x2.p);
            std::swap(cross_all.cap, x2.cap);
            n_found += cross_total;
        }
        std::swap(calls_a.p, calls_b.p);
        std::swap(calls_a.cap, calls_b.cap);
        n_calls = int64_t(kids_total);
    }
    // depth-first order of the crossings
    const int64_t nc = n_found;
    Buf order, k1, v1;
    rc = order.need(size_t(std::max<int64_t>(nc, 1)) * 4);
    if (rc != MLODS_OK) return rc;
    if (nc > 0) {
        rc = k1.need(size_t(nc) * 8);
        if (rc == MLODS_OK) rc = v1.need(size_t(nc) * 4);
        if (rc == MLODS_OK) rc = tmp.need(std::max(radix_temp_bytes(nc), scan_temp_bytes(6 * nc)));
        if (rc != MLODS_OK) return rc;
        std::vector<uint32_t> iota(static_cast<size_t>(nc));
        for (int64_t i = 0; i < nc; ++i) iota[size_t(i)] = uint32_t(i);
        MLODS_CUDA(cudaMemcpyAsync(order.p, iota.data(), size_t(nc) * 4, cudaMemcpyHostToDevice, s));
        bool alt = false;
        MLODS_CUDA(radix_sort_pairs_u64(ckey_all.as<uint64_t>(), order.as<uint32_t>(), k1.as<uint64_t>(),
                                        v1.as<uint32_t>(), nc, 64, &alt, tmp.p, s));
        if (alt) MLODS_CUDA(cudaMemcpyAsync(order.p, v1.p, size_t(nc) * 4, cudaMemcpyDeviceToDevice, s));
        MLODS_CUDA(cudaStreamSynchronize(s));  // the host iota goes out of scope
    }
    // first-use numbering of the 6 uses per crossing
    const int64_t nu = 6 * nc;
    Buf ukey, upos, ukey2, upos2, first, vert_at, cell_of_v;
    if (nc > 0) {
        rc = ukey.need(size_t(nu) * 8);
        if (rc == MLODS_OK) rc = upos.need(size_t(nu) * 4);
        if (rc == MLODS_OK) rc = ukey2.need(size_t(nu) * 8);
        if (rc == MLODS_OK) rc = upos2.need(size_t(nu) * 4);
        if (rc == MLODS_OK) rc = first.need(size_t(nu) * 4 + 4);
        if (rc == MLODS_OK) rc = vert_at.need(size_t(nu) * 4);
        if (rc == MLODS_OK) rc = cell_of_v.need(size_t(nu) * 4);
        if (rc == MLODS_OK) rc = tmp.need(std::max(radix_temp_bytes(nu), scan_temp_bytes(nu)));
        if (rc != MLODS_OK) return rc;
        uses_kernel<<<blocks_for(nu), kThreads, 0, s>>>(cross_all.as<Crossing>(), order.as<uint32_t>(), nc,
                                                        ukey.as<uint64_t>(), upos.as<uint32_t>());
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        int cbits = 1;
        while (cbits < 63 && (int64_t(1) << cbits) <= n_cells) ++cbits;
        bool alt = false;
        MLODS_CUDA(radix_sort_pairs_u64(ukey.as<uint64_t>(), upos.as<uint32_t>(), ukey2.as<uint64_t>(),
                                        upos2.as<uint32_t>(), nu, cbits, &alt, tmp.p, s));
        const uint64_t* sk = alt ? ukey2.as<uint64_t>() : ukey.as<uint64_t>();
        const uint32_t* sp = alt ? upos2.as<uint32_t>() : upos.as<uint32_t>();
        uint32_t* fl = first.as<uint32_t>();
        first_use_kernel<<<blocks_for(nu), kThreads, 0, s>>>(sk, sp, nu, fl);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        // rank = exclusive scan of the first-use flags (kept beside them)
        Buf rank;
        rc = rank.need(size_t(nu) * 4);
        if (rc != MLODS_OK) return rc;
        MLODS_CUDA(cudaMemcpyAsync(rank.p, fl, size_t(nu) * 4, cudaMemcpyDeviceToDevice, s));
        uint32_t nv = 0;
        rc = scan_total(rank.as<uint32_t>(), nu, tmp, total, &nv, s);
        if (rc != MLODS_OK) return rc;
        use_vertex_kernel<<<blocks_for(nu), kThreads, 0, s>>>(sk, sp, nu, rank.as<uint32_t>(), vert_at.as<uint32_t>(),
                                                              cell_of_v.as<int32_t>(), fl);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        // triangles
        Buf tcnt;
        rc = tcnt.need(size_t(nc) * 4 + 4);
        if (rc != MLODS_OK) return rc;
        tri_count_kernel<<<blocks_for(nc), kThreads, 0, s>>>(vert_at.as<uint32_t>(), nc, tcnt.as<uint32_t>());
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        uint32_t nt = 0;
        rc = scan_total(tcnt.as<uint32_t>(), nc, tmp, total, &nt, s);
        if (rc != MLODS_OK) return rc;
        rc = dmesh_reserve(out, int64_t(nv), int64_t(nt));
        if (rc != MLODS_OK) return rc;
        tri_write_kernel<<<blocks_for(nc), kThreads, 0, s>>>(cross_all.as<Crossing>(), order.as<uint32_t>(),
                                                            vert_at.as<uint32_t>(), tcnt.as<uint32_t>(), nc,
                                                            dmesh_tri(out));
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        gather_vertices_kernel<<<blocks_for(nv), kThreads, 0, s>>>(cell_of_v.as<int32_t>(), int64_t(nv),
                                                                  d_cell_vertex, dmesh_pos(out));
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        MLODS_CUDA(cudaMemsetAsync(dmesh_nrm(out), 0, size_t(nv) * 12, s));
        MLODS_CUDA(cudaStreamSynchronize(s));
    } else {
        rc = dmesh_reserve(out, 0, 0);
        if (rc != MLODS_OK) return rc;
    }
    return MLODS_OK;
}

}  // namespace mlods
