// dc_adaptive.cu -- the projection-driven dual-contouring grid, on the device.
//
// OctreeGenerator::generate (upsample.cpp:228-251) refines cells level by
// level: the centre of every candidate cell is projected once onto the
// surface (no step limit, find_stable_nodesGPU, upsample.cpp:304-331), the
// cell at the same depth that encloses the projection is kept (the root when
// the projection failed), its 8 children and their 26 neighbours become the
// next level's candidates (compute_leaves, :276-289).  Depth-0 cells next to
// the ones reached are explored the same way until no new one appears, and
// every level's candidates are collected.  uniformize (:262-273) then shifts
// the collection under one root (retreiveCorrectRoot / union_nodes,
// :369-402), grades, completes ancestors and siblings and optionally cuts at
// the maximum depth.
//
// The reference does the set work with std::sort / std::unique over octree_id
// vectors on one host thread.  Here a cell is a 64-bit key whose unsigned
// order is node_comparator's (depth, then z, y, x), every step generates keys
// with one kernel and a radix sort + unique makes the set; only the few
// depth-0 cells are handled on the host.  Two steps are regrouped without
// changing the result: the 26-neighbour expansion of the 8 children of a cell
// is the 4x4x4 block around them, generated directly; grade runs level by
// level from the deepest, which is the order the reference's loop visits.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>

#include "dc.h"
#include "primitives.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
using dcg::Cell;

// ---- cell keys: 4 bits depth | 20 bits z | 20 bits y | 20 bits x (biased)
constexpr int kCoordBits = 20;
constexpr int kBias = 1 << (kCoordBits - 1);
constexpr uint64_t kCoordMask = (uint64_t(1) << kCoordBits) - 1;
constexpr int kMaxKeyDepth = 15;
// bound on the depth-0 cells explored (the [-1, 1]^3 zone is one of them; a
// surface normalised into it reaches its 26 neighbours at most)
constexpr size_t kMaxRootCells = 4096;

__host__ __device__ inline bool encodable(int d, int x, int y, int z)
{
    return d >= 0 && d <= kMaxKeyDepth && x >= -kBias && x < kBias && y >= -kBias && y < kBias && z >= -kBias &&
           z < kBias;
}
__host__ __device__ inline uint64_t make_key(int d, int x, int y, int z)
{
    return (uint64_t(d) << 60) | (uint64_t(z + kBias) << 40) | (uint64_t(y + kBias) << 20) | uint64_t(x + kBias);
}
__host__ __device__ inline int key_depth(uint64_t k) { return int(k >> 60); }
__host__ __device__ inline int key_x(uint64_t k) { return int(k & kCoordMask) - kBias; }
__host__ __device__ inline int key_y(uint64_t k) { return int((k >> 20) & kCoordMask) - kBias; }
__host__ __device__ inline int key_z(uint64_t k) { return int((k >> 40) & kCoordMask) - kBias; }
__host__ __device__ inline int fl_half(int v) { return (v < 0 && (v % 2) != 0) ? v / 2 - 1 : v / 2; }
__host__ __device__ inline uint64_t key_parent(uint64_t k)
{
    return make_key(key_depth(k) - 1, fl_half(key_x(k)), fl_half(key_y(k)), fl_half(key_z(k)));
}
__host__ __device__ inline uint64_t key_ancestor(uint64_t k, int d)
{
    while (key_depth(k) > d) k = key_parent(k);
    return k;
}
inline Cell key_cell(uint64_t k) { return Cell{key_depth(k), key_x(k), key_y(k), key_z(k)}; }

constexpr unsigned kThreads = 256;
inline unsigned blocks_for(int64_t n) { return unsigned((n + kThreads - 1) / kThreads); }

// A set of cells on the device: sorted unique keys plus scratch of the same
// capacity, grown on demand.
// Device buffers of the generator come from the library's stream-ordered
// pool: every step runs on one stream, so a buffer freed there is reused by
// later steps without a cudaMalloc or a synchronising cudaFree.
template <typename T>
cudaError_t pool_alloc(T** p, size_t bytes, cudaStream_t s)
{
    return scratch_alloc(reinterpret_cast<void**>(p), bytes, s);
}

// A set of cells on the device: sorted unique keys plus scratch of the same
// capacity, grown on demand, on one stream.
struct CellSet {
    uint64_t* a = nullptr;  // the keys
    uint64_t* b = nullptr;  // scratch keys
    uint32_t* flags = nullptr;
    uint32_t* excl = nullptr;
    uint32_t* d_total = nullptr;
    void* tmp = nullptr;
    size_t cap = 0, tmp_cap = 0;
    int64_t n = 0;
    cudaStream_t s = nullptr;
    CellSet() = default;
    CellSet(const CellSet&) = delete;
    CellSet& operator=(const CellSet&) = delete;
    ~CellSet()
    {
        scratch_free(a, s);
        scratch_free(b, s);
        scratch_free(flags, s);
        scratch_free(excl, s);
        scratch_free(d_total, s);
        scratch_free(tmp, s);
    }
};

int reserve(CellSet& c, int64_t need, bool keep, cudaStream_t s)
{
    c.s = s;
    if (size_t(need) <= c.cap) return MLODS_OK;
    const size_t cap = std::max<size_t>(size_t(need), c.cap + c.cap / 2);
    uint64_t *a = nullptr, *b = nullptr;
    uint32_t *f = nullptr, *e = nullptr;
    MLODS_CUDA(pool_alloc(&a, cap * 8, s));
    cudaError_t err = pool_alloc(&b, cap * 8, s);
    if (err == cudaSuccess) err = pool_alloc(&f, cap * 4, s);
    if (err == cudaSuccess) err = pool_alloc(&e, cap * 4, s);
    if (err == cudaSuccess && !c.d_total) err = pool_alloc(&c.d_total, 256, s);
    if (err == cudaSuccess && keep && c.n > 0) err = cudaMemcpyAsync(a, c.a, size_t(c.n) * 8, cudaMemcpyDeviceToDevice, s);
    if (err != cudaSuccess) {
        scratch_free(a, s);
        scratch_free(b, s);
        scratch_free(f, s);
        scratch_free(e, s);
        return cuda_fail(err, "dc cells: grow", __FILE__, __LINE__);
    }
    // stream-ordered: the old buffers go after the copy above
    scratch_free(c.a, s);
    scratch_free(c.b, s);
    scratch_free(c.flags, s);
    scratch_free(c.excl, s);
    c.a = a;
    c.b = b;
    c.flags = f;
    c.excl = e;
    c.cap = cap;
    const size_t tb = std::max(radix_temp_bytes(int64_t(cap)), scan_temp_bytes(int64_t(cap)));
    if (tb > c.tmp_cap) {
        scratch_free(c.tmp, s);
        c.tmp = nullptr;
        c.tmp_cap = 0;
        MLODS_CUDA(pool_alloc(&c.tmp, tb, s));
        c.tmp_cap = tb;
    }
    return MLODS_OK;
}

__global__ void unique_flags_kernel(const uint64_t* __restrict__ k, int64_t n, uint32_t* __restrict__ f)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) f[i] = (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
}

__global__ void compact_kernel(const uint64_t* __restrict__ k, const uint32_t* __restrict__ f,
                               const uint32_t* __restrict__ e, int64_t n, uint64_t* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n && f[i]) out[e[i]] = k[i];
}

// Sorts c.a[0, c.n) and removes duplicates in place.
int sort_unique(CellSet& c, cudaStream_t s)
{
    if (c.n <= 1) return MLODS_OK;
    bool alt = false;
    MLODS_CUDA(radix_sort_pairs_u64(c.a, nullptr, c.b, nullptr, c.n, 64, &alt, c.tmp, s));
    if (alt) std::swap(c.a, c.b);
    unique_flags_kernel<<<blocks_for(c.n), kThreads, 0, s>>>(c.a, c.n, c.flags);
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    MLODS_CUDA(exclusive_scan_u32(c.flags, c.excl, c.n, c.d_total, c.tmp, s));
    compact_kernel<<<blocks_for(c.n), kThreads, 0, s>>>(c.a, c.flags, c.excl, c.n, c.b);
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    uint32_t total = 0;
    MLODS_CUDA(cudaMemcpyAsync(&total, c.d_total, 4, cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    std::swap(c.a, c.b);
    c.n = int64_t(total);
    return MLODS_OK;
}

// Appends n keys from device memory.
int append(CellSet& c, const uint64_t* d_keys, int64_t n, cudaStream_t s)
{
    if (n <= 0) return MLODS_OK;
    int rc = reserve(c, c.n + n, true, s);
    if (rc != MLODS_OK) return rc;
    MLODS_CUDA(cudaMemcpyAsync(c.a + c.n, d_keys, size_t(n) * 8, cudaMemcpyDeviceToDevice, s));
    c.n += n;
    return MLODS_OK;
}

int upload(CellSet& c, const std::vector<uint64_t>& keys, cudaStream_t s)
{
    c.n = 0;
    int rc = reserve(c, int64_t(keys.size()), false, s);
    if (rc != MLODS_OK) return rc;
    if (!keys.empty()) MLODS_CUDA(cudaMemcpyAsync(c.a, keys.data(), keys.size() * 8, cudaMemcpyHostToDevice, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    c.n = int64_t(keys.size());
    return MLODS_OK;
}

__global__ void key_cells_kernel(const uint64_t* __restrict__ k, int64_t n, int4* __restrict__ out);

// The sorted set as the caller's int32 (depth, x, y, z) rows and its
// deepest level (the depth of the last key).
int cells_to_host(CellSet& c, std::vector<int32_t>& cells_out, int& depth_out, cudaStream_t s)
{
    cells_out.resize(size_t(c.n) * 4);
    depth_out = 0;
    if (c.n == 0) return MLODS_OK;
    int4* d = nullptr;
    MLODS_CUDA(scratch_alloc(reinterpret_cast<void**>(&d), size_t(c.n) * 16, s));
    key_cells_kernel<<<blocks_for(c.n), kThreads, 0, s>>>(c.a, c.n, d);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(cells_out.data(), d, size_t(c.n) * 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    scratch_free(d, s);
    if (e != cudaSuccess) return cuda_fail(e, "dc cells: download", __FILE__, __LINE__);
    depth_out = cells_out[cells_out.size() - 4];
    return MLODS_OK;
}

int download(const CellSet& c, std::vector<uint64_t>& keys, cudaStream_t s)
{
    keys.resize(size_t(c.n));
    if (c.n) MLODS_CUDA(cudaMemcpyAsync(keys.data(), c.a, size_t(c.n) * 8, cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    return MLODS_OK;
}

// ---- kernels of the generator

// aabb_octree over [-1, 1]^3: cell centre, float arithmetic (octree.h:944-955)
__global__ void centres_kernel(const uint64_t* __restrict__ k, int64_t n, float* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = k[i];
    const float w = __fdiv_rn(2.0f, float(1 << key_depth(key)));
    const int p[3] = {key_x(key), key_y(key), key_z(key)};
    for (int a = 0; a < 3; ++a) {
        const float lo = __fadd_rn(-1.0f, __fmul_rn(w, float(p[a])));
        const float hi = __fadd_rn(-1.0f, __fmul_rn(w, float(p[a] + 1)));
        out[3 * i + a] = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
    }
}

// find_stable_nodesGPU's per-cell step: the cell at the same depth enclosing
// the projected centre (aabb_octree::enclosing, octree.h:957-965), or the
// root when the projection failed (|n|^2 < 0.5) or lands outside the key range
__global__ void enclosing_kernel(const uint64_t* __restrict__ k, int64_t n, const float* __restrict__ p,
                                 const float* __restrict__ nv, uint64_t* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d = key_depth(k[i]);
    const float n0 = nv[3 * i], n1 = nv[3 * i + 1], n2 = nv[3 * i + 2];
    const float l2 = __fadd_rn(__fadd_rn(__fmul_rn(n0, n0), __fmul_rn(n1, n1)), __fmul_rn(n2, n2));
    uint64_t r = make_key(0, 0, 0, 0);
    if (!(l2 < 0.5f)) {
        const float w = __fdiv_rn(1.0f, float(1 << d));
        int c[3];
        bool ok = true;
        for (int a = 0; a < 3; ++a) {
            const float t = floorf(__fdiv_rn(__fdiv_rn(__fsub_rn(p[3 * i + a], -1.0f), 2.0f), w));
            ok = ok && t >= float(-kBias) && t < float(kBias);
            c[a] = ok ? int(t) : 0;
        }
        if (ok) r = make_key(d, c[0], c[1], c[2]);
    }
    out[i] = r;
}

// compute_leaves' children + expand(depth + 1): a kept cell at the level
// depth gives the 4x4x4 block around its children (the union of their
// 27-neighbourhoods); a root kept for a failed projection deeper down gives
// its 8 children only (they are not at depth + 1, so not expanded)
__global__ void children_block_kernel(const uint64_t* __restrict__ k, int64_t n, int depth,
                                      uint64_t* __restrict__ out, const uint32_t* __restrict__ out_off)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = k[i];
    const int d = key_depth(key);
    const int x = 2 * key_x(key), y = 2 * key_y(key), z = 2 * key_z(key);
    uint64_t* o = out + out_off[i];
    if (d == depth) {
        int m = 0;
        for (int dz = -1; dz <= 2; ++dz)
            for (int dy = -1; dy <= 2; ++dy)
                for (int dx = -1; dx <= 2; ++dx) o[m++] = make_key(d + 1, x + dx, y + dy, z + dz);
    } else {
        for (int c = 0; c < 8; ++c) o[c] = make_key(d + 1, x + (c & 1), y + ((c >> 1) & 1), z + ((c >> 2) & 1));
    }
}

__global__ void block_sizes_kernel(const uint64_t* __restrict__ k, int64_t n, int depth, uint32_t* __restrict__ sz)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) sz[i] = key_depth(k[i]) == depth ? 64u : 8u;
}

__global__ void ancestor_kernel(const uint64_t* __restrict__ k, int64_t n, int depth, uint64_t* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = key_ancestor(k[i], depth);
}

// min / max of the depth-0 ancestors' positions (getRelativeDepth, union_nodes)
__global__ void root_box_kernel(const uint64_t* __restrict__ k, int64_t n, int only_depth0, int* __restrict__ mm)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (only_depth0 && key_depth(k[i]) != 0) return;
    const uint64_t a = key_ancestor(k[i], 0);
    const int p[3] = {key_x(a), key_y(a), key_z(a)};
    for (int c = 0; c < 3; ++c) {
        atomicMin(mm + c, p[c]);
        atomicMax(mm + 3 + c, p[c]);
    }
}

// union_nodes' shift: pos -= min * 2^depth, depth += dd
__global__ void shift_kernel(uint64_t* __restrict__ k, int64_t n, int mx, int my, int mz, int dd, int* bad)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = k[i];
    const int d = key_depth(key);
    const int s = 1 << d;
    const int x = key_x(key) - mx * s, y = key_y(key) - my * s, z = key_z(key) - mz * s;
    if (!encodable(d + dd, x, y, z)) {
        atomicExch(bad, 1);
        return;
    }
    k[i] = make_key(d + dd, x, y, z);
}

// grade's step for the cells of one depth: parents of the 8 corner neighbours
// (neighbour ids 0, 2, 6, 8, 18, 20, 24, 26, upsample.cpp:69)
__global__ void grade_kernel(const uint64_t* __restrict__ k, int64_t n, uint64_t* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = k[i];
    const int d = key_depth(key), x = key_x(key), y = key_y(key), z = key_z(key);
    for (int c = 0; c < 8; ++c) {
        const int dx = (c & 1) ? 1 : -1, dy = (c & 2) ? 1 : -1, dz = (c & 4) ? 1 : -1;
        out[8 * i + c] = make_key(d - 1, fl_half(x + dx), fl_half(y + dy), fl_half(z + dz));
    }
}

__global__ void parent_kernel(const uint64_t* __restrict__ k, int64_t n, uint64_t* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = key_parent(k[i]);
}


// (depth, x, y, z) of every key, for the caller's cell array.
__global__ void key_cells_kernel(const uint64_t* __restrict__ k, int64_t n, int4* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_int4(key_depth(k[i]), key_x(k[i]), key_y(k[i]), key_z(k[i]));
}

// The 8 children of every cell.
__global__ void child8_kernel(const uint64_t* __restrict__ k, int64_t n, uint64_t* __restrict__ out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = k[i];
    const int d = key_depth(key) + 1, x = 2 * key_x(key), y = 2 * key_y(key), z = 2 * key_z(key);
    for (int c = 0; c < 8; ++c) out[8 * i + c] = make_key(d, x + (c & 1), y + ((c >> 1) & 1), z + ((c >> 2) & 1));
}

// The root cell (the default octree_id).
__global__ void root_key_kernel(uint64_t* __restrict__ out) { *out = make_key(0, 0, 0, 0); }

// First position of each depth in a sorted key set (the depth is the top 4
// bits of the key): one binary search per depth, thread d, d in [0, 16].
// aabb_octree::enclosing at `depth` of every point (octree.h:957-965):
// P = (p - min) / diag / w, floored, in float as the host does; a point whose
// cell has no key sets *bad.
__global__ void enclosing_points_kernel(const float* __restrict__ p, int64_t n, int depth, float3 bmin, float3 diag,
                                        float w, uint64_t* __restrict__ out, int* __restrict__ bad)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float lo[3] = {bmin.x, bmin.y, bmin.z}, dg[3] = {diag.x, diag.y, diag.z};
    int c[3];
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
        const float t = __fdiv_rn(__fdiv_rn(__fsub_rn(p[3 * i + a], lo[a]), dg[a]), w);
        const float f = floorf(t);
        if (!(f >= -float(kBias) && f < float(kBias))) {  // NaN too
            ok = false;
            c[a] = 0;
        } else {
            c[a] = int(f);
        }
    }
    if (!ok) atomicOr(bad, 1);
    out[i] = make_key(depth, c[0], c[1], c[2]);
}

__global__ void depth_bounds_kernel(const uint64_t* __restrict__ k, int64_t n, long long* __restrict__ begin)
{
    const int d = threadIdx.x;
    if (d > 16) return;
    if (d == 16) {
        begin[16] = n;
        return;
    }
    const uint64_t want = uint64_t(d) << 60;
    int64_t lo = 0, hi = n;  // first key >= want
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (k[mid] < want)
            lo = mid + 1;
        else
            hi = mid;
    }
    begin[d] = lo;
}

// ---- host orchestration

struct Gen {
    mlods_tree_s* T;
    cudaStream_t s;
    int64_t projected = 0;
    float* d_proj = nullptr;  // 9 floats per cell (centre, projection, normal)
    size_t proj_cap = 0;
    uint32_t* d_off = nullptr;  // block sizes, then their exclusive scan (+ total)
    size_t off_cap = 0;
    void* d_scan = nullptr;
    size_t scan_cap = 0;
    int* d_mm = nullptr;
    long long* d_begin = nullptr;
    ~Gen()
    {
        scratch_free(d_proj, s);
        scratch_free(d_off, s);
        scratch_free(d_scan, s);
        scratch_free(d_mm, s);
        scratch_free(d_begin, s);
    }

    // first key of each depth of a sorted set (17 entries)
    int depth_ranges(const CellSet& c, int64_t begin[17])
    {
        if (c.n == 0) {
            for (int d = 0; d < 17; ++d) begin[d] = 0;
            return MLODS_OK;
        }
        if (!d_begin) MLODS_CUDA(pool_alloc(&d_begin, 17 * sizeof(long long), s));
        depth_bounds_kernel<<<1, 32, 0, s>>>(c.a, c.n, d_begin);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        long long h[17];
        MLODS_CUDA(cudaMemcpyAsync(h, d_begin, sizeof h, cudaMemcpyDeviceToHost, s));
        MLODS_CUDA(cudaStreamSynchronize(s));
        for (int d = 0; d < 17; ++d) begin[d] = int64_t(h[d]);
        return MLODS_OK;
    }

    // find_stable_nodesGPU: out = sorted unique enclosing cells of the
    // projected centres of `cur`
    int stable(const CellSet& cur, CellSet& out)
    {
        out.n = 0;
        if (cur.n == 0) return MLODS_OK;
        const int64_t n = cur.n;
        if (proj_cap < size_t(n)) {
            scratch_free(d_proj, s);
            d_proj = nullptr;
            proj_cap = 0;
            MLODS_CUDA(pool_alloc(&d_proj, size_t(n) * 36, s));
            proj_cap = size_t(n);
        }
        float* c = d_proj;
        float* p = d_proj + 3 * n;
        float* nv = d_proj + 6 * n;
        centres_kernel<<<blocks_for(n), kThreads, 0, s>>>(cur.a, n, c);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        const int rc = project_buffers(T, n, c, p, nv, 1, FLT_MAX, s);
        if (rc != MLODS_OK) return rc;
        projected += n;
        int r2 = reserve(out, n, false, s);
        if (r2 != MLODS_OK) return r2;
        enclosing_kernel<<<blocks_for(n), kThreads, 0, s>>>(cur.a, n, p, nv, out.a);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        out.n = n;
        return sort_unique(out, s);
    }

    // children + 26-neighbour expansion of the kept cells of level `depth`
    int children(const CellSet& sub, int depth, CellSet& out)
    {
        out.n = 0;
        const int64_t n = sub.n;
        if (n == 0) return MLODS_OK;
        if (off_cap < size_t(n) + 1) {
            scratch_free(d_off, s);
            d_off = nullptr;
            off_cap = 0;
            MLODS_CUDA(pool_alloc(&d_off, (size_t(n) + 1) * 4, s));
            off_cap = size_t(n) + 1;
        }
        if (scan_cap < scan_temp_bytes(n)) {
            scratch_free(d_scan, s);
            d_scan = nullptr;
            scan_cap = 0;
            MLODS_CUDA(pool_alloc(&d_scan, scan_temp_bytes(n), s));
            scan_cap = scan_temp_bytes(n);
        }
        if (n > (int64_t(1) << 25)) {  // 64 keys each must stay within 32-bit offsets
            set_last_error("dc adaptive grid: %lld kept cells in one level exceed the supported 2^25", (long long)n);
            return MLODS_ERR_CAPACITY;
        }
        block_sizes_kernel<<<blocks_for(n), kThreads, 0, s>>>(sub.a, n, depth, d_off);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        MLODS_CUDA(exclusive_scan_u32(d_off, d_off, n, d_off + n, d_scan, s));
        uint32_t total32 = 0;
        MLODS_CUDA(cudaMemcpyAsync(&total32, d_off + n, 4, cudaMemcpyDeviceToHost, s));
        MLODS_CUDA(cudaStreamSynchronize(s));
        const int64_t acc = int64_t(total32);
        int rc = reserve(out, acc, false, s);
        if (rc != MLODS_OK) return rc;
        children_block_kernel<<<blocks_for(n), kThreads, 0, s>>>(sub.a, n, depth, out.a, d_off);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        MLODS_CUDA(cudaStreamSynchronize(s));
        out.n = acc;
        return sort_unique(out, s);
    }

    int root_box(const CellSet& c, bool only_depth0, int mn[3], int mx[3], bool* any)
    {
        if (!d_mm) MLODS_CUDA(pool_alloc(&d_mm, 8 * sizeof(int), s));
        const int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
        MLODS_CUDA(cudaMemcpyAsync(d_mm, init, sizeof init, cudaMemcpyHostToDevice, s));
        if (c.n) {
            root_box_kernel<<<blocks_for(c.n), kThreads, 0, s>>>(c.a, c.n, only_depth0 ? 1 : 0, d_mm);
            note_launch();
            MLODS_CUDA(cudaGetLastError());
        }
        int h[6];
        MLODS_CUDA(cudaMemcpyAsync(h, d_mm, sizeof h, cudaMemcpyDeviceToHost, s));
        MLODS_CUDA(cudaStreamSynchronize(s));
        *any = h[0] != INT_MAX;
        for (int k = 0; k < 3; ++k) {
            mn[k] = h[k];
            mx[k] = h[3 + k];
        }
        return MLODS_OK;
    }

    // keys at `depth` of a sorted set -> launch(keys, n, out) writes per_key
    // keys each; they are added to the set, which is sorted again
    template <typename Launch>
    int grow_level(CellSet& set, int depth, int per_key, CellSet& scratch, Launch launch)
    {
        int64_t begin[17];
        int rc = depth_ranges(set, begin);
        if (rc != MLODS_OK) return rc;
        const int64_t n = begin[depth + 1] - begin[depth];
        if (n == 0) return MLODS_OK;
        rc = reserve(scratch, n * per_key, false, s);
        if (rc != MLODS_OK) return rc;
        launch(set.a + begin[depth], n, scratch.a);
        MLODS_CUDA(cudaGetLastError());
        rc = append(set, scratch.a, n * per_key, s);
        if (rc != MLODS_OK) return rc;
        return sort_unique(set, s);
    }
};

int log2_ceil_extent(int ext) { return int(std::ceil(float(std::log2(double(ext))))); }

// OctreeGenerator::generate: the collected candidates, cut to the adaptive
// maximum depth, sorted and unique, in `total`
int generate(Gen& G, int max_depth, CellSet& total)
{
    cudaStream_t s = G.s;
    std::vector<uint64_t> depth0 = {make_key(0, 0, 0, 0)};
    std::vector<uint64_t> old_depth0;
    int max_rel = max_depth;
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {-INT_MAX, -INT_MAX, -INT_MAX};
    CellSet cur, sub;
    total.n = 0;
    while (!depth0.empty()) {
        int rc = upload(cur, depth0, s);
        if (rc != MLODS_OK) return rc;
        rc = append(total, cur.a, cur.n, s);
        if (rc != MLODS_OK) return rc;
        for (int depth = 0; depth < max_rel + 1; ++depth) {  // compute_leaves
            if (depth + 1 > kMaxKeyDepth) {
                set_last_error("dc adaptive grid: depth %d beyond the supported %d", depth + 1, kMaxKeyDepth);
                return MLODS_ERR_CAPACITY;
            }
            rc = G.stable(cur, sub);
            if (rc == MLODS_OK) rc = G.children(sub, depth, cur);
            if (rc == MLODS_OK) rc = append(total, cur.a, cur.n, s);
            if (rc != MLODS_OK) return rc;
        }
        // getRelativeDepth with the running min / max
        int cmn[3], cmx[3];
        bool any = false;
        rc = G.root_box(cur, false, cmn, cmx, &any);
        if (rc != MLODS_OK) return rc;
        int rd = 0;
        if (any) {
            for (int k = 0; k < 3; ++k) {
                mn[k] = std::min(mn[k], cmn[k]);
                mx[k] = std::max(mx[k], cmx[k]);
            }
            for (int k = 0; k < 3; ++k) rd = std::max(rd, log2_ceil_extent(mx[k] - mn[k] + 1));
        }
        max_rel = std::max(0, max_depth - rd);
        old_depth0.insert(old_depth0.end(), depth0.begin(), depth0.end());
        // depth0_ancestors(current), expand(-1), minus the cells already explored
        CellSet anc;
        rc = reserve(anc, cur.n, false, s);
        if (rc != MLODS_OK) return rc;
        if (cur.n) {
            ancestor_kernel<<<blocks_for(cur.n), kThreads, 0, s>>>(cur.a, cur.n, 0, anc.a);
            note_launch();
            MLODS_CUDA(cudaGetLastError());
        }
        anc.n = cur.n;
        rc = sort_unique(anc, s);
        std::vector<uint64_t> a0;
        if (rc == MLODS_OK) rc = download(anc, a0, s);
        if (rc != MLODS_OK) return rc;
        std::vector<Cell> next;
        for (uint64_t k : a0) next.push_back(key_cell(k));
        dcg::expand(next, -1);
        std::vector<uint64_t> seen = old_depth0;
        std::sort(seen.begin(), seen.end());
        depth0.clear();
        for (const Cell& c : next) {
            if (!encodable(c.depth, c.x, c.y, c.z)) continue;
            const uint64_t k = make_key(c.depth, c.x, c.y, c.z);
            if (!std::binary_search(seen.begin(), seen.end(), k)) depth0.push_back(k);
        }
        if (old_depth0.size() + depth0.size() > kMaxRootCells) {
            set_last_error("dc adaptive grid: the surface spans more than %zu unit cells", kMaxRootCells);
            return MLODS_ERR_CAPACITY;
        }
    }
    // onlySetDepthNodes(total_tree, max_rel)
    CellSet tmp;
    int rc = reserve(tmp, total.n, false, s);
    if (rc != MLODS_OK) return rc;
    if (total.n) {
        ancestor_kernel<<<blocks_for(total.n), kThreads, 0, s>>>(total.a, total.n, max_rel, tmp.a);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        MLODS_CUDA(cudaMemcpyAsync(total.a, tmp.a, size_t(total.n) * 8, cudaMemcpyDeviceToDevice, s));
    }
    return sort_unique(total, s);
}

int grade_up_siblings(Gen& G, CellSet& nodes, int cut_depth, CellSet& scratch);

// uniformize (upsample.cpp:262-273) on the device
int uniformize(Gen& G, CellSet& nodes, int max_depth, bool cut, float nd[3], float no[3])
{
    cudaStream_t s = G.s;
    CellSet scratch;
    // nodes + depth0_ancestors(nodes)
    int rc = reserve(scratch, nodes.n, false, s);
    if (rc != MLODS_OK) return rc;
    if (nodes.n) {
        ancestor_kernel<<<blocks_for(nodes.n), kThreads, 0, s>>>(nodes.a, nodes.n, 0, scratch.a);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
    }
    rc = append(nodes, scratch.a, nodes.n, s);
    if (rc == MLODS_OK) rc = sort_unique(nodes, s);
    if (rc != MLODS_OK) return rc;
    // retreiveCorrectRoot / union_nodes
    int mn[3], mx[3];
    bool any = false;
    rc = G.root_box(nodes, true, mn, mx, &any);
    if (rc != MLODS_OK) return rc;
    int dd = 0;
    if (any)
        for (int k = 0; k < 3; ++k) dd = std::max(dd, log2_ceil_extent(mx[k] - mn[k] + 1));
    for (int k = 0; k < 3; ++k) {
        nd[k] = 1.0f;
        no[k] = 0.0f;
    }
    if (any && dd > 0) {
        int* d_bad = G.d_mm + 6;
        MLODS_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
        shift_kernel<<<blocks_for(nodes.n), kThreads, 0, s>>>(nodes.a, nodes.n, mn[0], mn[1], mn[2], dd, d_bad);
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        int bad = 0;
        MLODS_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, s));
        MLODS_CUDA(cudaStreamSynchronize(s));
        if (bad) {
            set_last_error("dc adaptive grid: the shifted grid exceeds the supported depth or extent");
            return MLODS_ERR_CAPACITY;
        }
        rc = sort_unique(nodes, s);  // the shift keeps the order within a depth only
        if (rc != MLODS_OK) return rc;
        for (int k = 0; k < 3; ++k) {
            no[k] = float(mn[k]);
            nd[k] = float(1 << dd);
        }
    }
    return grade_up_siblings(G, nodes, cut ? max_depth : -1, scratch);
}

// grade, regularize_up, the optional cut and regularize_siblings
// (upsample.cpp:40-93, :253-273) on a sorted unique set
// Adds m keys made by `launch` (which writes them at the given address) to
// set c and makes it sorted and unique again.
template <typename Launch>
int add_sorted(CellSet& c, int64_t m, cudaStream_t s, Launch launch)
{
    if (m <= 0) return MLODS_OK;
    int rc = reserve(c, c.n + m, true, s);
    if (rc != MLODS_OK) return rc;
    launch(c.a + c.n);
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    c.n += m;
    return sort_unique(c, s);
}

// grade, regularize_up, the optional cut and regularize_siblings on one set
// per depth: every step makes keys of a single depth (grade and the
// ancestors one level up, the siblings at their own level), so only that
// level is sorted again, and the levels concatenated in depth order are the
// sorted set (the depth is the key's top bits).
int grade_up_siblings(Gen& G, CellSet& nodes, int cut_depth, CellSet& scratch)
{
    cudaStream_t s = G.s;
    int64_t begin[17];
    int rc = G.depth_ranges(nodes, begin);
    if (rc != MLODS_OK) return rc;
    CellSet L[16];
    int deepest = 0;
    for (int d = 0; d < 16; ++d) {
        const int64_t n = begin[d + 1] - begin[d];
        L[d].s = s;
        if (n == 0) continue;
        deepest = d;
        rc = reserve(L[d], n, false, s);
        if (rc != MLODS_OK) return rc;
        MLODS_CUDA(cudaMemcpyAsync(L[d].a, nodes.a + begin[d], size_t(n) * 8, cudaMemcpyDeviceToDevice, s));
        L[d].n = n;
    }
    // grade, deepest level first (the order of the reference's loop): the
    // parents of a cell's 8 corner neighbours join the level above
    for (int d = deepest; d >= 1; --d) {
        const uint64_t* k = L[d].a;
        const int64_t n = L[d].n;
        rc = add_sorted(L[d - 1], 8 * n, s, [&](uint64_t* out) {
            grade_kernel<<<blocks_for(n), kThreads, 0, s>>>(k, n, out);
        });
        if (rc != MLODS_OK) return rc;
    }
    // regularize_up: every ancestor
    for (int d = deepest; d >= 1; --d) {
        const uint64_t* k = L[d].a;
        const int64_t n = L[d].n;
        rc = add_sorted(L[d - 1], n, s, [&](uint64_t* out) {
            parent_kernel<<<blocks_for(n), kThreads, 0, s>>>(k, n, out);
        });
        if (rc != MLODS_OK) return rc;
    }
    const int top = cut_depth >= 0 ? std::min(deepest, std::min(cut_depth, 15)) : deepest;
    // regularize_siblings: a level becomes the children of its cells'
    // parents (each cell is one of them); depth-0 cells add the root
    for (int d = 1; d <= top; ++d) {
        if (L[d].n == 0) continue;
        const uint64_t* k = L[d].a;
        const int64_t n = L[d].n;
        scratch.n = 0;
        rc = add_sorted(scratch, n, s, [&](uint64_t* out) {
            parent_kernel<<<blocks_for(n), kThreads, 0, s>>>(k, n, out);
        });
        if (rc != MLODS_OK) return rc;
        const uint64_t* pk = scratch.a;
        const int64_t np = scratch.n;
        L[d].n = 0;
        rc = add_sorted(L[d], 8 * np, s, [&](uint64_t* out) {
            child8_kernel<<<blocks_for(np), kThreads, 0, s>>>(pk, np, out);
        });
        if (rc != MLODS_OK) return rc;
    }
    if (L[0].n > 0) {
        rc = add_sorted(L[0], 1, s, [&](uint64_t* out) { root_key_kernel<<<1, 1, 0, s>>>(out); });
        if (rc != MLODS_OK) return rc;
    }
    nodes.n = 0;
    for (int d = 0; d <= top; ++d) {
        rc = append(nodes, L[d].a, L[d].n, s);
        if (rc != MLODS_OK) return rc;
    }
    return MLODS_OK;
}

}  // namespace

int dcgrid_from_points_device(const float* pts, int64_t n, int max_depth, const float box_min[3],
                              const float box_max[3], cudaStream_t s, std::vector<int32_t>& cells_out, int& depth_out,
                              bool* handled)
{
    *handled = false;
    if (n <= 0 || !pts || max_depth < 0 || max_depth > kMaxKeyDepth) return MLODS_OK;  // the host path decides
    float3 lo = make_float3(box_min[0], box_min[1], box_min[2]);
    float3 dg = make_float3(box_max[0] - box_min[0], box_max[1] - box_min[1], box_max[2] - box_min[2]);
    if (!(dg.x > 0.f && dg.y > 0.f && dg.z > 0.f)) return MLODS_OK;
    Gen G{nullptr, s};
    CellSet nodes, scratch;
    int rc = reserve(nodes, n, false, s);
    if (rc != MLODS_OK) return rc;
    float* d_pts = nullptr;
    MLODS_CUDA(scratch_alloc(reinterpret_cast<void**>(&d_pts), size_t(n) * 12 + 256, s));
    int* d_bad = reinterpret_cast<int*>(reinterpret_cast<char*>(d_pts) + ((size_t(n) * 12 + 15) / 16) * 16);
    cudaError_t e = cudaMemcpyAsync(d_pts, pts, size_t(n) * 12, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        const float w = 1.0f / float(1 << max_depth);
        enclosing_points_kernel<<<blocks_for(n), kThreads, 0, s>>>(d_pts, n, max_depth, lo, dg, w, nodes.a, d_bad);
        note_launch();
        e = cudaGetLastError();
    }
    int bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    scratch_free(d_pts, s);
    if (e != cudaSuccess) return cuda_fail(e, "dc grid from points", __FILE__, __LINE__);
    if (bad) return MLODS_OK;  // points off the key range: the host path
    nodes.n = n;
    rc = sort_unique(nodes, s);  // remove_duplicates
    if (rc == MLODS_OK) rc = grade_up_siblings(G, nodes, -1, scratch);  // uniformizeFromPoints
    if (rc != MLODS_OK) return rc;
    rc = cells_to_host(nodes, cells_out, depth_out, s);
    if (rc != MLODS_OK) return rc;
    *handled = true;
    return MLODS_OK;
}

int dcgrid_adaptive(mlods_tree_s* T, int max_depth, bool cut, cudaStream_t s, std::vector<int32_t>& cells_out,
                    int& depth_out, float xform[12], int64_t* n_projected)
{
    if (max_depth < 0 || max_depth > 12) {
        set_last_error("dc adaptive grid: max_depth=%d out of range [0, 12]", max_depth);
        return MLODS_ERR_INVALID;
    }
    if (!T->kernel_set) {
        set_last_error("dc adaptive grid: no kernel set (call mlods_set_kernel first)");
        return MLODS_ERR_STATE;
    }
    // the generator projects with the APSS object's project(), the MLoD (or
    // global) projection even when the octree is in kNN / ball mode
    const int saved_mode = T->params.mode;
    if (saved_mode == MLODS_MODE_KNN || saved_mode == MLODS_MODE_BALL) T->params.mode = MLODS_MODE_MLOD;
    Gen G{T, s};
    CellSet nodes;
    int rc = generate(G, max_depth, nodes);
    T->params.mode = saved_mode;
    if (rc != MLODS_OK) return rc;
    if (n_projected) *n_projected = G.projected;
    float nd[3], no[3];
    rc = uniformize(G, nodes, max_depth, cut, nd, no);
    if (rc != MLODS_OK) return rc;
    rc = cells_to_host(nodes, cells_out, depth_out, s);
    if (rc != MLODS_OK) return rc;
    // new2bbox = unit2bbox * sortedOctreeToUnit (scene.cpp:1259-1311), box [-1, 1]^3
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 4; ++c) xform[4 * r + c] = 0.f;
        xform[4 * r + r] = 2.0f * nd[r];
        xform[4 * r + 3] = 2.0f * no[r] + -1.0f;
    }
    return MLODS_OK;
}

}  // namespace mlods
