// tree_build.cu -- device octree build with the reference's exact topology.
//
// The reference builds its octree on the host by recursive midpoint splits
// (CPUUtils.cpp:271-329): split = (bb + BB) / 2.0 with the sum of the float
// bounds rounded to float first (so every split is a float value), child
// boxes stored as float, 1 point per leaf, depth <= maxDepth.  Each axis splits
// independently, so the split values form one binary table per axis that
// depends only on the root box.  A point's cell at every depth is therefore a
// binary descent through three tables, its path a Morton code (x lowest bit,
// child slot c = xi + 2yi + 4zi), and the reference tree is the set of
// Morton prefixes that hold at least two points one level up.  Breadth-first
// order (CPUUtils.cpp:601-619) is level-major Morton-prefix order.
//
// Passes (all on the device, one grid each):
//   bbox -> split tables (host, 3 x 4095 doubles) -> Morton codes -> radix
//   sort -> common-prefix lengths -> per-level node counts -> scan ->
//   node emission -> sibling links -> leaf areas -> bottom-up moments
//   (double, centred, parallel-axis merges) -> 64-byte node records.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "primitives.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
constexpr int kThreads = 256;
constexpr int kItems = 8;  // contiguous points per thread in the level passes
constexpr int kTile = kThreads * kItems;
constexpr int kLevels = kMaxTreeDepth + 1;

inline unsigned grid_for(int64_t n, int threads) { return unsigned((n + threads - 1) / threads); }

__global__ void bbox_kernel(const float* __restrict__ pts, int64_t n, float* __restrict__ out, int* __restrict__ bad)
{
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool finite = true;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            float v = pts[3 * i + a];
            finite = finite && isfinite(v);
            lo[a] = fminf(lo[a], v);
            hi[a] = fmaxf(hi[a], v);
        }
    if (!finite) atomicOr(bad, 1);
    __shared__ float s[6][kThreads];
    for (int a = 0; a < 3; ++a) {
        s[a][threadIdx.x] = lo[a];
        s[3 + a][threadIdx.x] = hi[a];
    }
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int a = 0; a < 3; ++a) {
                s[a][threadIdx.x] = fminf(s[a][threadIdx.x], s[a][threadIdx.x + w]);
                s[3 + a][threadIdx.x] = fmaxf(s[3 + a][threadIdx.x], s[3 + a][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) out[6 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

// Per point: cell path on each axis (compare as double against the double
// split, CPUUtils.cpp:298-308), interleaved into a Morton code, and the first
// depth at which the coordinate equals a split (255 if none).
__global__ void morton_kernel(const float* __restrict__ pts, int64_t n, int D, const double* __restrict__ splits,
                              int64_t split_stride, uint64_t* __restrict__ codes, uint32_t* __restrict__ idx,
                              uint8_t* __restrict__ tie_level)
{
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t cell[3];
    int tie = 255;
    for (int a = 0; a < 3; ++a) {
        const double x = double(pts[3 * i + a]);
        const double* S = splits + a * split_stride;
        uint32_t k = 0;
        for (int d = 0; d < D; ++d) {
            const double s = __ldg(S + ((1u << d) - 1u) + k);
            if (x == s && tie == 255) tie = d;
            k = 2u * k + (x > s ? 1u : 0u);
        }
        cell[a] = k;
    }
    uint64_t code = 0;
    for (int d = 0; d < D; ++d) {
        const int b = D - 1 - d;
        const uint64_t g = ((cell[0] >> b) & 1u) | (((cell[1] >> b) & 1u) << 1) | (((cell[2] >> b) & 1u) << 2);
        code |= g << (3 * b);
    }
    codes[i] = code;
    idx[i] = uint32_t(i);
    tie_level[i] = uint8_t(tie);
}

__device__ __forceinline__ int common_levels(uint64_t a, uint64_t b, int D)
{
    const uint64_t x = a ^ b;
    if (x == 0) return D;
    const int h = 63 - __clzll((long long)x);
    return (3 * D - 1 - h) / 3;
}

// lcp[i]: levels shared with the previous sorted code (-1 for i == 0);
// leafd[i]: depth of the leaf that holds point i (first depth at which it is
// alone in its cell, capped at D).
__global__ void lcp_kernel(const uint64_t* __restrict__ codes, int64_t n, int D, int8_t* __restrict__ lcp,
                           int8_t* __restrict__ leafd)
{
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t c = codes[i];
    const int lp = i == 0 ? -1 : common_levels(codes[i - 1], c, D);
    const int ln = i == n - 1 ? -1 : common_levels(c, codes[i + 1], D);
    lcp[i] = int8_t(lp);
    leafd[i] = int8_t(min(D, max(lp, ln) + 1));
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// counts[d * nb + b] = number of nodes at depth d headed by points of tile b.
__global__ void level_count_kernel(const int8_t* __restrict__ lcp, const int8_t* __restrict__ leafd, int64_t n,
                                   int D, int nb, uint32_t* __restrict__ counts)
{
    __shared__ uint32_t s[kLevels][kThreads / 32];
    const int64_t base = int64_t(blockIdx.x) * kTile + int64_t(threadIdx.x) * kItems;
    int lo[kItems], hi[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const int64_t i = base + k;
        lo[k] = i < n ? lcp[i] + 1 : 1;
        hi[k] = i < n ? leafd[i] : 0;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < kLevels; ++d) {
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k) c += (lo[k] <= d && d <= hi[k]) ? 1u : 0u;
        c = warp_sum(c);
        if (lane == 0) s[d][warp] = c;
    }
    __syncthreads();
    if (threadIdx.x < kLevels) {
        uint32_t t = 0;
        for (int w = 0; w < kThreads / 32; ++w) t += s[threadIdx.x][w];
        if (threadIdx.x <= D) counts[int64_t(threadIdx.x) * nb + blockIdx.x] = t;
    }
}

__device__ __forceinline__ uint32_t warp_incl(uint32_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t x = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += x;
    }
    return v;
}

// Assigns breadth-first indices: node (point i, depth d) gets
// base[d][tile] + rank among the tile's emitters at d (point order).
// Writes head/level/first flags and the chain links inside one point's
// nodes: node (i, d+1) is the first child of node (i, d).
__global__ void level_emit_kernel(const int8_t* __restrict__ lcp, const int8_t* __restrict__ leafd, int64_t n, int D,
                                  int nb, const uint32_t* __restrict__ bases, int32_t* __restrict__ head,
                                  uint8_t* __restrict__ level, uint8_t* __restrict__ is_first,
                                  int32_t* __restrict__ parent, int32_t* __restrict__ first_child)
{
    __shared__ uint32_t s_warp[kThreads / 32 + 1];
    const int64_t base = int64_t(blockIdx.x) * kTile + int64_t(threadIdx.x) * kItems;
    int lo[kItems], hi[kItems], lp[kItems];
    int32_t prev[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const int64_t i = base + k;
        lp[k] = i < n ? lcp[i] : 0;
        lo[k] = i < n ? lp[k] + 1 : 1;
        hi[k] = i < n ? leafd[i] : 0;
        prev[k] = -1;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d <= D; ++d) {
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k) c += (lo[k] <= d && d <= hi[k]) ? 1u : 0u;
        const uint32_t incl = warp_incl(c);
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = lane < kThreads / 32 ? s_warp[lane] : 0u;
            uint32_t wi = warp_incl(w);
            if (lane < kThreads / 32) s_warp[lane] = wi - w;
        }
        __syncthreads();
        uint32_t id = bases[int64_t(d) * nb + blockIdx.x] + s_warp[warp] + incl - c;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (lo[k] <= d && d <= hi[k]) {
                head[id] = int32_t(base + k);
                level[id] = uint8_t(d);
                const bool first = (d == 0) || (lp[k] < d - 1);
                is_first[id] = first ? 1 : 0;
                if (prev[k] >= 0) {
                    parent[id] = prev[k];
                    first_child[prev[k]] = int32_t(id);
                } else {
                    parent[id] = -1;
                }
                prev[k] = int32_t(id);
                ++id;
            }
        }
    }
}

// Siblings of one parent are contiguous within a level; the first of them
// knows its parent from the emission chain.  Non-first nodes copy it; first
// nodes count their group and store it in the parent.
__global__ void links_kernel(int64_t n_nodes, const uint8_t* __restrict__ level, const uint8_t* __restrict__ is_first,
                             const int64_t* __restrict__ level_off, int32_t* __restrict__ parent,
                             int32_t* __restrict__ n_children)
{
    int64_t id = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= n_nodes) return;
    const int d = level[id];
    if (d == 0) return;
    const int64_t end = level_off[d + 1];
    if (!is_first[id]) {
        int64_t k = id - 1;
        while (!is_first[k]) --k;
        parent[id] = parent[k];
    } else {
        int c = 1;
        while (id + c < end && !is_first[id + c]) ++c;
        n_children[parent[id]] = c;
    }
}

__device__ __forceinline__ void cell_coords(uint64_t code, int D, int d, uint32_t c[3])
{
    c[0] = c[1] = c[2] = 0;
    for (int l = 0; l < d; ++l) {
        const uint32_t g = uint32_t(code >> (3 * (D - 1 - l))) & 7u;
        c[0] = (c[0] << 1) | (g & 1u);
        c[1] = (c[1] << 1) | ((g >> 1) & 1u);
        c[2] = (c[2] << 1) | ((g >> 2) & 1u);
    }
}

__device__ __forceinline__ void node_box(const float* __restrict__ bounds, int64_t stride, uint64_t code, int D,
                                         int d, float bb[3], float BB[3])
{
    uint32_t c[3];
    cell_coords(code, D, d, c);
    const int64_t off = ((int64_t(1) << d) - 1) + d;
    for (int a = 0; a < 3; ++a) {
        bb[a] = bounds[a * stride + off + c[a]];
        BB[a] = bounds[a * stride + off + c[a] + 1];
    }
}

// Leaf point counts, per-sample areas (CPUUtils.cpp:236-252, float as the
// reference: diag^2 / #points) and the tie count.
__global__ void leaf_kernel(int64_t n_nodes, int64_t n, int D, const uint8_t* __restrict__ level,
                            const int32_t* __restrict__ head, const int32_t* __restrict__ first_child,
                            const int8_t* __restrict__ lcp, const int8_t* __restrict__ leafd,
                            const uint64_t* __restrict__ codes, const uint32_t* __restrict__ perm,
                            const float* __restrict__ bounds, int64_t stride, int32_t* __restrict__ leaf_cnt,
                            float* __restrict__ area, const uint8_t* __restrict__ tie_level,
                            unsigned long long* __restrict__ n_ties)
{
    int64_t id = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= n_nodes) return;
    if (first_child[id] >= 0) {
        leaf_cnt[id] = 0;
        return;
    }
    const int d = level[id];
    const int64_t h = head[id];
    int64_t cnt = 1;
    if (d == D)
        while (h + cnt < n && lcp[h + cnt] == D) ++cnt;
    leaf_cnt[id] = int32_t(cnt);
    float bb[3], BB[3];
    node_box(bounds, stride, codes[h], D, d, bb, BB);
    const float dx = __fsub_rn(BB[0], bb[0]), dy = __fsub_rn(BB[1], bb[1]), dz = __fsub_rn(BB[2], bb[2]);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    const float diag = __fsqrt_rn(d2);
    const float a = __fdiv_rn(__fmul_rn(diag, diag), float(cnt));
    unsigned long long ties = 0;
    for (int64_t k = 0; k < cnt; ++k) {
        const uint32_t orig = perm[h + k];
        area[orig] = a;
        if (int(tie_level[orig]) < int(leafd[h + k])) ++ties;
    }
    if (ties) atomicAdd(n_ties, ties);
}

// Bottom-up centred moments, one depth per launch (deepest first).
// mom: {m0, pbar[3] (local), n[3], cpn, cpp} in double.
__global__ void moments_kernel(int64_t lo, int64_t hi, const int32_t* __restrict__ head,
                               const int32_t* __restrict__ first_child, const int32_t* __restrict__ n_children,
                               const int32_t* __restrict__ leaf_cnt, const uint32_t* __restrict__ perm,
                               const float* __restrict__ pts, const float* __restrict__ nrm,
                               const float* __restrict__ area, double o0, double o1, double o2,
                               double* __restrict__ mom)
{
    const int64_t id = lo + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= hi) return;
    double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int32_t fc = first_child[id];
    if (fc < 0) {
        const int64_t h = head[id];
        const int cnt = leaf_cnt[id];
        double sp[3] = {0, 0, 0};
        for (int k = 0; k < cnt; ++k) {
            const uint32_t i = perm[h + k];
            const double a = area[i];
            m[0] += a;
            sp[0] += a * (double(pts[3 * i]) - o0);
            sp[1] += a * (double(pts[3 * i + 1]) - o1);
            sp[2] += a * (double(pts[3 * i + 2]) - o2);
        }
        for (int c = 0; c < 3; ++c) m[1 + c] = sp[c] / m[0];
        for (int k = 0; k < cnt; ++k) {
            const uint32_t i = perm[h + k];
            const double a = area[i];
            const double d0 = double(pts[3 * i]) - o0 - m[1];
            const double d1 = double(pts[3 * i + 1]) - o1 - m[2];
            const double d2 = double(pts[3 * i + 2]) - o2 - m[3];
            const double n0 = nrm[3 * i], n1 = nrm[3 * i + 1], n2 = nrm[3 * i + 2];
            m[4] += a * n0;
            m[5] += a * n1;
            m[6] += a * n2;
            m[7] += a * (d0 * n0 + d1 * n1 + d2 * n2);
            m[8] += a * (d0 * d0 + d1 * d1 + d2 * d2);
        }
    } else {
        const int nc = n_children[id];
        double M = 0, sp[3] = {0, 0, 0};
        for (int c = 0; c < nc; ++c) {
            const double* cm = mom + 9 * int64_t(fc + c);
            M += cm[0];
            sp[0] += cm[0] * cm[1];
            sp[1] += cm[0] * cm[2];
            sp[2] += cm[0] * cm[3];
        }
        m[0] = M;
        for (int c = 0; c < 3; ++c) m[1 + c] = sp[c] / M;
        for (int c = 0; c < nc; ++c) {
            const double* cm = mom + 9 * int64_t(fc + c);
            const double d0 = cm[1] - m[1], d1 = cm[2] - m[2], d2 = cm[3] - m[3];
            m[4] += cm[4];
            m[5] += cm[5];
            m[6] += cm[6];
            m[7] += cm[7] + d0 * cm[4] + d1 * cm[5] + d2 * cm[6];
            m[8] += cm[8] + cm[0] * (d0 * d0 + d1 * d1 + d2 * d2);
        }
    }
    double* out = mom + 9 * id;
    for (int c = 0; c < 9; ++c) out[c] = m[c];
}

__global__ void multi_count_kernel(int64_t n_nodes, const int32_t* __restrict__ leaf_cnt, uint32_t* __restrict__ cnt)
{
    int64_t id = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= n_nodes) return;
    const int c = leaf_cnt[id];
    cnt[id] = c > 1 ? uint32_t(c) : 0u;
}

__global__ void write_nodes_kernel(int64_t n_nodes, int D, const uint8_t* __restrict__ level,
                                   const int32_t* __restrict__ head, const int32_t* __restrict__ parent,
                                   const int32_t* __restrict__ first_child, const int32_t* __restrict__ n_children,
                                   const int32_t* __restrict__ leaf_cnt, const uint32_t* __restrict__ extra_off,
                                   const uint64_t* __restrict__ codes, const uint32_t* __restrict__ perm,
                                   const float* __restrict__ bounds, int64_t stride, const double* __restrict__ mom,
                                   double o0, double o1, double o2, NodeArrays nodes)
{
    int64_t id = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= n_nodes) return;
    const int d = level[id];
    const int64_t h = head[id];
    float bb[3], BB[3];
    node_box(bounds, stride, codes[h], D, d, bb, BB);
    DNode nd;
    nd.cx = float((double(bb[0]) + double(BB[0])) * 0.5 - o0);
    nd.cy = float((double(bb[1]) + double(BB[1])) * 0.5 - o1);
    nd.cz = float((double(bb[2]) + double(BB[2])) * 0.5 - o2);
    const float dx = __fsub_rn(BB[0], bb[0]), dy = __fsub_rn(BB[1], bb[1]), dz = __fsub_rn(BB[2], bb[2]);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    nd.r = __fdiv_rn(__fsqrt_rn(d2), 2.f);
    const double* m = mom + 9 * id;
    nd.px = float(m[1]);
    nd.py = float(m[2]);
    nd.pz = float(m[3]);
    nd.m0 = float(m[0]);
    nd.nx = float(m[4]);
    nd.ny = float(m[5]);
    nd.nz = float(m[6]);
    nd.cpn = float(m[7]);
    nd.cpp = float(m[8]);
    uint32_t info = uint32_t(d) << kDepthShift;
    const int32_t fc = first_child[id];
    if (fc >= 0) {
        nd.first = uint32_t(fc);
        info |= uint32_t(n_children[id]) & kCountMask;
    } else {
        const int cnt = leaf_cnt[id];
        info |= kLeafBit | (uint32_t(cnt) & kCountMask);
        if (cnt > 1) {
            info |= kMultiBit;
            nd.first = uint32_t(n_nodes + extra_off[id]);
        } else {
            nd.first = perm[h];
        }
    }
    nd.info = info;
    nd.parent = parent[id] < 0 ? 0xFFFFFFFFu : uint32_t(parent[id]);
    store_node(nodes, id, nd);
}

__global__ void write_point_records_kernel(int64_t n_nodes, const int32_t* __restrict__ head,
                                           const int32_t* __restrict__ leaf_cnt, const uint32_t* __restrict__ extra_off,
                                           const uint8_t* __restrict__ level, const uint32_t* __restrict__ perm,
                                           const float* __restrict__ pts, const float* __restrict__ nrm,
                                           const float* __restrict__ area, double o0, double o1, double o2,
                                           NodeArrays nodes)
{
    int64_t id = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= n_nodes) return;
    const int cnt = leaf_cnt[id];
    if (cnt <= 1) return;
    const int64_t h = head[id];
    for (int k = 0; k < cnt; ++k) {
        const uint32_t i = perm[h + k];
        const double a = area[i];
        DNode pr;
        pr.px = pr.cx = float(double(pts[3 * i]) - o0);
        pr.py = pr.cy = float(double(pts[3 * i + 1]) - o1);
        pr.pz = pr.cz = float(double(pts[3 * i + 2]) - o2);
        pr.r = 0.f;
        pr.m0 = float(a);
        pr.nx = float(a * nrm[3 * i]);
        pr.ny = float(a * nrm[3 * i + 1]);
        pr.nz = float(a * nrm[3 * i + 2]);
        pr.cpn = 0.f;
        pr.cpp = 0.f;
        pr.first = i;
        pr.info = kLeafBit | 1u | (uint32_t(level[id] + 1 < 31 ? level[id] + 1 : 31) << kDepthShift);
        pr.parent = uint32_t(id);
        store_node(nodes, n_nodes + extra_off[id] + k, pr);
    }
}

__global__ void sorted_points_kernel(int64_t n, const uint32_t* __restrict__ perm, const float* __restrict__ pts,
                                     const float* __restrict__ nrm, double o0, double o1, double o2,
                                     float4* __restrict__ spts, float4* __restrict__ snrm,
                                     float4* __restrict__ wspts)
{
    int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = perm[j];
    spts[j] = make_float4(float(double(pts[3 * i]) - o0), float(double(pts[3 * i + 1]) - o1),
                          float(double(pts[3 * i + 2]) - o2), __uint_as_float(i));
    snrm[j] = make_float4(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2], 0.f);
    wspts[j] = make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], __uint_as_float(i));
}

inline size_t al(size_t v) { return (v + 255) / 256 * 256; }

// A simple bump allocator over one cudaMalloc'd block of build temporaries.
struct Bump {
    char* base = nullptr;
    size_t off = 0, cap = 0;
    template <typename T>
    T* take(size_t count)
    {
        T* p = reinterpret_cast<T*>(base + off);
        off += al(count * sizeof(T));
        return p;
    }
};

}  // namespace

void free_tree_device(mlods_tree_s* T)
{
    cudaFree(T->nodes.geom);
    cudaFree(T->d_node_head);
    cudaFree(T->d_codes);
    cudaFree(T->d_perm);
    cudaFree(T->d_area);
    cudaFree(T->d_spts);
    cudaFree(T->d_snrm);
    cudaFree(T->d_wspts);
    cudaFree(T->d_bounds);
    T->nodes = NodeArrays{};
    T->d_node_head = nullptr;
    T->d_codes = nullptr;
    T->d_perm = nullptr;
    T->d_area = nullptr;
    T->d_spts = nullptr;
    T->d_snrm = nullptr;
    T->d_wspts = nullptr;
    T->d_bounds = nullptr;
}

int build_tree(mlods_tree_s* T, const float* d_pts, const float* d_nrm, int64_t n, int D, cudaStream_t s)
{
    if (n <= 0 || n >= (int64_t(1) << 31)) {
        set_last_error("tree build: n=%lld out of range [1, 2^31)", (long long)n);
        return MLODS_ERR_INVALID;
    }
    if (D < 0 || D > kMaxTreeDepth) {
        set_last_error("tree build: max_depth=%d out of range [0, %d]", D, kMaxTreeDepth);
        return MLODS_ERR_INVALID;
    }
    MLODS_CUDA(cudaGetDevice(&T->device));
    T->n_pts = n;
    T->max_depth = D;

    // ---- root box (CPUUtils.cpp:571-579)
    const int nbb = int(std::min<int64_t>(1024, (n + kThreads - 1) / kThreads));
    float* d_bb = nullptr;
    MLODS_CUDA(cudaMalloc(&d_bb, size_t(nbb) * 6 * sizeof(float) + sizeof(int)));
    int* d_bad = reinterpret_cast<int*>(d_bb + size_t(nbb) * 6);
    std::vector<float> hbb(size_t(nbb) * 6);
    int h_bad = 0;
    cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        bbox_kernel<<<nbb, kThreads, 0, s>>>(d_pts, n, d_bb, d_bad);
        note_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hbb.data(), d_bb, hbb.size() * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_bb);
    if (e != cudaSuccess) return cuda_fail(e, "tree build: bbox", __FILE__, __LINE__);
    if (h_bad) {
        set_last_error("tree build: non-finite point coordinates");
        return MLODS_ERR_INVALID;
    }
    for (int a = 0; a < 3; ++a) {
        T->bb[a] = INFINITY;
        T->BB[a] = -INFINITY;
    }
    for (int b = 0; b < nbb; ++b)
        for (int a = 0; a < 3; ++a) {
            T->bb[a] = std::min(T->bb[a], hbb[6 * b + a]);
            T->BB[a] = std::max(T->BB[a], hbb[6 * b + 3 + a]);
        }
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(T->bb[a]) || !std::isfinite(T->BB[a])) {
            set_last_error("tree build: non-finite point coordinates");
            return MLODS_ERR_INVALID;
        }
        T->origin[a] = (double(T->bb[a]) + double(T->BB[a])) / 2.0;
    }
    {
        const float dx = T->BB[0] - T->bb[0], dy = T->BB[1] - T->bb[1], dz = T->BB[2] - T->bb[2];
        volatile float xx = dx * dx, yy = dy * dy, zz = dz * dz;
        volatile float s2 = xx + yy;
        const float d2 = s2 + zz;
        T->root_radius = std::sqrt(d2) / 2.f;
    }

    // ---- per-axis split and bound tables (the reference recursion, per axis)
    const int64_t split_stride = (int64_t(1) << D) - 1 > 0 ? (int64_t(1) << D) - 1 : 1;
    const int64_t bound_stride = (int64_t(1) << (D + 1)) + D;
    std::vector<double> hs(size_t(3 * split_stride), 0.0);
    std::vector<float> hb(size_t(3 * bound_stride), 0.f);
    for (int a = 0; a < 3; ++a) {
        float* B = hb.data() + a * bound_stride;
        double* S = hs.data() + a * split_stride;
        B[0] = T->bb[a];
        B[1] = T->BB[a];
        for (int d = 0; d < D; ++d) {
            const int64_t bo = ((int64_t(1) << d) - 1) + d, bn = ((int64_t(1) << (d + 1)) - 1) + d + 1;
            const int64_t so = (int64_t(1) << d) - 1;
            const int64_t w = int64_t(1) << d;
            for (int64_t k = 0; k < w; ++k) {
                // `(bb[0] + BB[0]) / 2.0` with float bounds (CPUUtils.cpp:286-288):
                // the sum rounds to float before the division in double, so
                // the split is itself a float value
                const float bsum = B[bo + k] + B[bo + k + 1];
                const double sp = double(bsum) / 2.0;
                S[so + k] = sp;
                B[bn + 2 * k] = B[bo + k];
                B[bn + 2 * k + 1] = float(sp);
            }
            B[bn + 2 * w] = B[bo + w];
        }
    }

    // ---- temporaries
    const int64_t nb = (n + kTile - 1) / kTile;
    const int64_t ncounts = nb * kLevels;
    Bump bump;
    {
        size_t need = 0;
        need += al(size_t(3 * split_stride) * 8);
        need += 2 * al(size_t(n) * 8) + 2 * al(size_t(n) * 4);
        need += al(size_t(n)) * 3;  // tie, lcp, leafd
        need += al(size_t(ncounts) * 4) + al(64 * 8);
        need += std::max(radix_temp_bytes(n), scan_temp_bytes(ncounts));
        bump.cap = need;
        MLODS_CUDA(cudaMalloc(&bump.base, need));
    }
    double* d_splits = bump.take<double>(size_t(3 * split_stride));
    uint64_t* d_k0 = bump.take<uint64_t>(size_t(n));
    uint64_t* d_k1 = bump.take<uint64_t>(size_t(n));
    uint32_t* d_v0 = bump.take<uint32_t>(size_t(n));
    uint32_t* d_v1 = bump.take<uint32_t>(size_t(n));
    uint8_t* d_tie = bump.take<uint8_t>(size_t(n));
    int8_t* d_lcp = bump.take<int8_t>(size_t(n));
    int8_t* d_leafd = bump.take<int8_t>(size_t(n));
    uint32_t* d_counts = bump.take<uint32_t>(size_t(ncounts));
    int64_t* d_misc = bump.take<int64_t>(64);
    void* d_tmp = bump.base + bump.off;

    auto fail = [&](cudaError_t err, const char* what) {
        cudaFree(bump.base);
        return cuda_fail(err, what, __FILE__, __LINE__);
    };
#define BUILD_CHECK(call, what)                          \
    do {                                                 \
        cudaError_t _e2 = (call);                        \
        if (_e2 != cudaSuccess) return fail(_e2, what);  \
    } while (0)

    BUILD_CHECK(cudaMalloc(&T->d_bounds, size_t(3 * bound_stride) * sizeof(float)), "alloc bounds");
    T->bounds_stride = bound_stride;
    BUILD_CHECK(cudaMemcpyAsync(T->d_bounds, hb.data(), hb.size() * sizeof(float), cudaMemcpyHostToDevice, s),
                "upload bounds");
    BUILD_CHECK(cudaMemcpyAsync(d_splits, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, s),
                "upload splits");
    BUILD_CHECK(cudaMemsetAsync(d_misc, 0, 64 * 8, s), "memset misc");

    // ---- Morton codes and sort
    morton_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(d_pts, n, D, d_splits, split_stride, d_k0, d_v0, d_tie);
    note_launch();
    BUILD_CHECK(cudaGetLastError(), "morton");
    bool in_alt = false;
    BUILD_CHECK(radix_sort_pairs_u64(d_k0, d_v0, d_k1, d_v1, n, 3 * D, &in_alt, d_tmp, s), "radix sort");
    uint64_t* codes = in_alt ? d_k1 : d_k0;
    uint32_t* perm = in_alt ? d_v1 : d_v0;

    lcp_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(codes, n, D, d_lcp, d_leafd);

    note_launch();
    BUILD_CHECK(cudaGetLastError(), "lcp");

    // ---- per-level node counts -> breadth-first bases
    level_count_kernel<<<unsigned(nb), kThreads, 0, s>>>(d_lcp, d_leafd, n, D, int(nb), d_counts);
    note_launch();
    BUILD_CHECK(cudaGetLastError(), "level count");
    const int64_t nlev = int64_t(D + 1) * nb;
    uint32_t* d_total = reinterpret_cast<uint32_t*>(d_misc);
    BUILD_CHECK(exclusive_scan_u32(d_counts, d_counts, nlev, d_total, d_tmp, s), "level scan");
    std::vector<uint32_t> lvl_first(size_t(D + 2), 0);
    uint32_t h_total = 0;
    BUILD_CHECK(cudaMemcpyAsync(&h_total, d_total, 4, cudaMemcpyDeviceToHost, s), "read total");
    for (int d = 0; d <= D; ++d)
        BUILD_CHECK(cudaMemcpyAsync(&lvl_first[d], d_counts + int64_t(d) * nb, 4, cudaMemcpyDeviceToHost, s),
                    "read level offsets");
    BUILD_CHECK(cudaStreamSynchronize(s), "sync level offsets");
    const int64_t nn = int64_t(h_total);
    lvl_first[D + 1] = h_total;
    T->n_nodes = nn;
    int depth = 0;
    for (int d = 0; d <= D; ++d)
        if (lvl_first[d + 1] > lvl_first[d]) depth = d;
    T->depth = depth;

    // ---- node arrays
    char* nodebuf = nullptr;
    size_t nodebytes = al(size_t(nn) * 4) * 6 + al(size_t(nn)) * 2 + al(size_t(nn) * 72) + al(size_t(D + 2) * 8) +
                       scan_temp_bytes(nn) + 256;
    BUILD_CHECK(cudaMalloc(&nodebuf, nodebytes), "alloc node temporaries");
    Bump nbm;
    nbm.base = nodebuf;
    nbm.cap = nodebytes;
    int32_t* d_head = nbm.take<int32_t>(size_t(nn));
    int32_t* d_parent = nbm.take<int32_t>(size_t(nn));
    int32_t* d_first = nbm.take<int32_t>(size_t(nn));
    int32_t* d_nchild = nbm.take<int32_t>(size_t(nn));
    int32_t* d_lcnt = nbm.take<int32_t>(size_t(nn));
    uint32_t* d_xoff = nbm.take<uint32_t>(size_t(nn));
    uint8_t* d_level = nbm.take<uint8_t>(size_t(nn));
    uint8_t* d_isfirst = nbm.take<uint8_t>(size_t(nn));
    double* d_mom = nbm.take<double>(size_t(nn) * 9);
    int64_t* d_lvloff = nbm.take<int64_t>(size_t(D + 2));
    void* d_ntmp = nbm.base + nbm.off;
    auto fail2 = [&](cudaError_t err, const char* what) {
        cudaFree(nodebuf);
        return fail(err, what);
    };
#define NODE_CHECK(call, what)                            \
    do {                                                  \
        cudaError_t _e3 = (call);                         \
        if (_e3 != cudaSuccess) return fail2(_e3, what);  \
    } while (0)

    {
        std::vector<int64_t> lo64(size_t(D + 2));
        for (int d = 0; d <= D + 1; ++d) lo64[d] = lvl_first[d];
        NODE_CHECK(cudaMemcpyAsync(d_lvloff, lo64.data(), lo64.size() * 8, cudaMemcpyHostToDevice, s), "lvl off");
        NODE_CHECK(cudaStreamSynchronize(s), "sync lvl off");
    }
    NODE_CHECK(cudaMemsetAsync(d_first, 0xFF, size_t(nn) * 4, s), "memset first");
    NODE_CHECK(cudaMemsetAsync(d_nchild, 0, size_t(nn) * 4, s), "memset nchild");
    level_emit_kernel<<<unsigned(nb), kThreads, 0, s>>>(d_lcp, d_leafd, n, D, int(nb), d_counts, d_head, d_level,
                                                         d_isfirst, d_parent, d_first);
    note_launch();
    NODE_CHECK(cudaGetLastError(), "emit");
    links_kernel<<<grid_for(nn, kThreads), kThreads, 0, s>>>(nn, d_level, d_isfirst, d_lvloff, d_parent, d_nchild);
    note_launch();
    NODE_CHECK(cudaGetLastError(), "links");

    MLODS_CUDA(cudaMalloc(&T->d_area, size_t(n) * sizeof(float)));
    unsigned long long* d_ties = reinterpret_cast<unsigned long long*>(d_misc + 1);
    leaf_kernel<<<grid_for(nn, kThreads), kThreads, 0, s>>>(nn, n, D, d_level, d_head, d_first, d_lcp, d_leafd,
                                                            codes, perm, T->d_bounds, bound_stride, d_lcnt,
                                                            T->d_area, d_tie, d_ties);
    note_launch();
    NODE_CHECK(cudaGetLastError(), "leaf");
    for (int d = D; d >= 0; --d) {
        const int64_t lo = lvl_first[d], hi = lvl_first[d + 1];
        if (hi <= lo) continue;
        moments_kernel<<<grid_for(hi - lo, 128), 128, 0, s>>>(lo, hi, d_head, d_first, d_nchild, d_lcnt, perm, d_pts,
                                                               d_nrm, T->d_area, T->origin[0], T->origin[1],
                                                               T->origin[2], d_mom);
        note_launch();
        NODE_CHECK(cudaGetLastError(), "moments");
    }
    multi_count_kernel<<<grid_for(nn, kThreads), kThreads, 0, s>>>(nn, d_lcnt, d_xoff);
    note_launch();
    NODE_CHECK(cudaGetLastError(), "multi count");
    uint32_t* d_xtotal = reinterpret_cast<uint32_t*>(d_misc + 2);
    NODE_CHECK(exclusive_scan_u32(d_xoff, d_xoff, nn, d_xtotal, d_ntmp, s), "multi scan");
    uint32_t h_extra = 0;
    unsigned long long h_ties = 0;
    NODE_CHECK(cudaMemcpyAsync(&h_extra, d_xtotal, 4, cudaMemcpyDeviceToHost, s), "read extra");
    NODE_CHECK(cudaMemcpyAsync(&h_ties, d_ties, 8, cudaMemcpyDeviceToHost, s), "read ties");
    NODE_CHECK(cudaStreamSynchronize(s), "sync extra");
    T->n_extra = h_extra;
    T->n_ties = int64_t(h_ties);

    {
        const size_t rec = size_t(nn + h_extra);
        float4* base = nullptr;
        NODE_CHECK(cudaMalloc(&base, rec * 4 * sizeof(float4)), "alloc nodes");
        T->nodes.geom = base;
        T->nodes.pm = base + rec;
        T->nodes.nc = base + 2 * rec;
        T->nodes.aux = base + 3 * rec;
    }
    write_nodes_kernel<<<grid_for(nn, kThreads), kThreads, 0, s>>>(nn, D, d_level, d_head, d_parent, d_first, d_nchild,
                                                                   d_lcnt, d_xoff, codes, perm, T->d_bounds,
                                                                   bound_stride, d_mom, T->origin[0], T->origin[1],
                                                                   T->origin[2], T->nodes);
    note_launch();
    NODE_CHECK(cudaGetLastError(), "write nodes");
    if (h_extra > 0) {
        write_point_records_kernel<<<grid_for(nn, kThreads), kThreads, 0, s>>>(
            nn, d_head, d_lcnt, d_xoff, d_level, perm, d_pts, d_nrm, T->d_area, T->origin[0], T->origin[1],
            T->origin[2], T->nodes);
        note_launch();
        NODE_CHECK(cudaGetLastError(), "write point records");
    }

    // ---- kept for export, DC and neighbour gathers
    NODE_CHECK(cudaMalloc(&T->d_node_head, size_t(nn) * 4), "alloc head");
    NODE_CHECK(cudaMemcpyAsync(T->d_node_head, d_head, size_t(nn) * 4, cudaMemcpyDeviceToDevice, s), "copy head");
    NODE_CHECK(cudaMalloc(&T->d_codes, size_t(n) * 8), "alloc codes");
    NODE_CHECK(cudaMemcpyAsync(T->d_codes, codes, size_t(n) * 8, cudaMemcpyDeviceToDevice, s), "copy codes");
    NODE_CHECK(cudaMalloc(&T->d_perm, size_t(n) * 4), "alloc perm");
    NODE_CHECK(cudaMemcpyAsync(T->d_perm, perm, size_t(n) * 4, cudaMemcpyDeviceToDevice, s), "copy perm");
    NODE_CHECK(cudaMalloc(&T->d_spts, size_t(n) * sizeof(float4)), "alloc spts");
    NODE_CHECK(cudaMalloc(&T->d_snrm, size_t(n) * sizeof(float4)), "alloc snrm");
    NODE_CHECK(cudaMalloc(&T->d_wspts, size_t(n) * sizeof(float4)), "alloc wspts");
    sorted_points_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, perm, d_pts, d_nrm, T->origin[0], T->origin[1],
                                                                    T->origin[2], T->d_spts, T->d_snrm, T->d_wspts);
    note_launch();
    NODE_CHECK(cudaGetLastError(), "sorted points");
    NODE_CHECK(cudaStreamSynchronize(s), "sync build");
    {
        float4 root_pm;  // {pbar, m0} of the root: the total sample area
        NODE_CHECK(cudaMemcpy(&root_pm, T->nodes.pm, sizeof root_pm, cudaMemcpyDeviceToHost), "root mass");
        T->root_mass = root_pm.w;
    }
    cudaFree(nodebuf);
    cudaFree(bump.base);
#undef NODE_CHECK
#undef BUILD_CHECK
    T->device_bytes = int64_t((nn + h_extra) * 4 * sizeof(float4)) + nn * 4 + n * (8 + 4 + 4 + 48) +
                      3 * bound_stride * 4;
    return MLODS_OK;
}

namespace
{
__global__ void export_kernel(int64_t nn, int D, NodeArrays nodes, const int32_t* __restrict__ head,
                              const uint64_t* __restrict__ codes, const float* __restrict__ bounds, int64_t stride,
                              double o0, double o1, double o2, int32_t* depth, int32_t* parent, int32_t* first_child,
                              int32_t* n_children, int32_t* next_brother, int32_t* leaf_cnt, float* bmin, float* bmax,
                              double* mom)
{
    int64_t id = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= nn) return;
    const DNode nd = load_node_all(nodes, id);
    const int d = node_depth(nd.info);
    const bool leaf = (nd.info & kLeafBit) != 0;
    depth[id] = d;
    parent[id] = nd.parent == 0xFFFFFFFFu ? -1 : int32_t(nd.parent);
    first_child[id] = leaf ? -1 : int32_t(nd.first);
    n_children[id] = leaf ? 0 : int32_t(node_count(nd.info));
    leaf_cnt[id] = leaf ? int32_t(node_count(nd.info)) : 0;
    int32_t nb = -1;
    if (id + 1 < nn && nd.parent != 0xFFFFFFFFu && __float_as_uint(nodes.aux[id + 1].w) == nd.parent)
        nb = int32_t(id + 1);
    next_brother[id] = nb;
    float bb[3], BB[3];
    node_box(bounds, stride, codes[head[id]], D, d, bb, BB);
    for (int a = 0; a < 3; ++a) {
        bmin[3 * id + a] = bb[a];
        bmax[3 * id + a] = BB[a];
    }
    double* m = mom + 9 * id;
    m[0] = nd.m0;
    m[1] = double(nd.px) + o0;
    m[2] = double(nd.py) + o1;
    m[3] = double(nd.pz) + o2;
    m[4] = nd.nx;
    m[5] = nd.ny;
    m[6] = nd.nz;
    m[7] = nd.cpn;
    m[8] = nd.cpp;
}
}  // namespace

int export_tree(mlods_tree_s* T, int32_t* depth, int32_t* parent, int32_t* first_child, int32_t* n_children,
                int32_t* next_brother, int32_t* leaf_off, int32_t* leaf_cnt, int32_t* perm_out, float* bmin,
                float* bmax, double* mom, float* area)
{
    const int64_t nn = T->n_nodes, n = T->n_pts;
    std::vector<int32_t> v_depth(nn), v_parent(nn), v_first(nn), v_nc(nn), v_nb(nn), v_lc(nn);
    std::vector<float> v_bmin(nn * 3), v_bmax(nn * 3);
    std::vector<double> v_mom(nn * 9);
    char* buf = nullptr;
    const size_t bytes = size_t(nn) * (6 * 4 + 6 * 4 + 9 * 8);
    MLODS_CUDA(cudaMalloc(&buf, bytes));
    int32_t* d_depth = reinterpret_cast<int32_t*>(buf);
    int32_t* d_parent = d_depth + nn;
    int32_t* d_first = d_parent + nn;
    int32_t* d_nc = d_first + nn;
    int32_t* d_nb = d_nc + nn;
    int32_t* d_lc = d_nb + nn;
    float* d_bmin = reinterpret_cast<float*>(d_lc + nn);
    float* d_bmax = d_bmin + 3 * nn;
    double* d_mom = reinterpret_cast<double*>(d_bmax + 3 * nn);
    export_kernel<<<grid_for(nn, kThreads), kThreads>>>(nn, T->max_depth, T->nodes, T->d_node_head, T->d_codes,
                                                        T->d_bounds, T->bounds_stride, T->origin[0], T->origin[1],
                                                        T->origin[2], d_depth, d_parent, d_first, d_nc, d_nb, d_lc,
                                                        d_bmin, d_bmax, d_mom);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(v_depth.data(), d_depth, nn * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_parent.data(), d_parent, nn * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_first.data(), d_first, nn * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_nc.data(), d_nc, nn * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_nb.data(), d_nb, nn * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_lc.data(), d_lc, nn * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_bmin.data(), d_bmin, nn * 12, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_bmax.data(), d_bmax, nn * 12, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_mom.data(), d_mom, nn * 72, cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(e, "export", __FILE__, __LINE__);
    // leaf point lists: single-point leaves hold the point index in `first`,
    // multi-point leaves point at their point records.
    // aux = {cpp, first, info, parent}
    std::vector<float4> hx(size_t(nn + T->n_extra));
    MLODS_CUDA(cudaMemcpy(hx.data(), T->nodes.aux, hx.size() * sizeof(float4), cudaMemcpyDeviceToHost));
    auto first_of = [&](int64_t i) { uint32_t v; std::memcpy(&v, &hx[i].y, 4); return v; };
    auto info_of = [&](int64_t i) { uint32_t v; std::memcpy(&v, &hx[i].z, 4); return v; };
    if (perm_out || leaf_off) {
        int32_t pos = 0;
        for (int64_t id = 0; id < nn; ++id) {
            if (!(info_of(id) & kLeafBit)) {
                if (leaf_off) leaf_off[id] = -1;
                continue;
            }
            if (leaf_off) leaf_off[id] = pos;
            const int cnt = int(node_count(info_of(id)));
            if (cnt == 1) {
                if (perm_out) perm_out[pos] = int32_t(first_of(id));
                ++pos;
            } else {
                for (int k = 0; k < cnt; ++k) {
                    if (perm_out) perm_out[pos] = int32_t(first_of(first_of(id) + k));
                    ++pos;
                }
            }
        }
    }
    if (depth) std::memcpy(depth, v_depth.data(), nn * 4);
    if (parent) std::memcpy(parent, v_parent.data(), nn * 4);
    if (first_child) std::memcpy(first_child, v_first.data(), nn * 4);
    if (n_children) std::memcpy(n_children, v_nc.data(), nn * 4);
    if (next_brother) std::memcpy(next_brother, v_nb.data(), nn * 4);
    if (leaf_cnt) std::memcpy(leaf_cnt, v_lc.data(), nn * 4);
    if (bmin) std::memcpy(bmin, v_bmin.data(), nn * 12);
    if (bmax) std::memcpy(bmax, v_bmax.data(), nn * 12);
    if (mom) std::memcpy(mom, v_mom.data(), nn * 72);
    if (area) MLODS_CUDA(cudaMemcpy(area, T->d_area, size_t(n) * 4, cudaMemcpyDeviceToHost));
    return MLODS_OK;
}

}  // namespace mlods
