// mesh_dev.cu -- the dual-contouring refinement loop on the device.
//
// scene::computeDualContouring (scene.cpp:1402-1452) projects the extracted
// vertices, then twice smooths, 1->4 subdivides and projects again.  The
// reference runs smoothing and subdivision on the host (mesh::smoothMesh,
// mesh::subdivideMesh, upsample.h:55-133) and copies the vertices to the GPU
// and back around every projection.  Here the mesh stays in device memory
// for the whole loop and both edits are kernels that give the reference's
// results exactly:
//   * smoothing sums every vertex's neighbour contributions in triangle
//     order (a stable radix sort of the (vertex, 3t + slot) pairs, then one
//     thread per vertex adds its run sequentially in float), then divides by
//     the valence;
//   * subdivision numbers the edge midpoints in order of first sight, as the
//     reference's std::map lookups do: the (edge, 3t + slot) pairs are
//     stable-sorted by edge, the first occurrence of each edge is flagged at
//     its position and a scan of those flags gives the new vertex numbers.
#include <algorithm>
#include <new>
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
inline size_t al256(size_t v) { return (v + 255) / 256 * 256; }

// ---- smoothing

__global__ void smooth_pairs_kernel(const uint32_t* __restrict__ tri, int64_t nt, uint64_t* __restrict__ key,
                                    uint32_t* __restrict__ val)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= 3 * nt) return;
    key[i] = tri[i];
    val[i] = uint32_t(i);
}

// first index of v in the sorted vertex keys
__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t* k, int64_t n, uint64_t v)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if (k[m] < v) lo = m + 1;
        else hi = m;
    }
    return lo;
}

__global__ void smooth_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ slot, int64_t n_pairs,
                              const uint32_t* __restrict__ tri, const float* __restrict__ p, int64_t nv,
                              float* __restrict__ out)
{
    const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    int64_t i = lower_bound_u64(key, n_pairs, uint64_t(v));
    float acc[3] = {0.f, 0.f, 0.f};
    float val = 0.f;
    for (; i < n_pairs && key[i] == uint64_t(v); ++i) {
        const uint32_t e = slot[i];
        const uint32_t t = e / 3u, j = e - 3u * t;
        const uint32_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
        // newPos[a] += p[b] + p[c]; newPos[b] += p[a] + p[c]; newPos[c] += p[b] + p[a]
        const uint32_t u = j == 0 ? b : (j == 1 ? a : b);
        const uint32_t w = j == 0 ? c : (j == 1 ? c : a);
        for (int k = 0; k < 3; ++k) acc[k] = __fadd_rn(acc[k], __fadd_rn(p[3 * u + k], p[3 * w + k]));
        val = __fadd_rn(val, 2.f);
    }
    for (int k = 0; k < 3; ++k) out[3 * v + k] = __fdiv_rn(acc[k], val);
}

// ---- subdivision

// edges of triangle t in the reference's lookup order: ab, (c, b), (c, a)
__global__ void edge_pairs_kernel(const uint32_t* __restrict__ tri, int64_t nt, uint64_t* __restrict__ key,
                                  uint32_t* __restrict__ val)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= 3 * nt) return;
    const int64_t t = i / 3;
    const int j = int(i - 3 * t);
    const uint32_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
    const uint32_t u = j == 0 ? a : c;
    const uint32_t w = j == 0 ? b : (j == 1 ? b : a);
    key[i] = (uint64_t(min(u, w)) << 32) | uint64_t(max(u, w));
    val[i] = uint32_t(i);
}

// first occurrence of every edge, flagged at its position 3t + slot
__global__ void first_flags_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ pos, int64_t n,
                                   uint32_t* __restrict__ first)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    first[pos[i]] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

// every occurrence gets the number of its edge's first occurrence
__global__ void edge_ids_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ pos, int64_t n,
                                const uint32_t* __restrict__ rank, uint32_t base, uint32_t* __restrict__ id_at)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t h = i;
    while (h > 0 && key[h - 1] == key[i]) --h;  // runs are short: an edge has 1-2 (rarely more) triangles
    id_at[pos[i]] = base + rank[pos[h]];
}

__global__ void midpoints_kernel(const uint32_t* __restrict__ tri, int64_t nt, const uint32_t* __restrict__ first,
                                 const uint32_t* __restrict__ id_at, float* __restrict__ p, float* __restrict__ nrm)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= 3 * nt || !first[i]) return;
    const int64_t t = i / 3;
    const int j = int(i - 3 * t);
    const uint32_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
    const uint32_t u = j == 0 ? a : c;
    const uint32_t w = j == 0 ? b : (j == 1 ? b : a);
    const uint32_t id = id_at[i];
    for (int k = 0; k < 3; ++k) {
        p[3 * size_t(id) + k] = __fdiv_rn(__fadd_rn(p[3 * u + k], p[3 * w + k]), 2.f);
        nrm[3 * size_t(id) + k] = 0.f;  // normals.resize: new vertices get (0, 0, 0)
    }
}

__global__ void split_kernel(uint32_t* __restrict__ tri, int64_t nt, const uint32_t* __restrict__ id_at)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const uint32_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
    const uint32_t ab = id_at[3 * t], bc = id_at[3 * t + 1], ca = id_at[3 * t + 2];
    tri[3 * t] = a;
    tri[3 * t + 1] = ab;
    tri[3 * t + 2] = ca;
    uint32_t* o = tri + 3 * nt + 9 * t;
    o[0] = ab;
    o[1] = b;
    o[2] = bc;
    o[3] = ab;
    o[4] = bc;
    o[5] = ca;
    o[6] = ca;
    o[7] = bc;
    o[8] = c;
}

__global__ void xform_kernel(float* __restrict__ p, int64_t nv, const float* __restrict__ m)
{
    const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const float x = p[3 * v], y = p[3 * v + 1], z = p[3 * v + 2];
    for (int r = 0; r < 3; ++r) {
        float a = __fmul_rn(m[4 * r], x);
        a = __fadd_rn(a, __fmul_rn(m[4 * r + 1], y));
        a = __fadd_rn(a, __fmul_rn(m[4 * r + 2], z));
        p[3 * v + r] = __fadd_rn(a, m[4 * r + 3]);
    }
}

struct Buf {
    void* p = nullptr;
    size_t cap = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() { cudaFree(p); }
    void swap(Buf& o)
    {
        std::swap(p, o.p);
        std::swap(cap, o.cap);
    }
    int need(size_t bytes)
    {
        if (bytes <= cap) return MLODS_OK;
        cudaFree(p);
        p = nullptr;
        cap = 0;
        MLODS_CUDA(cudaMalloc(&p, bytes));
        cap = bytes;
        return MLODS_OK;
    }
};

}  // namespace

struct DeviceMesh {
    Buf pos, nrm, tri;  // float3, float3, uint3
    Buf k0, k1, v0, v1, first, rank, id_at, tmp, total;
    int64_t nv = 0, nt = 0;
};

DeviceMesh* dmesh_create() { return new (std::nothrow) DeviceMesh(); }

int dmesh_reserve(DeviceMesh& m, int64_t nv, int64_t nt)
{
    int rc = m.pos.need(size_t(std::max<int64_t>(nv, 1)) * 12);
    if (rc == MLODS_OK) rc = m.nrm.need(size_t(std::max<int64_t>(nv, 1)) * 12);
    if (rc == MLODS_OK) rc = m.tri.need(size_t(std::max<int64_t>(nt, 1)) * 12);
    if (rc != MLODS_OK) return rc;
    m.nv = nv;
    m.nt = nt;
    return MLODS_OK;
}
float* dmesh_pos(DeviceMesh& m) { return static_cast<float*>(m.pos.p); }
float* dmesh_nrm(DeviceMesh& m) { return static_cast<float*>(m.nrm.p); }
uint32_t* dmesh_tri(DeviceMesh& m) { return static_cast<uint32_t*>(m.tri.p); }
void dmesh_destroy(DeviceMesh* m) { delete m; }
int64_t dmesh_nv(const DeviceMesh& m) { return m.nv; }
int64_t dmesh_nt(const DeviceMesh& m) { return m.nt; }

int dmesh_get(const DeviceMesh& m, float* pos, float* nrm, uint32_t* tri, cudaStream_t s)
{
    if (m.nv && pos) MLODS_CUDA(cudaMemcpyAsync(pos, m.pos.p, size_t(m.nv) * 12, cudaMemcpyDeviceToHost, s));
    if (m.nv && nrm) MLODS_CUDA(cudaMemcpyAsync(nrm, m.nrm.p, size_t(m.nv) * 12, cudaMemcpyDeviceToHost, s));
    if (m.nt && tri) MLODS_CUDA(cudaMemcpyAsync(tri, m.tri.p, size_t(m.nt) * 12, cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    return MLODS_OK;
}

int dmesh_upload(DeviceMesh& m, const float* pos, int64_t nv, const uint32_t* tri, int64_t nt, cudaStream_t s)
{
    int rc = m.pos.need(size_t(nv) * 12);
    if (rc == MLODS_OK) rc = m.nrm.need(size_t(nv) * 12);
    if (rc == MLODS_OK) rc = m.tri.need(size_t(nt) * 12);
    if (rc != MLODS_OK) return rc;
    if (nv) MLODS_CUDA(cudaMemcpyAsync(m.pos.p, pos, size_t(nv) * 12, cudaMemcpyHostToDevice, s));
    if (nv) MLODS_CUDA(cudaMemsetAsync(m.nrm.p, 0, size_t(nv) * 12, s));
    if (nt) MLODS_CUDA(cudaMemcpyAsync(m.tri.p, tri, size_t(nt) * 12, cudaMemcpyHostToDevice, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    m.nv = nv;
    m.nt = nt;
    return MLODS_OK;
}

int dmesh_download(const DeviceMesh& m, std::vector<float>& pos, std::vector<float>& nrm, std::vector<uint32_t>& tri,
                   cudaStream_t s)
{
    pos.resize(size_t(m.nv) * 3);
    nrm.resize(size_t(m.nv) * 3);
    tri.resize(size_t(m.nt) * 3);
    if (m.nv) MLODS_CUDA(cudaMemcpyAsync(pos.data(), m.pos.p, size_t(m.nv) * 12, cudaMemcpyDeviceToHost, s));
    if (m.nv) MLODS_CUDA(cudaMemcpyAsync(nrm.data(), m.nrm.p, size_t(m.nv) * 12, cudaMemcpyDeviceToHost, s));
    if (m.nt) MLODS_CUDA(cudaMemcpyAsync(tri.data(), m.tri.p, size_t(m.nt) * 12, cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    return MLODS_OK;
}

int dmesh_transform(DeviceMesh& m, const float* xform, cudaStream_t s)
{
    if (m.nv == 0) return MLODS_OK;
    int rc = m.tmp.need(256);
    if (rc != MLODS_OK) return rc;
    MLODS_CUDA(cudaMemcpyAsync(m.tmp.p, xform, 12 * sizeof(float), cudaMemcpyHostToDevice, s));
    xform_kernel<<<blocks_for(m.nv), kThreads, 0, s>>>(static_cast<float*>(m.pos.p), m.nv,
                                                        static_cast<const float*>(m.tmp.p));
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    MLODS_CUDA(cudaStreamSynchronize(s));  // the xform staging buffer is reused
    return MLODS_OK;
}

int dmesh_project(mlods_tree_s* T, DeviceMesh& m, int iters, cudaStream_t s)
{
    if (m.nv == 0) return MLODS_OK;
    float* p = static_cast<float*>(m.pos.p);
    return project_buffers(T, m.nv, p, p, static_cast<float*>(m.nrm.p), iters, -1.f, s);
}

static int sort_pairs(DeviceMesh& m, int64_t n, int nbits, uint64_t** keys, uint32_t** vals, cudaStream_t s)
{
    bool alt = false;
    MLODS_CUDA(radix_sort_pairs_u64(static_cast<uint64_t*>(m.k0.p), static_cast<uint32_t*>(m.v0.p),
                                    static_cast<uint64_t*>(m.k1.p), static_cast<uint32_t*>(m.v1.p), n, nbits, &alt,
                                    m.tmp.p, s));
    *keys = static_cast<uint64_t*>(alt ? m.k1.p : m.k0.p);
    *vals = static_cast<uint32_t*>(alt ? m.v1.p : m.v0.p);
    return MLODS_OK;
}

static int reserve_pairs(DeviceMesh& m, int64_t n)
{
    int rc = m.k0.need(size_t(n) * 8);
    if (rc == MLODS_OK) rc = m.k1.need(size_t(n) * 8);
    if (rc == MLODS_OK) rc = m.v0.need(size_t(n) * 4);
    if (rc == MLODS_OK) rc = m.v1.need(size_t(n) * 4);
    if (rc == MLODS_OK) rc = m.tmp.need(std::max(radix_temp_bytes(n), scan_temp_bytes(n)));
    return rc;
}

static int bits_for(uint64_t v)
{
    int b = 1;
    while (b < 64 && (uint64_t(1) << b) <= v) ++b;
    return b;
}

// mesh::smoothMesh
int dmesh_smooth(DeviceMesh& m, cudaStream_t s)
{
    const int64_t n = 3 * m.nt;
    if (m.nv == 0) return MLODS_OK;
    int rc = reserve_pairs(m, std::max<int64_t>(n, 1));
    Buf out;
    if (rc == MLODS_OK) rc = out.need(size_t(m.nv) * 12);
    if (rc != MLODS_OK) return rc;
    uint64_t* keys = nullptr;
    uint32_t* vals = nullptr;
    if (n > 0) {
        smooth_pairs_kernel<<<blocks_for(n), kThreads, 0, s>>>(static_cast<const uint32_t*>(m.tri.p), m.nt,
                                                              static_cast<uint64_t*>(m.k0.p),
                                                              static_cast<uint32_t*>(m.v0.p));
        note_launch();
        MLODS_CUDA(cudaGetLastError());
        rc = sort_pairs(m, n, bits_for(uint64_t(m.nv)), &keys, &vals, s);
        if (rc != MLODS_OK) return rc;
    }
    smooth_kernel<<<blocks_for(m.nv), kThreads, 0, s>>>(keys, vals, n, static_cast<const uint32_t*>(m.tri.p),
                                                       static_cast<const float*>(m.pos.p), m.nv,
                                                       static_cast<float*>(out.p));
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    MLODS_CUDA(cudaMemcpyAsync(m.pos.p, out.p, size_t(m.nv) * 12, cudaMemcpyDeviceToDevice, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    return MLODS_OK;
}

// mesh::subdivideMesh
int dmesh_subdivide(DeviceMesh& m, cudaStream_t s)
{
    const int64_t n = 3 * m.nt;
    if (n == 0) return MLODS_OK;
    int rc = reserve_pairs(m, n);
    if (rc == MLODS_OK) rc = m.first.need(size_t(n) * 4);
    if (rc == MLODS_OK) rc = m.rank.need(size_t(n) * 4);
    if (rc == MLODS_OK) rc = m.id_at.need(size_t(n) * 4);
    if (rc == MLODS_OK) rc = m.total.need(256);
    if (rc != MLODS_OK) return rc;
    const uint32_t* tri = static_cast<const uint32_t*>(m.tri.p);
    edge_pairs_kernel<<<blocks_for(n), kThreads, 0, s>>>(tri, m.nt, static_cast<uint64_t*>(m.k0.p),
                                                        static_cast<uint32_t*>(m.v0.p));
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    uint64_t* keys = nullptr;
    uint32_t* pos = nullptr;
    rc = sort_pairs(m, n, 32 + bits_for(uint64_t(m.nv)), &keys, &pos, s);
    if (rc != MLODS_OK) return rc;
    uint32_t* first = static_cast<uint32_t*>(m.first.p);
    first_flags_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, pos, n, first);
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    uint32_t* d_total = static_cast<uint32_t*>(m.total.p);
    MLODS_CUDA(exclusive_scan_u32(first, static_cast<uint32_t*>(m.rank.p), n, d_total, m.tmp.p, s));
    uint32_t n_new = 0;
    MLODS_CUDA(cudaMemcpyAsync(&n_new, d_total, 4, cudaMemcpyDeviceToHost, s));
    MLODS_CUDA(cudaStreamSynchronize(s));
    const int64_t nv2 = m.nv + int64_t(n_new), nt2 = 4 * m.nt;
    if (nv2 > int64_t(UINT32_MAX)) {
        set_last_error("mesh subdivide: result would exceed 32-bit vertex indices");
        return MLODS_ERR_CAPACITY;
    }
    edge_ids_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, pos, n, static_cast<const uint32_t*>(m.rank.p),
                                                      uint32_t(m.nv), static_cast<uint32_t*>(m.id_at.p));
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    // grow the vertex and triangle arrays, keeping their contents
    Buf pos2, nrm2, tri2;
    rc = pos2.need(size_t(nv2) * 12);
    if (rc == MLODS_OK) rc = nrm2.need(size_t(nv2) * 12);
    if (rc == MLODS_OK) rc = tri2.need(size_t(nt2) * 12);
    if (rc != MLODS_OK) return rc;
    MLODS_CUDA(cudaMemcpyAsync(pos2.p, m.pos.p, size_t(m.nv) * 12, cudaMemcpyDeviceToDevice, s));
    MLODS_CUDA(cudaMemcpyAsync(nrm2.p, m.nrm.p, size_t(m.nv) * 12, cudaMemcpyDeviceToDevice, s));
    MLODS_CUDA(cudaMemcpyAsync(tri2.p, m.tri.p, size_t(m.nt) * 12, cudaMemcpyDeviceToDevice, s));
    midpoints_kernel<<<blocks_for(n), kThreads, 0, s>>>(static_cast<const uint32_t*>(tri2.p), m.nt, first,
                                                       static_cast<const uint32_t*>(m.id_at.p),
                                                       static_cast<float*>(pos2.p), static_cast<float*>(nrm2.p));
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    split_kernel<<<blocks_for(m.nt), kThreads, 0, s>>>(static_cast<uint32_t*>(tri2.p), m.nt,
                                                       static_cast<const uint32_t*>(m.id_at.p));
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    MLODS_CUDA(cudaStreamSynchronize(s));
    m.pos.swap(pos2);
    m.nrm.swap(nrm2);
    m.tri.swap(tri2);
    m.nv = nv2;
    m.nt = nt2;
    return MLODS_OK;
}

}  // namespace mlods
