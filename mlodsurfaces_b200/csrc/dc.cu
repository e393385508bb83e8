// dc.cu -- dual-contouring corner field and per-cell vertex on the device.
//
// The reference evaluates the signed field at the 8 corners of every cell of
// the DC octree, projecting every corner once per cell that owns it
// (scene.cpp:1361-1394: 8 x cells projections, duplicates included), then
// builds a vertex per cell from the edge crossings (dual_contouring.h:124-176).
// Here the corners are keyed on the integer lattice of the deepest level,
// radix-sorted and de-duplicated, projected once each with the MLoD kernel
// (one iteration, as scene.cpp:1385), and the field f = (c - x).n (NaN when
// the projection failed, |n|^2 < 0.5) is scattered back to the cells.  The
// vertex is solved in double.  With the reference's zero normal field
// (scene.cpp:1355-1358) the QEF has A = 0 and its minimum-norm solution is the
// mass point of the crossings; use_normals = 1 instead feeds the projected
// normals (interpolated along each edge) into a full 3x3 QEF.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dc.h"
#include "primitives.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) { return unsigned((n + kThreads - 1) / kThreads); }

struct Lattice {
    int bits;       // bits per axis in a key
    int64_t bias;   // added to lattice coordinates to make them non-negative
    int max_depth;
};

__device__ __forceinline__ void corner_lattice(const int4 c, int k, int max_depth, int64_t l[3])
{
    const int64_t delta = int64_t(1) << (max_depth - c.x);
    l[0] = (int64_t(c.y) + (k & 1)) * delta;
    l[1] = (int64_t(c.z) + ((k >> 1) & 1)) * delta;
    l[2] = (int64_t(c.w) + ((k >> 2) & 1)) * delta;
}

__global__ void corner_keys_kernel(const int4* __restrict__ cells, int64_t n_cells, Lattice L,
                                   uint64_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_cells * 8) return;
    const int4 c = cells[i >> 3];
    int64_t l[3];
    corner_lattice(c, int(i & 7), L.max_depth, l);
    keys[i] = (uint64_t(l[0] + L.bias) << (2 * L.bits)) | (uint64_t(l[1] + L.bias) << L.bits) |
              uint64_t(l[2] + L.bias);
    vals[i] = uint32_t(i);
}

// Cell checks: depth in [0, max_depth] and the cell's lattice box inside the
// key range.  err |= 1 (depth) or 2 (lattice); bad = lowest failing cell.
__global__ void check_cells_kernel(const int4* __restrict__ cells, int64_t n_cells, Lattice L,
                                   uint32_t* __restrict__ err, unsigned long long* __restrict__ bad)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_cells) return;
    const int4 c = cells[i];
    uint32_t e = 0;
    if (c.x < 0 || c.x > L.max_depth) {
        e = 1u;
    } else {
        const int64_t delta = int64_t(1) << (L.max_depth - c.x);
        const int v[3] = {c.y, c.z, c.w};
        for (int a = 0; a < 3; ++a) {
            const int64_t l0 = int64_t(v[a]) * delta, l1 = (int64_t(v[a]) + 1) * delta;
            if (l0 < -L.bias || l1 >= L.bias) e = 2u;
        }
    }
    if (e) {
        atomicOr(err, e);
        atomicMin(bad, (unsigned long long)i);
    }
}

__global__ void unique_flags_kernel(const uint64_t* __restrict__ keys, int64_t n, uint32_t* __restrict__ flags)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// Unique corners -> positions in the tree's frame: new2bbox applied to the
// unit-cube point lattice * w (scene.cpp:1370-1377), float arithmetic.
__global__ void unique_corners_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ excl,
                                      int64_t n, Lattice L, float w, const float* __restrict__ xf,
                                      float* __restrict__ pos)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i != 0 && keys[i] == keys[i - 1]) return;
    const uint64_t k = keys[i];
    const uint64_t m = (uint64_t(1) << L.bits) - 1;
    const float u[3] = {float(int64_t((k >> (2 * L.bits)) & m) - L.bias) * w,
                        float(int64_t((k >> L.bits) & m) - L.bias) * w, float(int64_t(k & m) - L.bias) * w};
    const int64_t j = excl[i];
    for (int r = 0; r < 3; ++r)
        pos[3 * j + r] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(xf[4 * r], u[0]), __fmul_rn(xf[4 * r + 1], u[1])),
                                             __fmul_rn(xf[4 * r + 2], u[2])),
                                   xf[4 * r + 3]);
}

// f = (c - x).n, NaN when |n|^2 < 0.5 (scene.cpp:1388-1394)
__global__ void field_kernel(const float* __restrict__ c, const float* __restrict__ x, const float* __restrict__ nv,
                             int64_t n, float* __restrict__ f)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float n0 = nv[3 * i], n1 = nv[3 * i + 1], n2 = nv[3 * i + 2];
    const float l2 = __fadd_rn(__fadd_rn(__fmul_rn(n0, n0), __fmul_rn(n1, n1)), __fmul_rn(n2, n2));
    if (l2 < 0.5f) {
        f[i] = __int_as_float(0x7fc00000);
        return;
    }
    const float d0 = __fsub_rn(c[3 * i], x[3 * i]), d1 = __fsub_rn(c[3 * i + 1], x[3 * i + 1]),
                d2 = __fsub_rn(c[3 * i + 2], x[3 * i + 2]);
    f[i] = __fadd_rn(__fadd_rn(__fmul_rn(d0, n0), __fmul_rn(d1, n1)), __fmul_rn(d2, n2));
}

__global__ void scatter_kernel(const uint32_t* __restrict__ vals, const uint32_t* __restrict__ excl,
                               const uint32_t* __restrict__ flags, int64_t n, const float* __restrict__ f,
                               const float* __restrict__ nv, float* __restrict__ corner_f, float* __restrict__ corner_n)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t u = int64_t(excl[i]) + int64_t(flags[i]) - 1;
    const uint32_t v = vals[i];
    corner_f[v] = f[u];
    if (corner_n)
        for (int r = 0; r < 3; ++r) corner_n[3 * int64_t(v) + r] = nv[3 * u + r];
}

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations (double).
__device__ void jacobi3(double a[3][3], double v[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) v[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 12; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off < 1e-30) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (fabs(a[p][q]) < 1e-300) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < 3; ++k) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = cs * akp - sn * akq;
                    a[k][q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = cs * apk - sn * aqk;
                    a[q][k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = cs * vkp - sn * vkq;
                    v[k][q] = sn * vkp + cs * vkq;
                }
            }
    }
}

// Per cell: crossings on the 12 edges (node_edges, dual_contouring.h:132-137)
// with a sign change ((val < 0) compared, so NaN counts as non-negative), the
// linear crossing x = -fu / (fv - fu), then the vertex (dual_contouring.h:143-175).
__global__ void vertex_kernel(const int4* __restrict__ cells, int64_t n_cells, int max_depth,
                              const float* __restrict__ corner_f, const float* __restrict__ corner_n,
                              float* __restrict__ vertex, int32_t* __restrict__ n_cross)
{
    const int64_t ci = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ci >= n_cells) return;
    const int edges[12][2] = {{0, 1}, {0, 2}, {1, 3}, {2, 3}, {4, 5}, {4, 6}, {5, 7}, {6, 7},
                              {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    const int4 c = cells[ci];
    if (!corner_n) {
        // The reference's zero normal field (scene.cpp:1355-1358): its QEF
        // has A = 0, so the vertex is the mass point of the crossings
        // (QEF::center, dual_contouring.h:98-111), computed here in float in
        // the reference's order with every operation rounded once, so that
        // the vertex is the reference's bit for bit: x = -fu / (fv - fu),
        // p = x v + (1 - x) u (intersection, :116-121), sum += p, sum / count.
        const float wf = 1.0f / float(int64_t(1) << max_depth);
        float sum[3] = {0.f, 0.f, 0.f};
        int cnt = 0;
        for (int e = 0; e < 12; ++e) {
            const int ka = edges[e][0], kb = edges[e][1];
            const float fa = corner_f[8 * ci + ka], fb = corner_f[8 * ci + kb];
            if ((fa < 0.f) == (fb < 0.f)) continue;
            int64_t la[3], lb[3];
            corner_lattice(c, ka, max_depth, la);
            corner_lattice(c, kb, max_depth, lb);
            const float x = -__fdiv_rn(fa, __fsub_rn(fb, fa));
            const float omx = __fsub_rn(1.f, x);
            for (int r = 0; r < 3; ++r) {
                const float u = __fmul_rn(float(la[r]), wf), v = __fmul_rn(float(lb[r]), wf);
                sum[r] = __fadd_rn(sum[r], __fadd_rn(__fmul_rn(x, v), __fmul_rn(omx, u)));
            }
            ++cnt;
        }
        // no crossing (a minimal edge through a larger cell, :163-169) or a
        // NaN mass point: the cell centre (unit_octree::center, octree.h:808-812)
        const float width = 1.0f / float(int64_t(1) << c.x);
        const int pos[3] = {c.y, c.z, c.w};
        float out[3];
        bool bad = cnt == 0;
        for (int r = 0; r < 3; ++r) {
            out[r] = cnt ? __fdiv_rn(sum[r], float(cnt)) : 0.f;
            bad = bad || isnan(out[r]);
        }
        if (bad)
            for (int r = 0; r < 3; ++r) out[r] = __fmul_rn(__fadd_rn(float(pos[r]), 0.5f), width);
        for (int r = 0; r < 3; ++r) vertex[3 * ci + r] = out[r];
        n_cross[ci] = cnt;
        return;
    }
    const double w = 1.0 / double(int64_t(1) << max_depth);
    const double width = 1.0 / double(int64_t(1) << c.x);
    const double lo[3] = {c.y * width, c.z * width, c.w * width};
    double sum[3] = {0, 0, 0};
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double b[3] = {0, 0, 0};
    int cnt = 0;
    for (int e = 0; e < 12; ++e) {
        const int ka = edges[e][0], kb = edges[e][1];
        const double fa = corner_f[8 * ci + ka], fb = corner_f[8 * ci + kb];
        if ((fa < 0) == (fb < 0)) continue;
        int64_t la[3], lb[3];
        corner_lattice(c, ka, max_depth, la);
        corner_lattice(c, kb, max_depth, lb);
        const double x = -fa / (fb - fa);
        double p[3];
        for (int r = 0; r < 3; ++r) p[r] = x * (double(lb[r]) * w) + (1.0 - x) * (double(la[r]) * w);
        for (int r = 0; r < 3; ++r) sum[r] += p[r];
        if (corner_n) {
            double nn[3];
            for (int r = 0; r < 3; ++r)
                nn[r] = x * corner_n[3 * (8 * ci + kb) + r] + (1.0 - x) * corner_n[3 * (8 * ci + ka) + r];
            const double l = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
            if (l > 0) {
                for (int r = 0; r < 3; ++r) nn[r] /= l;
                const double pd = p[0] * nn[0] + p[1] * nn[1] + p[2] * nn[2];
                for (int r = 0; r < 3; ++r) {
                    b[r] += pd * nn[r];
                    for (int s = 0; s < 3; ++s) A[r][s] += nn[r] * nn[s];
                }
            }
        }
        ++cnt;
    }
    double out[3];
    const double center[3] = {lo[0] + 0.5 * width, lo[1] + 0.5 * width, lo[2] + 0.5 * width};
    if (cnt == 0) {
        for (int r = 0; r < 3; ++r) out[r] = center[r];
    } else {
        double m[3];
        for (int r = 0; r < 3; ++r) m[r] = sum[r] / cnt;
        for (int r = 0; r < 3; ++r) out[r] = m[r];
        if (corner_n) {
            // minimum-norm solution of A y = b - A m, vertex = y + m
            double rhs[3];
            for (int r = 0; r < 3; ++r) rhs[r] = b[r] - (A[r][0] * m[0] + A[r][1] * m[1] + A[r][2] * m[2]);
            double V[3][3];
            jacobi3(A, V);
            const double lmax = fmax(fabs(A[0][0]), fmax(fabs(A[1][1]), fabs(A[2][2])));
            double y[3] = {0, 0, 0};
            for (int k = 0; k < 3; ++k) {
                const double lk = A[k][k];
                if (lmax > 0 && fabs(lk) > 1e-6 * lmax) {
                    const double proj = (V[0][k] * rhs[0] + V[1][k] * rhs[1] + V[2][k] * rhs[2]) / lk;
                    for (int r = 0; r < 3; ++r) y[r] += proj * V[r][k];
                }
            }
            for (int r = 0; r < 3; ++r) out[r] = y[r] + m[r];
            bool inside = true;
            for (int r = 0; r < 3; ++r) inside = inside && lo[r] <= out[r] && out[r] <= lo[r] + width;
            if (!inside)
                for (int r = 0; r < 3; ++r) out[r] = m[r];
        }
    }
    if (isnan(out[0]) || isnan(out[1]) || isnan(out[2]))
        for (int r = 0; r < 3; ++r) out[r] = center[r];
    for (int r = 0; r < 3; ++r) vertex[3 * ci + r] = float(out[r]);
    n_cross[ci] = cnt;
}

inline size_t al(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

int dc_field_device(mlods_tree_s* T, int64_t n_cells, const int32_t* cells, bool cells_on_device, int max_depth,
                    const float* xform, int use_normals, DcField& out, cudaStream_t s)
{
    dc_field_free(out);
    if (n_cells <= 0 || !cells || !xform) {
        set_last_error("dc evaluate: bad arguments");
        return MLODS_ERR_INVALID;
    }
    if (max_depth < 0 || max_depth > 17 || n_cells * 8 >= (int64_t(1) << 31)) {
        set_last_error("dc evaluate: max_depth %d or %lld cells out of range", max_depth, (long long)n_cells);
        return MLODS_ERR_CAPACITY;
    }
    Lattice L;
    L.max_depth = max_depth;
    L.bits = max_depth + 4;
    L.bias = int64_t(1) << (max_depth + 2);
    const int64_t nc8 = n_cells * 8;
    size_t bytes = al(size_t(n_cells) * 16) + 2 * al(size_t(nc8) * 8) + 2 * al(size_t(nc8) * 4) +
                   2 * al(size_t(nc8) * 4) + al(128) + std::max(radix_temp_bytes(nc8), scan_temp_bytes(nc8));
    bytes += al(size_t(nc8) * 4) + (use_normals ? al(size_t(nc8) * 12) : 0) + al(size_t(n_cells) * 16);
    char* base = nullptr;
    MLODS_CUDA(scratch_alloc(reinterpret_cast<void**>(&base), bytes, s));
    out.base = base;
    out.stream = s;
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base + off;
        off += al(b);
        return p;
    };
    int4* d_cells = reinterpret_cast<int4*>(take(size_t(n_cells) * 16));
    uint64_t* k0 = reinterpret_cast<uint64_t*>(take(size_t(nc8) * 8));
    uint64_t* k1 = reinterpret_cast<uint64_t*>(take(size_t(nc8) * 8));
    uint32_t* v0 = reinterpret_cast<uint32_t*>(take(size_t(nc8) * 4));
    uint32_t* v1 = reinterpret_cast<uint32_t*>(take(size_t(nc8) * 4));
    uint32_t* flags = reinterpret_cast<uint32_t*>(take(size_t(nc8) * 4));
    uint32_t* excl = reinterpret_cast<uint32_t*>(take(size_t(nc8) * 4));
    uint32_t* d_total = reinterpret_cast<uint32_t*>(take(128));  // unique count, cell errors, first bad cell, xform
    uint32_t* d_err = d_total + 1;
    unsigned long long* d_bad = reinterpret_cast<unsigned long long*>(d_total + 2);
    float* d_xf = reinterpret_cast<float*>(d_total + 4);
    void* tmp = take(std::max(radix_temp_bytes(nc8), scan_temp_bytes(nc8)));
    float* d_cf = reinterpret_cast<float*>(take(size_t(nc8) * 4));
    float* d_cn = use_normals ? reinterpret_cast<float*>(take(size_t(nc8) * 12)) : nullptr;
    float* d_vert = reinterpret_cast<float*>(take(size_t(n_cells) * 12));
    int32_t* d_ncross = reinterpret_cast<int32_t*>(d_vert + 3 * n_cells);
    auto fail = [&](cudaError_t e, const char* what) {
        dc_field_free(out);
        return cuda_fail(e, what, __FILE__, __LINE__);
    };
#define DC_CHECK(call, what)                            \
    do {                                                \
        cudaError_t _e = (call);                        \
        if (_e != cudaSuccess) return fail(_e, what);   \
    } while (0)

    DC_CHECK(cudaMemcpyAsync(d_cells, cells, size_t(n_cells) * 16,
                             cells_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s),
             "upload cells");
    DC_CHECK(cudaMemcpyAsync(d_xf, xform, 12 * sizeof(float), cudaMemcpyHostToDevice, s), "upload xform");
    DC_CHECK(cudaMemsetAsync(d_err, 0, 4, s), "clear cell errors");
    DC_CHECK(cudaMemsetAsync(d_bad, 0xff, 8, s), "clear first bad cell");
    check_cells_kernel<<<grid_for(n_cells), kThreads, 0, s>>>(d_cells, n_cells, L, d_err, d_bad);
    note_launch();
    DC_CHECK(cudaGetLastError(), "check cells");
    corner_keys_kernel<<<grid_for(nc8), kThreads, 0, s>>>(d_cells, n_cells, L, k0, v0);
    note_launch();
    DC_CHECK(cudaGetLastError(), "corner keys");
    bool alt = false;
    DC_CHECK(radix_sort_pairs_u64(k0, v0, k1, v1, nc8, 3 * L.bits, &alt, tmp, s), "corner sort");
    uint64_t* keys = alt ? k1 : k0;
    uint32_t* vals = alt ? v1 : v0;
    unique_flags_kernel<<<grid_for(nc8), kThreads, 0, s>>>(keys, nc8, flags);
    note_launch();
    DC_CHECK(cudaGetLastError(), "unique flags");
    DC_CHECK(exclusive_scan_u32(flags, excl, nc8, d_total, tmp, s), "unique scan");
    uint32_t h_head[4] = {0, 0, 0, 0};  // unique count, cell errors, first bad cell
    DC_CHECK(cudaMemcpyAsync(h_head, d_total, 16, cudaMemcpyDeviceToHost, s), "read unique count");
    DC_CHECK(cudaStreamSynchronize(s), "sync unique count");
    if (h_head[1]) {
        unsigned long long bad = 0;
        std::memcpy(&bad, h_head + 2, 8);
        dc_field_free(out);
        if (h_head[1] & 1u) {
            set_last_error("dc evaluate: cell %llu has a depth outside [0, %d]", bad, max_depth);
            return MLODS_ERR_INVALID;
        }
        set_last_error("dc evaluate: cell %llu lies outside the supported lattice", bad);
        return MLODS_ERR_CAPACITY;
    }
    const int64_t U = h_head[0];
    // U unique corners x (3 position + 3 projection + 3 normal + field)
    DC_CHECK(scratch_alloc(&out.base2, size_t(std::max<int64_t>(U, 1)) * 40, s), "unique corner buffers");
    float* pos = static_cast<float*>(out.base2);
    float* cpos = pos;
    float* cproj = pos + 3 * U;
    float* cnrm = pos + 6 * U;
    float* cf = pos + 9 * U;
    const float w = 1.0f / float(1 << max_depth);
    unique_corners_kernel<<<grid_for(nc8), kThreads, 0, s>>>(keys, excl, nc8, L, w, d_xf, cpos);
    note_launch();
    DC_CHECK(cudaGetLastError(), "unique corners");
    // one projection step of every unique corner (scene.cpp:1382-1386)
    int rc = project_buffers(T, U, cpos, cproj, cnrm, 1, -1.f, s);
    if (rc != MLODS_OK) {
        dc_field_free(out);
        return rc;
    }
    field_kernel<<<grid_for(U), kThreads, 0, s>>>(cpos, cproj, cnrm, U, cf);
    note_launch();
    DC_CHECK(cudaGetLastError(), "field");
    scatter_kernel<<<grid_for(nc8), kThreads, 0, s>>>(vals, excl, flags, nc8, cf, cnrm, d_cf, d_cn);
    note_launch();
    DC_CHECK(cudaGetLastError(), "scatter");
    vertex_kernel<<<grid_for(n_cells), kThreads, 0, s>>>(d_cells, n_cells, max_depth, d_cf, d_cn, d_vert, d_ncross);
    note_launch();
    DC_CHECK(cudaGetLastError(), "vertex");
    DC_CHECK(scratch_free(out.base2, s), "free unique corner buffers");  // stream-ordered: after the scatter
    out.base2 = nullptr;
    DC_CHECK(cudaStreamSynchronize(s), "sync dc");
#undef DC_CHECK
    out.cells = d_cells;
    out.cf = d_cf;
    out.vert = d_vert;
    out.ncross = d_ncross;
    out.n = n_cells;
    out.n_unique = U;
    return MLODS_OK;
}

void dc_field_free(DcField& f)
{
    scratch_free(f.base, f.stream);
    scratch_free(f.base2, f.stream);
    f = DcField{};
}

int dc_evaluate(mlods_tree_s* T, int64_t n_cells, const int32_t* cells, bool cells_on_device, int max_depth,
                const float* xform, int use_normals, float* corner_f, float* vertex, int32_t* n_cross,
                int64_t* n_unique, cudaStream_t s)
{
    if (!corner_f || !vertex || !n_cross) {
        set_last_error("dc evaluate: bad arguments");
        return MLODS_ERR_INVALID;
    }
    DcField f;
    int rc = dc_field_device(T, n_cells, cells, cells_on_device, max_depth, xform, use_normals, f, s);
    if (rc != MLODS_OK) return rc;
    // cudaMemcpyDefault: host or device outputs, told apart by address (unified addressing)
    cudaError_t e = cudaMemcpyAsync(corner_f, f.cf, size_t(n_cells) * 32, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(vertex, f.vert, size_t(n_cells) * 12, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(n_cross, f.ncross, size_t(n_cells) * 4, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (n_unique) *n_unique = f.n_unique;
    dc_field_free(f);
    if (e != cudaSuccess) return cuda_fail(e, "dc evaluate: download", __FILE__, __LINE__);
    return MLODS_OK;
}

}  // namespace mlods
