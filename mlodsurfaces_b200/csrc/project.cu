// project.cu -- MLoD projection: one warp per query, lanes = tree nodes.
//
// The reference (Fastapss.cu:160-437) gives each query one thread that walks
// the octree with a per-depth accumulator array in local memory.  Here a warp
// owns a query and its 32 lanes evaluate 32 nodes at a time, taken from a
// per-warp stack of sibling ranges in shared memory.
//
// The traversal is rewritten as a linear recursion so that no per-depth
// partial sums are needed.  For a node n reached with factor f (product of
// ancestor blend weights) and inherited coefficient A:
//   terminal (leaf or far):  accumulate (f * w_n + A) * S_n(q)
//   near (|q-c| <= cutoff r): each child c gets
//       f_c = f * beta_c,   A_c = A + K_n,
//       K_n = f * w_n * sum_c (1 - beta_c) rho_c
//   with beta_c = (1 - cos(pi t)) / 2, t = dP / (dP + max(dC, 0)),
//   rho_c = a_c / a_n (GPU rule, Fastapss.cu:244) or 1 / #children (CPU rule,
//   CPUUtils.cpp:485).  This equals the reference's
//       sum_c [beta_c R(c) + (1 - beta_c) w_n rho_c S_n]
//   because S_n = sum_c S_c exactly (node moments are sums of child moments).
// Lanes of one sibling range cooperate: each computes its own beta_c and a
// segmented shuffle reduction gives K_n, so every lane does the same work.
//
// Moments are accumulated per lane in float, in the query-centred frame
// (S_p = sum c m0 (pbar - q), S_pn = sum c (cpn + (pbar - q).n),
// S_pp = sum c (cpp + |pbar - q|^2 m0)), reduced across the warp, and the
// algebraic sphere is solved in double (Fastapss.cu:354-395).
#include <cmath>

#include "primitives.cuh"
#include "project.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kEntCount = 0x00FFFFFFu;
constexpr uint32_t kEntNoBlend = 1u << 31;
constexpr uint32_t kEntLastOnly = 1u << 30;  // CPU rule multi-point leaf: only the last point is weighted
constexpr float kPiRef = 3.14159265f;         // the reference's literal (Fastapss.cu:93)

template <int CAP>
struct WarpStack {
    uint32_t first[CAP];
    uint32_t cnt[CAP];
    float f[CAP];
    float A[CAP];
    float dP[CAP];
    float g[CAP];
};

__device__ __forceinline__ int warp_incl_scan_i(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int n = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

__device__ __forceinline__ float warp_sum_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ DNode load_node(const DNode* __restrict__ nodes, uint32_t i)
{
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    DNode n;
    n.cx = a.x; n.cy = a.y; n.cz = a.z; n.r = a.w;
    n.px = b.x; n.py = b.y; n.pz = b.z; n.m0 = b.w;
    n.nx = c.x; n.ny = c.y; n.nz = c.z; n.cpn = c.w;
    n.cpp = d.x;
    n.first = __float_as_uint(d.y);
    n.info = __float_as_uint(d.z);
    n.parent = __float_as_uint(d.w);
    return n;
}

// Sphere fit + projection of the query (frame origin) in double; mirrors
// Fastapss.cu:354-395 (GPU rule) and CPUUtils.cpp:744-781 (CPU rule).
// Returns false when the result is NaN (caller keeps the input, normal 0).
template <int RULE>
__device__ __forceinline__ bool fit_sphere(const float* s, double step_max, double x[3], float nrm[3])
{
    const double Sw = s[0];
    const double Sn[3] = {s[1], s[2], s[3]};
    const double Sp[3] = {s[4], s[5], s[6]};
    const double Spn = s[7], Spp = s[8];
    const double u4 = 0.5 * (Spn - (Sp[0] * Sn[0] + Sp[1] * Sn[1] + Sp[2] * Sn[2]) / Sw) /
                      (Spp - (Sp[0] * Sp[0] + Sp[1] * Sp[1] + Sp[2] * Sp[2]) / Sw);
    double u123[3];
    for (int a = 0; a < 3; ++a) u123[a] = (Sn[a] - 2.0 * u4 * Sp[a]) / Sw;
    const double u0 = -((Sp[0] * u123[0] + Sp[1] * u123[1] + Sp[2] * u123[2]) + u4 * Spp) / Sw;
    const double thr = RULE == MLODS_BLEND_GPU ? 1e-6 : 1e-12;
    double nv[3];
    if (fabs(u4) < thr) {
        const double m[3] = {-u123[0], -u123[1], -u123[2]};
        const double lambda = u0 / (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        for (int a = 0; a < 3; ++a) x[a] = lambda * m[a];
        for (int a = 0; a < 3; ++a) nv[a] = Sn[a];
    } else {
        double c[3];
        for (int a = 0; a < 3; ++a) c[a] = u123[a] / (-2.0 * u4);
        const double r2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] - u0 / u4;
        const double rad = sqrt(r2 > 0.0 ? r2 : 0.0);
        double pc[3] = {-c[0], -c[1], -c[2]};
        const double pl = sqrt(pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
        if (pl != 0.0 || RULE == MLODS_BLEND_CPU)
            for (int a = 0; a < 3; ++a) pc[a] /= pl;
        else
            pc[0] = pc[1] = pc[2] = 0.0;
        for (int a = 0; a < 3; ++a) x[a] = c[a] + rad * pc[a];
        for (int a = 0; a < 3; ++a) nv[a] = u123[a] + 2.0 * u4 * x[a];
    }
    const double nl = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    if (nl != 0.0 || RULE == MLODS_BLEND_CPU)
        for (int a = 0; a < 3; ++a) nv[a] /= nl;
    else
        nv[0] = nv[1] = nv[2] = 0.0;
    if (isnan(x[0]) || isnan(x[1]) || isnan(x[2])) return false;
    const double step = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (step > step_max)
        for (int a = 0; a < 3; ++a) x[a] *= step_max / step;
    for (int a = 0; a < 3; ++a) nrm[a] = float(nv[a]);
    return true;
}

template <int KTYPE, int RULE, int CAP>
__global__ void __launch_bounds__(kProjectThreads) mlod_project_kernel(ProjectArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    WarpStack<CAP>& st = reinterpret_cast<WarpStack<CAP>*>(smem_raw)[warp];
    const uint32_t lt_mask = (1u << lane) - 1u;
    const DNode* __restrict__ nodes = a.nodes;
    const float cutoff = a.cutoff;
    const int min_depth = a.min_depth;

    int64_t visits = 0;
    int64_t rounds = 0;
    int max_top = 0;
    int64_t overflows = 0;

    for (;;) {
        unsigned int qs = 0;
        if (lane == 0) qs = atomicAdd(a.counter, 1u);
        qs = __shfl_sync(kFull, qs, 0);
        if (int64_t(qs) >= a.nq) break;
        const uint32_t qi = a.order ? a.order[qs] : qs;
        // iterate in the tree's local frame, in double
        double qd[3] = {double(a.q_in[3 * int64_t(qi)]) - a.o0, double(a.q_in[3 * int64_t(qi) + 1]) - a.o1,
                        double(a.q_in[3 * int64_t(qi) + 2]) - a.o2};
        float nrm[3] = {0.f, 0.f, 0.f};
        bool failed = false;
        bool overflow = false;
        for (int it = 0; it < a.n_iter && !failed; ++it) {
            const float qx = float(qd[0]), qy = float(qd[1]), qz = float(qd[2]);
            float acc[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[k] = 0.f;
            int top = 1;
            if (lane == 0) {
                st.first[0] = 0;
                st.cnt[0] = 1u | kEntNoBlend;
                st.f[0] = 1.f;
                st.A[0] = 0.f;
                st.dP[0] = 0.f;
                st.g[0] = 0.f;
            }
            __syncwarp();
            while (top > 0) {
                // ---- pop sibling ranges from the top until 32 lanes are filled
                uint32_t e_first = 0, e_cnt = 0;
                float e_f = 0.f, e_A = 0.f, e_dP = 0.f, e_g = 0.f;
                int c = 0;
                if (lane < top) {
                    const int slot = top - 1 - lane;
                    e_first = st.first[slot];
                    e_cnt = st.cnt[slot];
                    e_f = st.f[slot];
                    e_A = st.A[slot];
                    e_dP = st.dP[slot];
                    e_g = st.g[slot];
                    c = int(e_cnt & kEntCount);
                }
                const int incl = warp_incl_scan_i(c);
                const uint32_t fit = __ballot_sync(kFull, lane < top && incl <= 32);
                int npop = __popc(fit);
                const bool partial = npop == 0;  // top range wider than a warp (multi-point leaf)
                int total;
                uint32_t headbit;
                if (partial) {
                    total = 32;
                    headbit = lane == 0 ? 1u : 0u;
                } else {
                    total = __shfl_sync(kFull, incl, npop - 1);
                    headbit = lane < npop ? (1u << (incl - c)) : 0u;
                }
                const uint32_t heads = __reduce_or_sync(kFull, headbit);
                const bool active = lane < total;
                const int e = active ? __popc(heads & (lane == 31 ? kFull : ((2u << lane) - 1u))) - 1 : 0;
                const uint32_t r_first = __shfl_sync(kFull, e_first, e);
                const uint32_t r_cnt = __shfl_sync(kFull, e_cnt, e);
                const float r_f = __shfl_sync(kFull, e_f, e);
                const float r_A = __shfl_sync(kFull, e_A, e);
                const float r_dP = __shfl_sync(kFull, e_dP, e);
                const float r_g = __shfl_sync(kFull, e_g, e);
                const int r_start = partial ? 0 : __shfl_sync(kFull, incl - c, e);
                const int r_len = partial ? 32 : int(r_cnt & kEntCount);
                if (partial) {
                    if (lane == 0) {
                        st.first[top - 1] = e_first + 32u;
                        st.cnt[top - 1] = e_cnt - 32u;
                    }
                } else {
                    top -= npop;
                }
                visits += total;
                ++rounds;

                // ---- evaluate one node per lane
                const uint32_t node = r_first + uint32_t(lane - r_start);
                DNode nd;
                if (active) {
                    nd = load_node(nodes, node);
                } else {
                    nd.cx = nd.cy = nd.cz = 0.f;
                    nd.r = 0.f;
                    nd.px = nd.py = nd.pz = 0.f;
                    nd.m0 = 0.f;
                    nd.nx = nd.ny = nd.nz = nd.cpn = nd.cpp = 0.f;
                    nd.first = 0;
                    nd.info = kLeafBit | 1u;
                    nd.parent = 0;
                }
                const float cx = nd.cx - qx, cy = nd.cy - qy, cz = nd.cz - qz;
                const float dist = sqrtf(fmaf(cx, cx, fmaf(cy, cy, cz * cz)));
                float beta = 1.f, kcon = 0.f;
                if (active && !(r_cnt & kEntNoBlend)) {
                    const float dC = fmaxf(dist - cutoff * nd.r, 0.f);
                    const float t = __fdividef(r_dP, r_dP + dC);
                    beta = 0.5f - 0.5f * __cosf(kPiRef * t);
                    kcon = (1.f - beta) * r_g * (RULE == MLODS_BLEND_GPU ? nd.m0 : 1.f);
                }
                // segmented sum over the range (blend ranges hold <= 8 lanes)
                {
                    const int seg_end = r_start + r_len;
#pragma unroll
                    for (int o = 1; o < 8; o <<= 1) {
                        const float nv = __shfl_down_sync(kFull, kcon, o);
                        if (lane + o < seg_end) kcon += nv;
                    }
                }
                const float K = __shfl_sync(kFull, kcon, r_start);
                float f = r_f * beta;
                const float A = r_A + K;
                if (RULE == MLODS_BLEND_CPU && (r_cnt & kEntLastOnly) && node != r_first + uint32_t(r_len) - 1u &&
                    !partial)
                    f = 0.f;
                if (RULE == MLODS_BLEND_CPU && (r_cnt & kEntLastOnly) && partial) f = 0.f;

                const float px = nd.px - qx, py = nd.py - qy, pz = nd.pz - qz;
                const float d2 = fmaf(px, px, fmaf(py, py, pz * pz));
                const float w = kernel_weight<KTYPE>(a.kc, d2);
                const uint32_t info = nd.info;
                const bool leaf = (info & kLeafBit) != 0;
                const bool multi = (info & kMultiBit) != 0;
                const int cnt = int(node_count(info));
                bool terminal = false, push = false;
                uint32_t p_first = 0, p_cnt = 0;
                float p_dP = 0.f, p_g = 0.f;
                if (active) {
                    if (leaf) {
                        if (!multi) {
                            terminal = true;
                        } else {
                            push = true;
                            p_first = nd.first;
                            p_cnt = uint32_t(cnt) | kEntNoBlend | (RULE == MLODS_BLEND_CPU ? kEntLastOnly : 0u);
                        }
                    } else if (node_depth(info) < min_depth) {
                        push = true;
                        p_first = nd.first;
                        p_cnt = uint32_t(cnt) | kEntNoBlend;
                    } else if (dist > cutoff * nd.r) {
                        terminal = true;
                    } else {
                        push = true;
                        p_first = nd.first;
                        p_cnt = uint32_t(cnt);
                        p_dP = cutoff * nd.r - dist;
                        p_g = f * w / (RULE == MLODS_BLEND_GPU ? nd.m0 : float(cnt));
                    }
                }
                if (terminal) {
                    const float coef = fmaf(f, w, A);
                    const float cm = coef * nd.m0;
                    acc[0] += cm;
                    acc[1] = fmaf(coef, nd.nx, acc[1]);
                    acc[2] = fmaf(coef, nd.ny, acc[2]);
                    acc[3] = fmaf(coef, nd.nz, acc[3]);
                    acc[4] = fmaf(cm, px, acc[4]);
                    acc[5] = fmaf(cm, py, acc[5]);
                    acc[6] = fmaf(cm, pz, acc[6]);
                    acc[7] = fmaf(coef, fmaf(px, nd.nx, fmaf(py, nd.ny, fmaf(pz, nd.nz, nd.cpn))), acc[7]);
                    acc[8] = fmaf(coef, fmaf(d2, nd.m0, nd.cpp), acc[8]);
                }
                // ---- push child ranges
                const uint32_t pm = __ballot_sync(kFull, push);
                const int npush = __popc(pm);
                if (top + npush > CAP) {
                    overflow = true;  // the query is reported as failed
                } else {
                    if (push) {
                        const int pos = top + __popc(pm & lt_mask);
                        st.first[pos] = p_first;
                        st.cnt[pos] = p_cnt;
                        st.f[pos] = f;
                        st.A[pos] = A;
                        st.dP[pos] = p_dP;
                        st.g[pos] = p_g;
                    }
                    top += npush;
                }
                if (top > max_top) max_top = top;
                __syncwarp();
            }
            float s[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) s[k] = warp_sum_f(acc[k]);
            double x[3];
            if (overflow || !fit_sphere<RULE>(s, double(a.step_max), x, nrm)) {
                failed = true;
                break;
            }
            qd[0] += x[0];
            qd[1] += x[1];
            qd[2] += x[2];
        }
        if (lane == 0) {
            float* op = a.out_p + 3 * int64_t(qi);
            float* on = a.out_n + 3 * int64_t(qi);
            if (failed) {
                // Fastapss.cu:385-391: keep the point, zero normal.  The in-place
                // buffer already holds the start of the failing iteration.
                op[0] = float(qd[0] + a.o0);
                op[1] = float(qd[1] + a.o1);
                op[2] = float(qd[2] + a.o2);
                on[0] = on[1] = on[2] = 0.f;
            } else {
                op[0] = float(qd[0] + a.o0);
                op[1] = float(qd[1] + a.o1);
                op[2] = float(qd[2] + a.o2);
                on[0] = nrm[0];
                on[1] = nrm[1];
                on[2] = nrm[2];
            }
        }
        if (overflow) ++overflows;
    }
    if (lane == 0 && a.stats) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[0]), (unsigned long long)visits);
        atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[4]), (unsigned long long)rounds);
        atomicMax(reinterpret_cast<unsigned long long*>(&a.stats[1]), (unsigned long long)max_top);
        if (overflows) atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[2]), (unsigned long long)overflows);
    }
}

template <int KTYPE, int RULE>
cudaError_t launch_typed(const ProjectArgs& a, int sm_count, cudaStream_t s)
{
    constexpr int CAP = kProjectStackCap;
    auto kern = mlod_project_kernel<KTYPE, RULE, CAP>;
    const size_t smem = size_t(kProjectThreads / 32) * sizeof(WarpStack<CAP>);
    static bool attr_done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        attr_done[dev] = true;
    }
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kProjectThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int64_t want = (a.nq + kProjectThreads / 32 - 1) / (kProjectThreads / 32);
    int64_t grid = int64_t(per_sm) * sm_count;
    if (grid > want) grid = want;
    if (grid < 1) grid = 1;
    kern<<<unsigned(grid), kProjectThreads, smem, s>>>(a);
    note_launch();
    return cudaGetLastError();
}

__global__ void query_codes_kernel(const float* __restrict__ q, int64_t n, double o0, double o1, double o2,
                                   float inv_ext, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx)
{
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c[3];
    const double o[3] = {o0, o1, o2};
    for (int k = 0; k < 3; ++k) {
        float u = float(double(q[3 * i + k]) - o[k]) * inv_ext + 0.5f;  // [0, 1) inside the root box
        u = fminf(fmaxf(u, 0.f), 0.99999994f);
        c[k] = uint32_t(u * 1024.f);
    }
    uint64_t code = 0;
    for (int b = 9; b >= 0; --b)
        code = (code << 3) | ((c[0] >> b) & 1u) | (((c[1] >> b) & 1u) << 1) | (((c[2] >> b) & 1u) << 2);
    keys[i] = code;
    idx[i] = uint32_t(i);
}

__global__ void reorganize_kernel(float* __restrict__ q, const uint32_t* __restrict__ inv, int64_t n_inv,
                                  uint32_t end_valid)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_inv) return;
    const int64_t a = inv[i], b = int64_t(end_valid) - 1 - i;
    for (int c = 0; c < 3; ++c) {
        const float t = q[3 * a + c];
        q[3 * a + c] = q[3 * b + c];
        q[3 * b + c] = t;
    }
}

}  // namespace

cudaError_t launch_reorganize(float* d_q, const uint32_t* d_invalid, int64_t n_invalid, uint32_t end_valid,
                              cudaStream_t s)
{
    reorganize_kernel<<<unsigned((n_invalid + 255) / 256), 256, 0, s>>>(d_q, d_invalid, n_invalid, end_valid);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_mlod_project(const ProjectArgs& a, int ktype, int rule, int sm_count, cudaStream_t s)
{
    if (rule == MLODS_BLEND_GPU) {
        switch (ktype) {
        case MLODS_GAUSSIAN: return launch_typed<MLODS_GAUSSIAN, MLODS_BLEND_GPU>(a, sm_count, s);
        case MLODS_SINGULAR: return launch_typed<MLODS_SINGULAR, MLODS_BLEND_GPU>(a, sm_count, s);
        default: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, MLODS_BLEND_GPU>(a, sm_count, s);
        }
    }
    switch (ktype) {
    case MLODS_GAUSSIAN: return launch_typed<MLODS_GAUSSIAN, MLODS_BLEND_CPU>(a, sm_count, s);
    case MLODS_SINGULAR: return launch_typed<MLODS_SINGULAR, MLODS_BLEND_CPU>(a, sm_count, s);
    default: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, MLODS_BLEND_CPU>(a, sm_count, s);
    }
}

size_t query_order_temp_bytes(int64_t n)
{
    const size_t al = 256;
    auto up = [&](size_t v) { return (v + al - 1) / al * al; };
    return 2 * up(size_t(n) * 8) + up(size_t(n) * 4) + radix_temp_bytes(n);
}

cudaError_t compute_query_order(const float* d_q, int64_t n, const double origin[3], float extent, uint32_t* d_order,
                                void* temp, cudaStream_t s)
{
    const size_t al = 256;
    auto up = [&](size_t v) { return (v + al - 1) / al * al; };
    char* t = static_cast<char*>(temp);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(t);
    uint64_t* k1 = reinterpret_cast<uint64_t*>(t + up(size_t(n) * 8));
    uint32_t* v1 = reinterpret_cast<uint32_t*>(t + 2 * up(size_t(n) * 8));
    void* rt = t + 2 * up(size_t(n) * 8) + up(size_t(n) * 4);
    const float inv_ext = extent > 0.f ? 1.f / extent : 1.f;
    query_codes_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(d_q, n, origin[0], origin[1], origin[2], inv_ext, k0,
                                                                 d_order);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    bool alt = false;
    e = radix_sort_pairs_u64(k0, d_order, k1, v1, n, 30, &alt, rt, s);
    if (e != cudaSuccess) return e;
    if (alt) e = cudaMemcpyAsync(d_order, v1, size_t(n) * 4, cudaMemcpyDeviceToDevice, s);
    return e;
}

}  // namespace mlods
