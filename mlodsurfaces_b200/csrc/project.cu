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
//
// Two kernels share the per-query walk: one for a single tree, and a batched
// one that serves many resident trees (each with its own kernel and options)
// from one persistent launch.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "primitives.cuh"
#include "project.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kEntCount = 0x00FFFFFFu;   // bits 0-23: nodes in the range
constexpr int kEntLiveShift = 24;             // bits 24-27: the warp's queries the range is live for
constexpr uint32_t kEntNoBlend = 1u << 31;
constexpr uint32_t kEntLastOnly = 1u << 30;  // CPU rule multi-point leaf: only the last point is weighted
constexpr float kPiRef = 3.14159265f;         // the reference's literal (Fastapss.cu:93)

// Per-warp stack of sibling ranges: h = {first, count | live mask | flags},
// v[x] = {f, A, dP, g} of query x of the warp; cnt repeats the count word so
// that the pop scan reads 4 bytes.
template <int CAP, int QPW>
struct WarpStack {
    uint2 h[CAP];
    float4 v[CAP][QPW];
    uint32_t cnt[CAP];
};
static_assert(sizeof(uint2) * 2 == sizeof(float4), "the stack arrays stay 16-byte aligned for even CAP");

// Inclusive prefix sum over groups of 16 lanes (4 shuffle steps): exact for
// lanes 0-15, which are the only ones the pop reads.  A round takes at most
// 16 ranges (sibling sets of up to 8 nodes fill the warp with 4): measured
// faster than both the full 5-step scan over 32 ranges and a 3-step scan over
// 8 (precision workload 166.5 / 168.7 / 167.6 ms, torus 7.18 / 7.33 /
// 7.50 ms with two queries per warp).
__device__ __forceinline__ int warp_incl_scan16(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
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

// Sphere fit + projection of the query (frame origin) in double; mirrors
// Fastapss.cu:354-395 (GPU rule) and CPUUtils.cpp:744-781 (CPU rule).
// Returns false when the result is NaN (caller keeps the input, normal 0).
__device__ __forceinline__ bool fit_sphere(const float* s, double step_max, bool gpu_rule, double x[3], float nrm[3])
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
    const double thr = gpu_rule ? 1e-6 : 1e-12;
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
        if (pl != 0.0 || !gpu_rule)
            for (int a = 0; a < 3; ++a) pc[a] /= pl;
        else
            pc[0] = pc[1] = pc[2] = 0.0;
        for (int a = 0; a < 3; ++a) x[a] = c[a] + rad * pc[a];
        for (int a = 0; a < 3; ++a) nv[a] = u123[a] + 2.0 * u4 * x[a];
    }
    const double nl = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    if (nl != 0.0 || !gpu_rule)
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

// Weight with the number of multi-Gaussian terms fixed at compile time
// (NSIG > 0) or read at run time (NSIG == 0); KTYPE < 0 reads the kernel type
// at run time too (uniform across a warp).
template <int KTYPE, int NSIG>
__device__ __forceinline__ float weight_n(const KernelConsts& kc, float d2)
{
    if (KTYPE < 0) {
        if (kc.type == MLODS_GAUSSIAN) return kernel_weight<MLODS_GAUSSIAN>(kc, d2);
        if (kc.type == MLODS_SINGULAR) return kernel_weight<MLODS_SINGULAR>(kc, d2);
        return kernel_weight<MLODS_GAUSSIAN_MULTIPLE>(kc, d2);
    }
    if (KTYPE == MLODS_GAUSSIAN_MULTIPLE && NSIG > 0) {
        float s = 0.f;
#pragma unroll
        for (int i = 0; i < NSIG; ++i) s = fmaf(exp2f(d2 * kc.ms_scale[i]), kc.ms_w[i], s);
        return s;
    }
    return kernel_weight<KTYPE>(kc, d2);
}

struct WalkStats {
    uint32_t pruned = 0;        // near nodes taken as aggregates by kernel-weight pruning (lane sum)
    uint32_t visits = 0;        // query-node visits (nodes each query's own walk touches)
    uint32_t lane_visits = 0;   // node evaluations of the warp (a node shared by the queries counts once)
    uint32_t rounds = 0, iterations = 0;
    int max_top = 0;
    bool overflow = false;
};

// Projects the nq (<= QPW) queries qi[0..nq) of one tree together: n_iter
// iterations each (fewer with a convergence mode), results written to
// out_p / out_n (world frame, or local with c.local_out).  KTYPE / RULE < 0
// take the kernel type / blend rule from c at run time.
//
// The queries of a warp are neighbours in Morton order, so their walks touch
// nearly the same nodes: the warp walks the union once.  Every stack range
// carries the set of queries it is live for (the queries for which the parent
// was near); a lane evaluates its node for each live query -- distance,
// blend weight, kernel weight -- and the node is opened for the queries that
// find it near, or ends the walk as an aggregate for those that find it far.
// Node loads, the pop / push bookkeeping and the leaf logic are paid once for
// all the warp's queries.  Each query's arithmetic is that of its own walk
// (QPW = 1 is the one-query-per-warp walk; two queries per warp run the
// packed form below); only the lane on which a node's contribution is
// accumulated, and so the order of the float sums, depends on the partner
// query.
template <int KTYPE, int NSIG, int RULE, int CAP, int QPW, bool PRUNE>
__device__ __forceinline__ void project_walk(const CloudArgs& c, const uint32_t (&qi)[QPW], int nq,
                                             WarpStack<CAP, QPW>& st, WalkStats& ws)
{
    static_assert(QPW >= 1 && QPW <= 4, "one to four queries per warp");
    const bool gpu_rule = RULE < 0 ? c.rule == MLODS_BLEND_GPU : RULE == MLODS_BLEND_GPU;
    const int lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t le_mask = lane == 31 ? kFull : ((2u << lane) - 1u);
    const float4* __restrict__ ngeom = c.nodes.geom;
    const float4* __restrict__ npm = c.nodes.pm;
    const float4* __restrict__ nnc = c.nodes.nc;
    const float4* __restrict__ naux = c.nodes.aux;
    const float cutoff = c.cutoff;
    const int min_depth = c.min_depth;

    // lane x < nq holds the iterate of query x in the tree's local frame, in
    // double; the other lanes shadow query 0 (their results are not written)
    uint32_t my_q = qi[0];
#pragma unroll
    for (int x = 1; x < QPW; ++x)
        if (lane == x && x < nq) my_q = qi[x];
    double qd[3] = {double(c.q_in[3 * int64_t(my_q)]) - c.o0, double(c.q_in[3 * int64_t(my_q) + 1]) - c.o1,
                    double(c.q_in[3 * int64_t(my_q) + 2]) - c.o2};
    float nrm[3] = {0.f, 0.f, 0.f};
    uint32_t live = (1u << nq) - 1u;  // queries still iterating (warp-uniform)
    uint32_t failed = 0;
    for (int it = 0; it < c.n_iter && live; ++it) {
        float qx[QPW], qy[QPW], qz[QPW];
        {
            const float mx = float(qd[0]), my = float(qd[1]), mz = float(qd[2]);
#pragma unroll
            for (int x = 0; x < QPW; ++x) {  // lane x holds query x's iterate
                qx[x] = __shfl_sync(kFull, mx, x);
                qy[x] = __shfl_sync(kFull, my, x);
                qz[x] = __shfl_sync(kFull, mz, x);
            }
        }
        float acc[QPW][9];
#pragma unroll
        for (int x = 0; x < QPW; ++x)
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[x][k] = 0.f;
        int top = 1;
        if (lane == 0) {
            const uint32_t w0 = 1u | kEntNoBlend | (live << kEntLiveShift);
            st.h[0] = make_uint2(0u, w0);
#pragma unroll
            for (int x = 0; x < QPW; ++x) st.v[0][x] = make_float4(1.f, 0.f, 0.f, 0.f);
            st.cnt[0] = w0;
        }
        __syncwarp();
        while (top > 0) {
            // ---- pop sibling ranges from the top (at most 16) until 32 lanes are filled
            int cn = 0;
            if (lane < top && lane < 16) cn = int(st.cnt[top - 1 - lane] & kEntCount);
            const int incl = warp_incl_scan16(cn);
            const uint32_t fit = __ballot_sync(kFull, lane < top && lane < 16 && incl <= 32);
            const int npop = __popc(fit);
            const bool partial = npop == 0;  // top range wider than a warp (multi-point leaf)
            const int total = partial ? 32 : __shfl_sync(kFull, incl, npop - 1);
            const uint32_t heads = partial ? 1u : __reduce_or_sync(kFull, lane < npop ? (1u << (incl - cn)) : 0u);
            const bool active = lane < total;
            // entry of this lane: the e-th popped range, which starts at the
            // highest head bit at or below the lane
            const uint32_t hb = heads & le_mask;
            const int e = __popc(hb) - 1;
            const int r_start = 31 - __clz(hb);
            const int slot = top - 1 - e;
            const uint2 E = st.h[slot];
            float4 V[QPW];
#pragma unroll
            for (int x = 0; x < QPW; ++x) V[x] = st.v[slot][x];
            const uint32_t r_first = E.x, r_cnt = E.y;
            const uint32_t r_live = (r_cnt >> kEntLiveShift) & ((1u << QPW) - 1u);
            const int r_len = partial ? 32 : int(r_cnt & kEntCount);
            const int old_top = top;
            if (!partial) top -= npop;
            ws.lane_visits += uint32_t(total);
            ws.visits += QPW == 1 ? uint32_t(total) : __reduce_add_sync(kFull, active ? uint32_t(__popc(r_live)) : 0u);
            ++ws.rounds;

            // ---- evaluate one node per lane, for each of its live queries
            const uint32_t node = r_first + uint32_t(lane - r_start);
            float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f), p4 = g4;
            float4 x4 = make_float4(0.f, 0.f, __uint_as_float(kLeafBit | 1u), 0.f);
            if (active) {
                g4 = __ldg(ngeom + node);
                p4 = __ldg(npm + node);
                x4 = __ldg(naux + node);
            }
            const float cr = cutoff * g4.w;
            const bool blend = active && !(r_cnt & kEntNoBlend);
            const int seg_end = r_start + r_len;
            float dist[QPW], f[QPW], A[QPW];
#pragma unroll
            for (int x = 0; x < QPW; ++x) {
                const float cx = g4.x - qx[x], cy = g4.y - qy[x], cz = g4.z - qz[x];
                dist[x] = sqrtf(fmaf(cx, cx, fmaf(cy, cy, cz * cz)));
                float beta = 1.f, kcon = 0.f;
                if (blend && ((r_live >> x) & 1u)) {
                    const float dC = fmaxf(dist[x] - cr, 0.f);
                    const float t = __fdividef(V[x].z, V[x].z + dC);
                    beta = 0.5f - 0.5f * __cosf(kPiRef * t);
                    kcon = (1.f - beta) * V[x].w * (gpu_rule ? p4.w : 1.f);
                }
                // segmented sum over the range (blend ranges hold <= 8 lanes)
#pragma unroll
                for (int o = 1; o < 8; o <<= 1) {
                    const float nv = __shfl_down_sync(kFull, kcon, o);
                    if (lane + o < seg_end) kcon += nv;
                }
                const float K = __shfl_sync(kFull, kcon, r_start);
                f[x] = V[x].x * beta;
                A[x] = V[x].y + K;
            }
            if (!gpu_rule && (r_cnt & kEntLastOnly) && (partial || node != r_first + uint32_t(r_len) - 1u))
#pragma unroll
                for (int x = 0; x < QPW; ++x) f[x] = 0.f;

            const uint32_t info = __float_as_uint(x4.z);
            const uint32_t nfirst = __float_as_uint(x4.y);
            const bool leaf = (info & kLeafBit) != 0;
            const bool multi = (info & kMultiBit) != 0;
            const uint32_t cnt = node_count(info);
            // opened for every live query whatever its distance: the points of
            // a multi-point leaf, the children of a node above min_depth
            const bool opens_all = leaf ? multi : node_depth(info) < min_depth;
            uint32_t term = 0, near = 0;
            if (active && !opens_all) {
#pragma unroll
                for (int x = 0; x < QPW; ++x) {
                    if (!((r_live >> x) & 1u)) continue;
                    if (leaf || dist[x] > cr) term |= 1u << x;
                    else near |= 1u << x;
                }
            }
            if (PRUNE && near) {
                // kernel-weight pruning (extension, off by default): a near
                // node whose whole subtree can weigh no more than the
                // threshold -- the kernel decreases with distance, so w at
                // the distance to the node's bounding sphere bounds every
                // point in it -- is taken as an aggregate instead of opened
#pragma unroll
                for (int x = 0; x < QPW; ++x) {
                    if (!((near >> x) & 1u)) continue;
                    const float dmin = fmaxf(dist[x] - g4.w, 0.f);
                    const float wub = weight_n<KTYPE, NSIG>(c.kc, dmin * dmin);
                    if (f[x] * wub * p4.w < c.prune_thr) {
                        near &= ~(1u << x);
                        term |= 1u << x;
                        ++ws.pruned;
                    }
                }
            }
            const uint32_t child_live = active ? (opens_all ? r_live : near) : 0u;
            const bool push = child_live != 0;
            const uint32_t p_cnt = cnt | (child_live << kEntLiveShift) |
                                   (opens_all ? (kEntNoBlend | (leaf && !gpu_rule ? kEntLastOnly : 0u)) : 0u);

            float4 n4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (term) n4 = __ldg(nnc + node);
            float pv_dP[QPW], pv_g[QPW];
#pragma unroll
            for (int x = 0; x < QPW; ++x) {
                const float px = p4.x - qx[x], py = p4.y - qy[x], pz = p4.z - qz[x];
                const float d2 = fmaf(px, px, fmaf(py, py, pz * pz));
                const float w = weight_n<KTYPE, NSIG>(c.kc, d2);
                pv_dP[x] = cr - dist[x];
                pv_g[x] = f[x] * w / (gpu_rule ? p4.w : float(cnt));
                if ((term >> x) & 1u) {
                    const float coef = fmaf(f[x], w, A[x]);
                    const float cm = coef * p4.w;
                    acc[x][0] += cm;
                    acc[x][1] = fmaf(coef, n4.x, acc[x][1]);
                    acc[x][2] = fmaf(coef, n4.y, acc[x][2]);
                    acc[x][3] = fmaf(coef, n4.z, acc[x][3]);
                    acc[x][4] = fmaf(cm, px, acc[x][4]);
                    acc[x][5] = fmaf(cm, py, acc[x][5]);
                    acc[x][6] = fmaf(cm, pz, acc[x][6]);
                    acc[x][7] = fmaf(coef, fmaf(px, n4.x, fmaf(py, n4.y, fmaf(pz, n4.z, n4.w))), acc[x][7]);
                    acc[x][8] = fmaf(coef, fmaf(d2, p4.w, x4.x), acc[x][8]);
                }
            }
            // ---- push child ranges (every lane has read its entry: the
            // shuffles above depend on those reads)
            __syncwarp();
            if (partial && lane == 0) {
                uint2 rest = st.h[old_top - 1];
                rest.x += 32u;
                rest.y -= 32u;
                st.h[old_top - 1] = rest;
                st.cnt[old_top - 1] = rest.y;
            }
            const uint32_t pm = __ballot_sync(kFull, push);
            const int npush = __popc(pm);
            if (top + npush > CAP) {
                ws.overflow = true;  // the warp's live queries are reported as failed
            } else {
                if (push) {
                    const int pos = top + __popc(pm & lt_mask);
                    st.h[pos] = make_uint2(nfirst, p_cnt);
#pragma unroll
                    for (int x = 0; x < QPW; ++x) st.v[pos][x] = make_float4(f[x], A[x], pv_dP[x], pv_g[x]);
                    st.cnt[pos] = p_cnt;
                }
                top += npush;
            }
            if (top > ws.max_top) ws.max_top = top;
            __syncwarp();
        }
        ws.iterations += uint32_t(__popc(live));
        // warp sums; lane x then fits query x (the other lanes repeat query 0)
        float sv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            sv[k] = warp_sum_f(acc[0][k]);
#pragma unroll
            for (int x = 1; x < QPW; ++x) {
                const float t = warp_sum_f(acc[x][k]);
                if (lane == x) sv[k] = t;
            }
        }
        const bool mine = lane < QPW && ((live >> lane) & 1u);
        double xr[3] = {0.0, 0.0, 0.0};
        const bool ok = !ws.overflow && fit_sphere(sv, double(c.step_max), gpu_rule, xr, nrm);
        bool stop = false;
        if (mine && !ok) {
            failed |= 1u << lane;
            stop = true;
        } else if (mine) {
            // the projection of the float query just evaluated
            const float fx = float(qd[0]), fy = float(qd[1]), fz = float(qd[2]);
            qd[0] = double(fx) + xr[0];
            qd[1] = double(fy) + xr[1];
            qd[2] = double(fz) + xr[2];
            if (c.conv_mode == MLODS_CONVERGE_EXACT) {
                // the next iteration would evaluate the same float query:
                // every remaining iteration returns this result again
                stop = float(qd[0]) == fx && float(qd[1]) == fy && float(qd[2]) == fz;
            } else if (c.conv_mode == MLODS_CONVERGE_TOL) {
                stop = xr[0] * xr[0] + xr[1] * xr[1] + xr[2] * xr[2] < double(c.conv_tol) * double(c.conv_tol);
            }
        }
        live &= ~__ballot_sync(kFull, mine && stop);
    }
    failed = __reduce_or_sync(kFull, failed);
    if (lane < nq) {
        float* op = c.out_p + 3 * int64_t(my_q);
        float* on = c.out_n + 3 * int64_t(my_q);
        // on failure (Fastapss.cu:385-391) the point stays where the failing
        // iteration started and the normal is zero
        const bool bad = (failed >> lane) & 1u;
        if (c.local_out) {
            op[0] = float(qd[0]);
            op[1] = float(qd[1]);
            op[2] = float(qd[2]);
        } else {
            op[0] = float(qd[0] + c.o0);
            op[1] = float(qd[1] + c.o1);
            op[2] = float(qd[2] + c.o2);
        }
        on[0] = bad ? 0.f : nrm[0];
        on[1] = bad ? 0.f : nrm[1];
        on[2] = bad ? 0.f : nrm[2];
    }
}

// ---- two or four queries per warp in packed f32x2 arithmetic --------------
// With several queries per warp every node is evaluated for each with the
// same node data, so their arithmetic pairs up: sm_100's packed instructions
// (FADD2 / FMUL2 / FFMA2) do two queries' operation in one issue slot, each
// element rounded as the scalar instruction would.  The walk is otherwise the
// general one; its stack entries hold each pair's values interleaved
// ({f0, f1, A0, A1}, {dP0, dP1, g0, g1}) so that a pair sits in a register
// pair.

__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b, exactly as a scalar subtraction rounds it
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <int KTYPE, int NSIG>
__device__ __forceinline__ float2 weight_pair(const KernelConsts& kc, float2 d2)
{
    if (KTYPE == MLODS_GAUSSIAN) {
        const float2 t = mul2(d2, splat2(kc.g_scale));
        return add2(make_float2(exp2f(t.x), exp2f(t.y)), splat2(kc.shift));
    } else if (KTYPE == MLODS_GAUSSIAN_MULTIPLE && NSIG > 0) {
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 0; i < NSIG; ++i) {
            const float2 t = mul2(d2, splat2(kc.ms_scale[i]));
            s = fma2(make_float2(exp2f(t.x), exp2f(t.y)), splat2(kc.ms_w[i]), s);
        }
        return s;
    } else if (KTYPE == MLODS_SINGULAR) {
        const float2 u = add2(d2, splat2(kc.shift));
        const float2 l = mul2(splat2(-kc.exponent), make_float2(__log2f(u.x), __log2f(u.y)));
        return mul2(splat2(kc.num), make_float2(exp2f(l.x), exp2f(l.y)));
    } else {
        return make_float2(weight_n<KTYPE, NSIG>(kc, d2.x), weight_n<KTYPE, NSIG>(kc, d2.y));
    }
}

template <int KTYPE, int NSIG, int RULE, int CAP, int NP, bool PRUNE, bool EARLY_NC>
__device__ __forceinline__ void project_packed(const CloudArgs& c, const uint32_t (&qi)[2 * NP], int nq,
                                               WarpStack<CAP, 2 * NP>& st, WalkStats& ws)
{
    constexpr int QPW = 2 * NP;
    const bool gpu_rule = RULE < 0 ? c.rule == MLODS_BLEND_GPU : RULE == MLODS_BLEND_GPU;
    const int lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t le_mask = lane == 31 ? kFull : ((2u << lane) - 1u);
    const float4* __restrict__ ngeom = c.nodes.geom;
    const float4* __restrict__ npm = c.nodes.pm;
    const float4* __restrict__ nnc = c.nodes.nc;
    const float4* __restrict__ naux = c.nodes.aux;
    const float cutoff = c.cutoff;
    const int min_depth = c.min_depth;

    // lane x < nq holds the iterate of query x in the tree's local frame, in
    // double; the other lanes shadow query 0 (their results are not written)
    uint32_t my_q = qi[0];
#pragma unroll
    for (int x = 1; x < QPW; ++x)
        if (lane == x && x < nq) my_q = qi[x];
    double qd[3] = {double(c.q_in[3 * int64_t(my_q)]) - c.o0, double(c.q_in[3 * int64_t(my_q) + 1]) - c.o1,
                    double(c.q_in[3 * int64_t(my_q) + 2]) - c.o2};
    float nrm[3] = {0.f, 0.f, 0.f};
    uint32_t live = (1u << nq) - 1u;  // queries still iterating (warp-uniform)
    uint32_t failed = 0;
    for (int it = 0; it < c.n_iter && live; ++it) {
        // queries 2j and 2j + 1 form pair j
        float2 qx[NP], qy[NP], qz[NP];
        {
            const float mx = float(qd[0]), my = float(qd[1]), mz = float(qd[2]);
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                qx[j] = make_float2(__shfl_sync(kFull, mx, 2 * j), __shfl_sync(kFull, mx, 2 * j + 1));
                qy[j] = make_float2(__shfl_sync(kFull, my, 2 * j), __shfl_sync(kFull, my, 2 * j + 1));
                qz[j] = make_float2(__shfl_sync(kFull, mz, 2 * j), __shfl_sync(kFull, mz, 2 * j + 1));
            }
        }
        float2 acc[NP][9];
#pragma unroll
        for (int j = 0; j < NP; ++j)
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[j][k] = make_float2(0.f, 0.f);
        int top = 1;
        if (lane == 0) {
            const uint32_t w0 = 1u | kEntNoBlend | (live << kEntLiveShift);
            st.h[0] = make_uint2(0u, w0);
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                st.v[0][2 * j] = make_float4(1.f, 1.f, 0.f, 0.f);  // f f A A
                st.v[0][2 * j + 1] = make_float4(0.f, 0.f, 0.f, 0.f);  // dP dP g g
            }
            st.cnt[0] = w0;
        }
        __syncwarp();
        while (top > 0) {
            // ---- pop sibling ranges from the top (at most 16) until 32 lanes are filled
            int cn = 0;
            if (lane < top && lane < 16) cn = int(st.cnt[top - 1 - lane] & kEntCount);
            const int incl = warp_incl_scan16(cn);
            const uint32_t fit = __ballot_sync(kFull, lane < top && lane < 16 && incl <= 32);
            const int npop = __popc(fit);
            const bool partial = npop == 0;  // top range wider than a warp (multi-point leaf)
            const int total = partial ? 32 : __shfl_sync(kFull, incl, npop - 1);
            const uint32_t heads = partial ? 1u : __reduce_or_sync(kFull, lane < npop ? (1u << (incl - cn)) : 0u);
            const bool active = lane < total;
            const uint32_t hb = heads & le_mask;
            const int e = __popc(hb) - 1;
            const int r_start = 31 - __clz(hb);
            const int slot = top - 1 - e;
            const uint2 E = st.h[slot];
            float4 VA[NP], VB[NP];  // {f, f, A, A} and {dP, dP, g, g} of each pair
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                VA[j] = st.v[slot][2 * j];
                VB[j] = st.v[slot][2 * j + 1];
            }
            const uint32_t r_first = E.x, r_cnt = E.y;
            const uint32_t r_live = (r_cnt >> kEntLiveShift) & ((1u << QPW) - 1u);
            const int r_len = partial ? 32 : int(r_cnt & kEntCount);
            const int old_top = top;
            if (!partial) top -= npop;
            ws.lane_visits += uint32_t(total);
            ws.visits += __reduce_add_sync(kFull, active ? uint32_t(__popc(r_live)) : 0u);
            ++ws.rounds;

            // ---- evaluate one node per lane, for every query at once
            const uint32_t node = r_first + uint32_t(lane - r_start);
            float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f), p4 = g4;
            float4 x4 = make_float4(0.f, 0.f, __uint_as_float(kLeafBit | 1u), 0.f);
            // the normal record is needed only where the node ends a walk;
            // loading it with the others hides its latency, which measured
            // faster in the single-tree kernel and slower in the queue kernel
            float4 n4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (active) {
                g4 = __ldg(ngeom + node);
                p4 = __ldg(npm + node);
                x4 = __ldg(naux + node);
                if (EARLY_NC) n4 = __ldg(nnc + node);
            }
            const float cr = cutoff * g4.w;
            const bool blend = active && !(r_cnt & kEntNoBlend);
            const int seg_end = r_start + r_len;
            float2 dist[NP], f[NP], A[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                const float2 cx = sub2(splat2(g4.x), qx[j]), cy = sub2(splat2(g4.y), qy[j]),
                             cz = sub2(splat2(g4.z), qz[j]);
                const float2 dd = fma2(cx, cx, fma2(cy, cy, mul2(cz, cz)));
                dist[j] = make_float2(sqrtf(dd.x), sqrtf(dd.y));
                float2 beta = make_float2(1.f, 1.f), kcon = make_float2(0.f, 0.f);
                if (blend) {
                    const float2 dCs = sub2(dist[j], splat2(cr));
                    const float2 dC = make_float2(fmaxf(dCs.x, 0.f), fmaxf(dCs.y, 0.f));
                    const float2 dP = make_float2(VB[j].x, VB[j].y);
                    const float2 den = add2(dP, dC);
                    const float2 t = mul2(dP, make_float2(__fdividef(1.f, den.x), __fdividef(1.f, den.y)));
                    const float2 a = mul2(splat2(kPiRef), t);
                    beta = fma2(splat2(-0.5f), make_float2(__cosf(a.x), __cosf(a.y)), splat2(0.5f));
                    kcon = mul2(sub2(splat2(1.f), beta), make_float2(VB[j].z, VB[j].w));
                    if (gpu_rule) kcon = mul2(kcon, splat2(p4.w));
                    // a query the range is not live for takes no part
                    if (!((r_live >> (2 * j)) & 1u)) {
                        beta.x = 1.f;
                        kcon.x = 0.f;
                    }
                    if (!((r_live >> (2 * j + 1)) & 1u)) {
                        beta.y = 1.f;
                        kcon.y = 0.f;
                    }
                }
                // segmented sums over the range (blend ranges hold <= 8 lanes)
#pragma unroll
                for (int o = 1; o < 8; o <<= 1) {
                    const float2 nv =
                        make_float2(__shfl_down_sync(kFull, kcon.x, o), __shfl_down_sync(kFull, kcon.y, o));
                    if (lane + o < seg_end) kcon = add2(kcon, nv);
                }
                const float2 K =
                    make_float2(__shfl_sync(kFull, kcon.x, r_start), __shfl_sync(kFull, kcon.y, r_start));
                f[j] = mul2(make_float2(VA[j].x, VA[j].y), beta);
                A[j] = add2(make_float2(VA[j].z, VA[j].w), K);
            }
            if (!gpu_rule && (r_cnt & kEntLastOnly) && (partial || node != r_first + uint32_t(r_len) - 1u))
#pragma unroll
                for (int j = 0; j < NP; ++j) f[j] = make_float2(0.f, 0.f);

            const uint32_t info = __float_as_uint(x4.z);
            const uint32_t nfirst = __float_as_uint(x4.y);
            const bool leaf = (info & kLeafBit) != 0;
            const bool multi = (info & kMultiBit) != 0;
            const uint32_t cnt = node_count(info);
            // opened for every live query whatever its distance: the points of
            // a multi-point leaf, the children of a node above min_depth
            const bool opens_all = leaf ? multi : node_depth(info) < min_depth;
            uint32_t term = 0, near = 0;
            if (active && !opens_all) {
#pragma unroll
                for (int x = 0; x < QPW; ++x) {
                    if (!((r_live >> x) & 1u)) continue;
                    const float d = (x & 1) ? dist[x >> 1].y : dist[x >> 1].x;
                    if (leaf || d > cr) term |= 1u << x;
                    else near |= 1u << x;
                }
            }
            if (PRUNE && near) {
                // kernel-weight pruning (extension, off by default), as in the
                // general walk
#pragma unroll
                for (int x = 0; x < QPW; ++x) {
                    if (!((near >> x) & 1u)) continue;
                    const float d = (x & 1) ? dist[x >> 1].y : dist[x >> 1].x;
                    const float fx = (x & 1) ? f[x >> 1].y : f[x >> 1].x;
                    const float dmin = fmaxf(d - g4.w, 0.f);
                    const float wub = weight_n<KTYPE, NSIG>(c.kc, dmin * dmin);
                    if (fx * wub * p4.w < c.prune_thr) {
                        near &= ~(1u << x);
                        term |= 1u << x;
                        ++ws.pruned;
                    }
                }
            }
            const uint32_t child_live = active ? (opens_all ? r_live : near) : 0u;
            const bool push = child_live != 0;
            const uint32_t p_cnt = cnt | (child_live << kEntLiveShift) |
                                   (opens_all ? (kEntNoBlend | (leaf && !gpu_rule ? kEntLastOnly : 0u)) : 0u);

            const float inv_m = __fdividef(1.f, gpu_rule ? p4.w : float(cnt));
            if (!EARLY_NC && term) n4 = __ldg(nnc + node);
            float2 pv_dP[NP], pv_g[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                const float2 px = sub2(splat2(p4.x), qx[j]), py = sub2(splat2(p4.y), qy[j]),
                             pz = sub2(splat2(p4.z), qz[j]);
                const float2 d2 = fma2(px, px, fma2(py, py, mul2(pz, pz)));
                const float2 w = weight_pair<KTYPE, NSIG>(c.kc, d2);
                pv_dP[j] = sub2(splat2(cr), dist[j]);
                pv_g[j] = mul2(mul2(f[j], w), splat2(inv_m));
                const uint32_t tj = (term >> (2 * j)) & 3u;
                if (tj) {
                    const float2 cf = fma2(f[j], w, A[j]);
                    // a query for which the node is not an aggregate adds zero
                    const float2 coef = make_float2((tj & 1u) ? cf.x : 0.f, (tj & 2u) ? cf.y : 0.f);
                    const float2 cm = mul2(coef, splat2(p4.w));
                    acc[j][0] = add2(acc[j][0], cm);
                    acc[j][1] = fma2(coef, splat2(n4.x), acc[j][1]);
                    acc[j][2] = fma2(coef, splat2(n4.y), acc[j][2]);
                    acc[j][3] = fma2(coef, splat2(n4.z), acc[j][3]);
                    acc[j][4] = fma2(cm, px, acc[j][4]);
                    acc[j][5] = fma2(cm, py, acc[j][5]);
                    acc[j][6] = fma2(cm, pz, acc[j][6]);
                    acc[j][7] = fma2(
                        coef, fma2(px, splat2(n4.x), fma2(py, splat2(n4.y), fma2(pz, splat2(n4.z), splat2(n4.w)))),
                        acc[j][7]);
                    acc[j][8] = fma2(coef, fma2(d2, splat2(p4.w), splat2(x4.x)), acc[j][8]);
                }
            }
            // ---- push child ranges (every lane has read its entry: the
            // shuffles above depend on those reads)
            __syncwarp();
            if (partial && lane == 0) {
                uint2 rest = st.h[old_top - 1];
                rest.x += 32u;
                rest.y -= 32u;
                st.h[old_top - 1] = rest;
                st.cnt[old_top - 1] = rest.y;
            }
            const uint32_t pmask = __ballot_sync(kFull, push);
            const int npush = __popc(pmask);
            if (top + npush > CAP) {
                ws.overflow = true;  // the warp's live queries are reported as failed
            } else {
                if (push) {
                    const int pos = top + __popc(pmask & lt_mask);
                    st.h[pos] = make_uint2(nfirst, p_cnt);
#pragma unroll
                    for (int j = 0; j < NP; ++j) {
                        st.v[pos][2 * j] = make_float4(f[j].x, f[j].y, A[j].x, A[j].y);
                        st.v[pos][2 * j + 1] = make_float4(pv_dP[j].x, pv_dP[j].y, pv_g[j].x, pv_g[j].y);
                    }
                    st.cnt[pos] = p_cnt;
                }
                top += npush;
            }
            if (top > ws.max_top) ws.max_top = top;
            __syncwarp();
        }
        ws.iterations += uint32_t(__popc(live));
        // warp sums; lane x then fits query x (the other lanes repeat query 0)
        float sv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            sv[k] = warp_sum_f(acc[0][k].x);
#pragma unroll
            for (int x = 1; x < QPW; ++x) {
                const float t = warp_sum_f((x & 1) ? acc[x >> 1][k].y : acc[x >> 1][k].x);
                if (lane == x) sv[k] = t;
            }
        }
        const bool mine = lane < QPW && ((live >> lane) & 1u);
        double xr[3] = {0.0, 0.0, 0.0};
        const bool ok = !ws.overflow && fit_sphere(sv, double(c.step_max), gpu_rule, xr, nrm);
        bool stop = false;
        if (mine && !ok) {
            failed |= 1u << lane;
            stop = true;
        } else if (mine) {
            // the projection of the float query just evaluated
            const float fx = float(qd[0]), fy = float(qd[1]), fz = float(qd[2]);
            qd[0] = double(fx) + xr[0];
            qd[1] = double(fy) + xr[1];
            qd[2] = double(fz) + xr[2];
            if (c.conv_mode == MLODS_CONVERGE_EXACT) {
                // the next iteration would evaluate the same float query:
                // every remaining iteration returns this result again
                stop = float(qd[0]) == fx && float(qd[1]) == fy && float(qd[2]) == fz;
            } else if (c.conv_mode == MLODS_CONVERGE_TOL) {
                stop = xr[0] * xr[0] + xr[1] * xr[1] + xr[2] * xr[2] < double(c.conv_tol) * double(c.conv_tol);
            }
        }
        live &= ~__ballot_sync(kFull, mine && stop);
    }
    failed = __reduce_or_sync(kFull, failed);
    if (lane < nq) {
        float* op = c.out_p + 3 * int64_t(my_q);
        float* on = c.out_n + 3 * int64_t(my_q);
        // on failure (Fastapss.cu:385-391) the point stays where the failing
        // iteration started and the normal is zero
        const bool bad = (failed >> lane) & 1u;
        if (c.local_out) {
            op[0] = float(qd[0]);
            op[1] = float(qd[1]);
            op[2] = float(qd[2]);
        } else {
            op[0] = float(qd[0] + c.o0);
            op[1] = float(qd[1] + c.o1);
            op[2] = float(qd[2] + c.o2);
        }
        on[0] = bad ? 0.f : nrm[0];
        on[1] = bad ? 0.f : nrm[1];
        on[2] = bad ? 0.f : nrm[2];
    }
}

// Projects the nq (<= QPW) queries qi[0..nq) of one tree together (the
// general walk for one query per warp, the packed form for two or four).
template <int KTYPE, int NSIG, int RULE, int CAP, int QPW, bool PRUNE = false, bool EARLY_NC = true>
__device__ __forceinline__ void project_queries(const CloudArgs& c, const uint32_t (&qi)[QPW], int nq,
                                                WarpStack<CAP, QPW>& st, WalkStats& ws)
{
    if constexpr (QPW == 2 || QPW == 4)
        project_packed<KTYPE, NSIG, RULE, CAP, QPW / 2, PRUNE, EARLY_NC>(c, qi, nq, st, ws);
    else project_walk<KTYPE, NSIG, RULE, CAP, QPW, PRUNE>(c, qi, nq, st, ws);
}

// Per-warp totals of the walks, kept in 64 bits across queries.
struct WarpTotals {
    WalkStats sum;  // max_top only
    int64_t overflows = 0;
    int64_t visits = 0, lane_visits = 0, rounds = 0, iterations = 0, pruned = 0;
    __device__ void add(const WalkStats& ws, int nq)
    {
        pruned += ws.pruned;
        visits += ws.visits;
        lane_visits += ws.lane_visits;
        rounds += ws.rounds;
        iterations += ws.iterations;
        if (ws.max_top > sum.max_top) sum.max_top = ws.max_top;
        overflows += ws.overflow ? nq : 0;
    }
    __device__ void flush(int64_t* stats)
    {
        if ((threadIdx.x & 31) != 0 || !stats) return;
        atomicAdd(reinterpret_cast<unsigned long long*>(&stats[0]), (unsigned long long)visits);
        atomicAdd(reinterpret_cast<unsigned long long*>(&stats[4]), (unsigned long long)rounds);
        atomicAdd(reinterpret_cast<unsigned long long*>(&stats[5]), (unsigned long long)iterations);
        atomicAdd(reinterpret_cast<unsigned long long*>(&stats[6]), (unsigned long long)lane_visits);
        atomicMax(reinterpret_cast<unsigned long long*>(&stats[1]), (unsigned long long)sum.max_top);
        if (overflows) atomicAdd(reinterpret_cast<unsigned long long*>(&stats[2]), (unsigned long long)overflows);
    }
    // per-lane counts, summed over the warp first
    __device__ void flush_pruned(int64_t* stats)
    {
        unsigned long long p = (unsigned long long)pruned;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(kFull, p, o);
        if ((threadIdx.x & 31) == 0 && stats && p) atomicAdd(reinterpret_cast<unsigned long long*>(&stats[7]), p);
    }
};

// Blocks per SM the single-tree kernel is compiled for and its stack
// capacity: one query per warp fits 48 registers at 10 blocks; two and four
// need more registers (64, 96) and wider stack entries.
template <int QPW>
struct WalkShape {
    static constexpr int kMinBlocks = QPW == 1 ? kProjectMinBlocks : (QPW == 2 ? kProjectPairMinBlocks : 5);
    static constexpr int kCap = QPW == 1 ? kProjectStackCap : kProjectPairStackCap;
};

template <int KTYPE, int NSIG, int RULE, int QPW, bool PRUNE>
__global__ void __launch_bounds__(kProjectThreads, WalkShape<QPW>::kMinBlocks) mlod_project_kernel(ProjectArgs a)
{
    constexpr int CAP = WalkShape<QPW>::kCap;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    WarpStack<CAP, QPW>& st = reinterpret_cast<WarpStack<CAP, QPW>*>(smem_raw)[threadIdx.x >> 5];
    WarpTotals tot;
    for (;;) {
        unsigned int qs = 0;
        if (lane == 0) qs = atomicAdd(a.counter, unsigned(QPW));
        qs = __shfl_sync(kFull, qs, 0);
        if (int64_t(qs) >= a.nq) break;
        const int nq = int(min(int64_t(QPW), a.nq - int64_t(qs)));
        uint32_t qi[QPW];
#pragma unroll
        for (int x = 0; x < QPW; ++x) {
            const uint32_t s = qs + uint32_t(x < nq ? x : 0);
            qi[x] = a.order ? __ldg(a.order + s) - a.order_base : s;
        }
        WalkStats ws;
        project_queries<KTYPE, NSIG, RULE, CAP, QPW, PRUNE>(a.cloud, qi, nq, st, ws);
        tot.add(ws, nq);
    }
    tot.flush(a.stats);
    tot.flush_pruned(a.stats);
}

// ---- many trees in one persistent launch ---------------------------------
// The launch arguments of up to kQueueMaxClouds clouds travel BY VALUE in the
// queue kernel's parameters (__grid_constant__: read in place from the
// parameter bank), as the single-tree kernel's one cloud does: the walk
// reads them from read-only memory that no store can alias.  The clouds are
// laid out along a virtual slot line, the clouds with the most work first,
// each padded to a multiple of 4 slots, so that the queries a warp takes
// together are those a launch of the cloud alone would pair.
struct QueueLaunch {
    const uint32_t* order;
    unsigned long long* counter;
    int64_t* stats;
    int n;                          // clouds in this launch
    int64_t v_total;                // length of the virtual slot line
    int64_t vbase[kQueueMaxClouds + 1];  // virtual start of the j-th cloud in processing order
    int64_t base[kQueueMaxClouds];  // first slot (and global query index) of each cloud
    int64_t len[kQueueMaxClouds];   // its query count
    int32_t cloud_at[kQueueMaxClouds];  // the cloud at the j-th place of the line
    int32_t spec[kQueueMaxClouds];  // its walk specialisation
    CloudArgs clouds[kQueueMaxClouds];
};
static_assert(sizeof(QueueLaunch) <= 32000, "queue launch parameters must fit the 32 KB kernel parameter space");

// The specialisation of the walk a cloud runs with: kernel family and number
// of multi-Gaussian terms (2-6 and 8 have their own code, other counts share
// one) and blend rule.
constexpr int kWalkSpecs = 18;
inline int walk_spec_id(const CloudArgs& c)
{
    int k = 8;  // multi-Gaussian, terms counted at run time
    if (c.kc.type == MLODS_GAUSSIAN) k = 0;
    else if (c.kc.type == MLODS_SINGULAR) k = 1;
    else if (c.kc.nsig >= 2 && c.kc.nsig <= 6) k = c.kc.nsig;
    else if (c.kc.nsig == 8) k = 7;
    return (c.rule == MLODS_BLEND_GPU ? 0 : 1) * 9 + k;
}

template <int RULE, int CAP, int QPW>
__device__ __forceinline__ void walk_k(int k, const CloudArgs& c, const uint32_t (&qi)[QPW], int nq,
                                       WarpStack<CAP, QPW>& st, WalkStats& ws)
{
    switch (k) {
    case 0: project_queries<MLODS_GAUSSIAN, 0, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    case 1: project_queries<MLODS_SINGULAR, 0, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    case 2: project_queries<MLODS_GAUSSIAN_MULTIPLE, 2, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    case 3: project_queries<MLODS_GAUSSIAN_MULTIPLE, 3, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    case 4: project_queries<MLODS_GAUSSIAN_MULTIPLE, 4, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    case 5: project_queries<MLODS_GAUSSIAN_MULTIPLE, 5, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    case 6: project_queries<MLODS_GAUSSIAN_MULTIPLE, 6, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    case 7: project_queries<MLODS_GAUSSIAN_MULTIPLE, 8, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    default: project_queries<MLODS_GAUSSIAN_MULTIPLE, 0, RULE, CAP, QPW, false, false>(c, qi, nq, st, ws); break;
    }
}

// Every cloud of a group in ONE persistent launch: each warp takes QPW
// consecutive virtual slots from the counter (consecutive warps take
// consecutive queries, as in the single-tree kernel, so the warps working at
// any moment share node records in L1 and L2), finds their cloud by binary
// search over the line and walks them with the cloud's own specialisation;
// the kernel is compiled with the schedule's registers and blocks per SM.
template <int QPW>
__global__ void __launch_bounds__(kProjectThreads, WalkShape<QPW>::kMinBlocks)
    mlod_queue_kernel(const __grid_constant__ QueueLaunch p)
{
    constexpr int CAP = WalkShape<QPW>::kCap;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    WarpStack<CAP, QPW>& st = reinterpret_cast<WarpStack<CAP, QPW>*>(smem_raw)[threadIdx.x >> 5];
    WarpTotals tot;
    for (;;) {
        unsigned long long v = 0;
        if (lane == 0) v = atomicAdd(p.counter, (unsigned long long)QPW);
        v = __shfl_sync(kFull, v, 0);
        if (int64_t(v) >= p.v_total) break;
        int lo = 0, hi = p.n;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (int64_t(v) >= p.vbase[mid]) lo = mid; else hi = mid;
        }
        const int ci = p.cloud_at[lo];
        const int64_t off = int64_t(v) - p.vbase[lo];
        const int nq = int(min(int64_t(QPW), p.len[ci] - off));
        if (nq <= 0) continue;  // the padding at the end of a cloud
        const int64_t b = p.base[ci];
        uint32_t qi[QPW];
#pragma unroll
        for (int x = 0; x < QPW; ++x) {
            const int64_t slot = b + off + (x < nq ? x : 0);
            qi[x] = uint32_t((p.order ? int64_t(__ldg(p.order + slot)) : slot) - b);
        }
        const CloudArgs& c = p.clouds[ci];
        const int sp = p.spec[ci];
        WalkStats ws;
        if (sp < 9) walk_k<MLODS_BLEND_GPU, CAP, QPW>(sp, c, qi, nq, st, ws);
        else walk_k<MLODS_BLEND_CPU, CAP, QPW>(sp - 9, c, qi, nq, st, ws);
        tot.add(ws, nq);
    }
    tot.flush(p.stats);
    tot.flush_pruned(p.stats);
}

template <typename Kern>
int64_t persistent_grid(Kern kern, size_t smem, int64_t work_warps, int sm_count, cudaError_t* err)
{
    int per_sm = 0;
    *err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kProjectThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const int64_t want = (work_warps + kProjectThreads / 32 - 1) / (kProjectThreads / 32);
    int64_t grid = int64_t(per_sm) * sm_count;
    if (grid > want) grid = want;
    return grid < 1 ? 1 : grid;
}

template <int KTYPE, int NSIG, int RULE, int QPW>
cudaError_t launch_typed(const ProjectArgs& a, int sm_count, cudaStream_t s)
{
    constexpr int CAP = WalkShape<QPW>::kCap;
    // kernel-weight pruning is a variant of its own (four queries per warp
    // has none), so the default walk carries none of its code
    constexpr bool kCanPrune = QPW <= 2;
    auto kern = (kCanPrune && a.cloud.prune_thr > 0.f) ? mlod_project_kernel<KTYPE, NSIG, RULE, QPW, kCanPrune>
                                                       : mlod_project_kernel<KTYPE, NSIG, RULE, QPW, false>;
    const size_t smem = size_t(kProjectThreads / 32) * sizeof(WarpStack<CAP, QPW>);
    cudaError_t e = cudaSuccess;
    const int64_t grid = persistent_grid(kern, smem, (a.nq + QPW - 1) / QPW, sm_count, &e);
    if (e != cudaSuccess) return e;
    kern<<<unsigned(grid), kProjectThreads, smem, s>>>(a);
    note_launch();
    return cudaGetLastError();
}

template <int RULE, int QPW>
cudaError_t launch_rule(const ProjectArgs& a, int ktype, int sm_count, cudaStream_t s)
{
    if (ktype == MLODS_GAUSSIAN) return launch_typed<MLODS_GAUSSIAN, 0, RULE, QPW>(a, sm_count, s);
    if (ktype == MLODS_SINGULAR) return launch_typed<MLODS_SINGULAR, 0, RULE, QPW>(a, sm_count, s);
    switch (a.cloud.kc.nsig) {
    case 2: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, 2, RULE, QPW>(a, sm_count, s);
    case 3: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, 3, RULE, QPW>(a, sm_count, s);
    case 4: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, 4, RULE, QPW>(a, sm_count, s);
    case 5: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, 5, RULE, QPW>(a, sm_count, s);
    case 6: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, 6, RULE, QPW>(a, sm_count, s);
    case 8: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, 8, RULE, QPW>(a, sm_count, s);
    default: return launch_typed<MLODS_GAUSSIAN_MULTIPLE, 0, RULE, QPW>(a, sm_count, s);
    }
}

// Morton key of a query on a 1024^3 grid over its tree's root box, prefixed
// by the cloud index in the batched case.
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

__global__ void batch_codes_kernel(const float* __restrict__ q, int64_t n, const int64_t* __restrict__ q_offsets,
                                   int n_clouds, const BatchFrame* __restrict__ frames, int morton,
                                   uint64_t* __restrict__ keys, uint32_t* __restrict__ idx)
{
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = n_clouds;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (i >= q_offsets[mid]) lo = mid; else hi = mid;
    }
    const BatchFrame fr = frames[lo];
    uint32_t c[3];
    const double o[3] = {fr.o0, fr.o1, fr.o2};
    for (int k = 0; k < 3; ++k) {
        float u = float(double(q[3 * i + k]) - o[k]) * fr.inv_ext + 0.5f;
        u = fminf(fmaxf(u, 0.f), 0.99999994f);
        c[k] = uint32_t(u * 1024.f);
    }
    uint64_t code = uint64_t(fr.rank);
    for (int b = 9; b >= 0; --b)
        code = (code << 3) | ((c[0] >> b) & 1u) | (((c[1] >> b) & 1u) << 1) | (((c[2] >> b) & 1u) << 2);
    keys[i] = morton ? code : (uint64_t(fr.rank) << 30);
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

inline size_t up256(size_t v) { return (v + 255) / 256 * 256; }

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
        if (a.queries_per_warp == 4) return launch_rule<MLODS_BLEND_GPU, 4>(a, ktype, sm_count, s);
        if (a.queries_per_warp == 2) return launch_rule<MLODS_BLEND_GPU, 2>(a, ktype, sm_count, s);
        return launch_rule<MLODS_BLEND_GPU, 1>(a, ktype, sm_count, s);
    }
    if (a.queries_per_warp == 4) return launch_rule<MLODS_BLEND_CPU, 4>(a, ktype, sm_count, s);
    if (a.queries_per_warp == 2) return launch_rule<MLODS_BLEND_CPU, 2>(a, ktype, sm_count, s);
    return launch_rule<MLODS_BLEND_CPU, 1>(a, ktype, sm_count, s);
}

namespace
{
template <int QPW>
cudaError_t launch_queue_typed(const QueueArgs& a, int sm_count, int grid_pct, cudaStream_t s)
{
    constexpr int CAP = WalkShape<QPW>::kCap;
    const size_t smem = size_t(kProjectThreads / 32) * sizeof(WarpStack<CAP, QPW>);
    const int n_groups = queue_groups(a.n_clouds);
    for (int g = 0; g < n_groups; ++g) {
        const int c0 = g * kQueueMaxClouds, nc = std::min(kQueueMaxClouds, a.n_clouds - c0);
        QueueLaunch p;
        std::memset(&p, 0, sizeof p);
        p.order = a.order;
        p.counter = a.counters + g;
        p.stats = a.stats;
        p.n = nc;
        std::vector<int> idx(static_cast<size_t>(nc));
        for (int i = 0; i < nc; ++i) {
            idx[size_t(i)] = i;
            p.clouds[i] = a.clouds[c0 + i];
            p.base[i] = a.base[c0 + i];
            p.len[i] = a.len[c0 + i];
            p.spec[i] = walk_spec_id(p.clouds[i]);
        }
        // the clouds with the most work first, so that the launch ends on
        // small ones; optionally grouped by specialisation first
        auto work = [&](int i) { return p.len[i] * int64_t(std::max(p.clouds[i].n_iter, 1)); };
        int64_t spec_work[kWalkSpecs] = {};
        for (int i = 0; i < nc; ++i) spec_work[p.spec[i]] += work(i);
        const bool by_spec = a.line_order == kQueueBySpecialisation;
        std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
            if (by_spec && p.spec[x] != p.spec[y]) {
                const int64_t wx = spec_work[p.spec[x]], wy = spec_work[p.spec[y]];
                return wx != wy ? wx > wy : p.spec[x] < p.spec[y];
            }
            return work(x) > work(y);
        });
        int64_t v = 0;
        for (int j = 0; j < nc; ++j) {
            p.cloud_at[j] = idx[size_t(j)];
            p.vbase[j] = v;
            v += (p.len[idx[size_t(j)]] + 3) / 4 * 4;
        }
        p.vbase[nc] = v;
        p.v_total = v;
        if (v == 0) continue;
        cudaError_t e = cudaSuccess;
        int64_t grid = persistent_grid(mlod_queue_kernel<QPW>, smem, (v + QPW - 1) / QPW, sm_count, &e);
        if (e != cudaSuccess) return e;
        if (grid_pct > 0 && grid_pct < 100) grid = std::max<int64_t>(1, grid * grid_pct / 100);
        mlod_queue_kernel<QPW><<<unsigned(grid), kProjectThreads, smem, s>>>(p);
        note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
}  // namespace

cudaError_t launch_mlod_queue(const QueueArgs& a, int queries_per_warp, int sm_count, int grid_pct, cudaStream_t s)
{
    if (queries_per_warp == 2) return launch_queue_typed<2>(a, sm_count, grid_pct, s);
    return launch_queue_typed<1>(a, sm_count, grid_pct, s);
}

int64_t project_resident_queries(int queries_per_warp, int sm_count)
{
    const int per_sm = queries_per_warp == 4 ? WalkShape<4>::kMinBlocks
                                             : (queries_per_warp == 2 ? WalkShape<2>::kMinBlocks : WalkShape<1>::kMinBlocks);
    return int64_t(per_sm) * (kProjectThreads / 32) * queries_per_warp * sm_count;
}

size_t query_order_temp_bytes(int64_t n)
{
    return 2 * up256(size_t(n) * 8) + up256(size_t(n) * 4) + radix_temp_bytes(n);
}

cudaError_t compute_query_order(const float* d_q, int64_t n, const double origin[3], float extent, uint32_t* d_order,
                                void* temp, cudaStream_t s)
{
    char* t = static_cast<char*>(temp);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(t);
    uint64_t* k1 = reinterpret_cast<uint64_t*>(t + up256(size_t(n) * 8));
    uint32_t* v1 = reinterpret_cast<uint32_t*>(t + 2 * up256(size_t(n) * 8));
    void* rt = t + 2 * up256(size_t(n) * 8) + up256(size_t(n) * 4);
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

cudaError_t compute_batch_order(const float* d_q, int64_t n, const int64_t* d_q_offsets, int n_clouds,
                                const BatchFrame* d_frames, bool morton, uint32_t* d_order, void* temp,
                                cudaStream_t s)
{
    char* t = static_cast<char*>(temp);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(t);
    uint64_t* k1 = reinterpret_cast<uint64_t*>(t + up256(size_t(n) * 8));
    uint32_t* v1 = reinterpret_cast<uint32_t*>(t + 2 * up256(size_t(n) * 8));
    void* rt = t + 2 * up256(size_t(n) * 8) + up256(size_t(n) * 4);
    batch_codes_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(d_q, n, d_q_offsets, n_clouds, d_frames,
                                                                 morton ? 1 : 0, k0, d_order);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int cbits = 1;
    while ((1 << cbits) < n_clouds) ++cbits;
    bool alt = false;
    e = radix_sort_pairs_u64(k0, d_order, k1, v1, n, 30 + cbits, &alt, rt, s);
    if (e != cudaSuccess) return e;
    if (alt) e = cudaMemcpyAsync(d_order, v1, size_t(n) * 4, cudaMemcpyDeviceToDevice, s);
    return e;
}

}  // namespace mlods
