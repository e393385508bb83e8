// gather.cu -- kNN and ball gathers over the device octree and the APSS
// projection built on them (APSSOctree::projectAPSSCPU, CPUUtils.cpp:690-737),
// plus the all-points (global) APSS projection (GlobalAPSS.cu:113-235).
//
// One warp per query.  Neighbour candidates are ranked by the squared
// distance evaluated exactly as the reference kd-tree does (kdTreeNN.h:424):
// float differences of the world coordinates, float products, left-to-right
// float sums, no contraction.  The k best (k <= 32) live one per lane, sorted
// across the warp; batches of candidates are merged with a bitonic network
// (keys (distance, original index), so ties at the k-th distance resolve to
// the lower index; the reference resolves them by kd-tree visiting order).
// The search starts from the 32 points around the query's Morton position
// (an upper bound for the k-th distance) and walks the octree with the
// bounding sphere of each node box, widened by the float rounding of the
// local frame.  The fit is the reference's CPU one (|u4| < 1e-12).
#include <cfloat>
#include <cmath>

#include "gather.cuh"
#include "tree.cuh"

namespace mlods
{
namespace
{
constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kGCount = 0x7FFFFFFFu;
constexpr uint32_t kGPoints = 1u << 31;  // entry is a range of sorted point positions
#ifndef MLODS_GATHER_MIN_BLOCKS
#define MLODS_GATHER_MIN_BLOCKS 10
#endif
constexpr int kGatherMinBlocks = MLODS_GATHER_MIN_BLOCKS;  // resident blocks per SM the register budget aims at
#ifndef MLODS_KNN_MIN_BLOCKS
#define MLODS_KNN_MIN_BLOCKS 9
#endif
constexpr int kKnnMinBlocks = MLODS_KNN_MIN_BLOCKS;  // the same for the kNN projection (56 registers)
constexpr int kGatherCap = 256;          // stack entries per warp
// A range entry holds at most 8 nodes, each pushing at most one entry, so a
// depth-first walk below any entry adds at most 7 entries per level for the
// 12 node levels and the point level, plus one: 92.  The walk pops as many
// entries as fill the warp while the stack has room for one such walk after
// a full batch (32 pushes), and only the top entry beyond that, so the
// stack stays below kGatherCap.
constexpr int kDfsReserve = 7 * (kMaxTreeDepth + 1) + 1;
constexpr int kBatchPopLimit = kGatherCap - kDfsReserve - 32;
static_assert(kBatchPopLimit > 0, "gather stack too small for a depth-first walk");

struct GStack {
    uint32_t first[kGatherCap];
    uint32_t cnt[kGatherCap];
};

// Per-warp state of a kNN projection query between iterations (uniform over
// the warp, so it is kept in shared memory rather than in every lane's
// registers): the previous iterate p and bounds from the last octree
// search, carried to p by the triangle inequality:
// every point outside the kept k is at least out_lo away from p, the
// (k+1)-th nearest at most out_hi.
struct KnnCarry {
    double out_lo, out_hi;
    float px, py, pz;
    uint32_t searches;  // octree searches of this warp
};

__device__ __forceinline__ float kd_dist2(const float4 p, float qx, float qy, float qz)
{
    const float dx = __fsub_rn(p.x, qx), dy = __fsub_rn(p.y, qy), dz = __fsub_rn(p.z, qz);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ __forceinline__ bool key_less(float da, uint32_t oa, float db, uint32_t ob)
{
    return da < db || (da == db && oa < ob);
}

// Bitonic sort of one (d, o, p) per lane; ascending unless `desc`.
__device__ __forceinline__ void warp_sort(float& d, uint32_t& o, uint32_t& p, bool desc)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const float od = __shfl_xor_sync(kFull, d, j);
            const uint32_t oo = __shfl_xor_sync(kFull, o, j);
            const uint32_t op = __shfl_xor_sync(kFull, p, j);
            const bool up = (((lane & k) == 0) != desc);
            const bool lower = (lane & j) == 0;
            const bool other_less = key_less(od, oo, d, o);
            const bool take = (lower == up) ? other_less : (!other_less && (od != d || oo != o));
            if (take) {
                d = od;
                o = oo;
                p = op;
            }
        }
    }
}

// Ascending best list (d, o, p) merged with candidate batch (cd, co, cp).
// `lost` receives this lane's entry that left the union (the 32 largest of
// list and batch, one per lane): their minimum is the union's 33rd distance.
__device__ __forceinline__ void warp_merge(float& d, uint32_t& o, uint32_t& p, float cd, uint32_t co, uint32_t cp,
                                           float& lost)
{
    const int lane = threadIdx.x & 31;
    warp_sort(cd, co, cp, true);
    if (key_less(cd, co, d, o)) {
        lost = d;
        d = cd;
        o = co;
        p = cp;
    } else {
        lost = cd;
    }
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        const float od = __shfl_xor_sync(kFull, d, j);
        const uint32_t oo = __shfl_xor_sync(kFull, o, j);
        const uint32_t op = __shfl_xor_sync(kFull, p, j);
        const bool lower = (lane & j) == 0;
        const bool other_less = key_less(od, oo, d, o);
        if (lower ? other_less : (!other_less && (od != d || oo != o))) {
            d = od;
            o = oo;
            p = op;
        }
    }
}

__device__ __forceinline__ float warp_sum_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ float warp_max_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

__device__ __forceinline__ float warp_min_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

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

// Morton code of a world point on the tree's split lattice (the descent of
// the build, with the split recomputed from the float bound table).
__device__ uint64_t lattice_code(const GatherArgs& a, float wx, float wy, float wz)
{
    const float w[3] = {wx, wy, wz};
    uint32_t cell[3];
    for (int ax = 0; ax < 3; ++ax) {
        const float* B = a.bounds + ax * a.bounds_stride;
        const double x = double(w[ax]);
        uint32_t k = 0;
        for (int d = 0; d < a.max_depth; ++d) {
            const int64_t off = ((int64_t(1) << d) - 1) + d;
            const double s = (double(__ldg(B + off + k)) + double(__ldg(B + off + k + 1))) / 2.0;
            k = 2u * k + (x > s ? 1u : 0u);
        }
        cell[ax] = k;
    }
    uint64_t code = 0;
    for (int d = 0; d < a.max_depth; ++d) {
        const int b = a.max_depth - 1 - d;
        const uint64_t g = ((cell[0] >> b) & 1u) | (((cell[1] >> b) & 1u) << 1) | (((cell[2] >> b) & 1u) << 2);
        code |= g << (3 * b);
    }
    return code;
}

// First sorted position whose code is > qcode, found with 32-way splits.
__device__ int64_t warp_upper_bound(const uint64_t* __restrict__ codes, int64_t n, uint64_t qcode)
{
    const int lane = threadIdx.x & 31;
    int64_t lo = 0, hi = n;  // answer in [lo, hi]
    while (hi - lo > 32) {
        const int64_t step = (hi - lo) / 32;
        const int64_t idx = lo + step * lane;
        const bool le = __ldg(codes + idx) <= qcode;
        const uint32_t m = __ballot_sync(kFull, le);
        const int last = m ? 31 - __clz(m) : -1;  // last lane with code <= q
        if (last < 0) {
            hi = lo;
            break;
        }
        const int64_t nlo = lo + step * last + 1;
        const int64_t nhi = last == 31 ? hi : lo + step * (last + 1);
        lo = nlo;
        hi = nhi;
    }
    const int64_t idx = lo + lane;
    const bool le = idx < hi && __ldg(codes + idx) <= qcode;
    const uint32_t m = __ballot_sync(kFull, le);
    return lo + __popc(m);
}

template <int KTYPE>
__device__ __forceinline__ float weight_cpu(const KernelConsts& kc, float d2)
{
    float w = kernel_weight<KTYPE>(kc, d2);
    if (KTYPE == MLODS_GAUSSIAN_MULTIPLE && w == 0.f) w = kc.shift;  // Kernel.cpp:70-74
    return w;
}

// CPU-rule fit (CPUUtils.cpp:744-781) of the query-frame sums, in double.
__device__ bool fit_cpu(const float* s, double step_max, double x[3], float nrm[3])
{
    const double Sw = s[0];
    const double Sn[3] = {s[1], s[2], s[3]};
    const double Sp[3] = {s[4], s[5], s[6]};
    const double Spn = s[7], Spp = s[8];
    const double u4 = 0.5 * (Spn - (Sp[0] * Sn[0] + Sp[1] * Sn[1] + Sp[2] * Sn[2]) / Sw) /
                      (Spp - (Sp[0] * Sp[0] + Sp[1] * Sp[1] + Sp[2] * Sp[2]) / Sw);
    double u123[3];
    for (int c = 0; c < 3; ++c) u123[c] = (Sn[c] - 2.0 * u4 * Sp[c]) / Sw;
    const double u0 = -((Sp[0] * u123[0] + Sp[1] * u123[1] + Sp[2] * u123[2]) + u4 * Spp) / Sw;
    double nv[3];
    if (fabs(u4) < 1e-12) {
        const double m[3] = {-u123[0], -u123[1], -u123[2]};
        const double lambda = u0 / (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        for (int c = 0; c < 3; ++c) x[c] = lambda * m[c];
        for (int c = 0; c < 3; ++c) nv[c] = Sn[c];
    } else {
        double cc[3];
        for (int c = 0; c < 3; ++c) cc[c] = u123[c] / (-2.0 * u4);
        const double r2 = cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2] - u0 / u4;
        const double rad = sqrt(r2 > 0.0 ? r2 : 0.0);
        const double pl = sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
        for (int c = 0; c < 3; ++c) x[c] = cc[c] + rad * (-cc[c] / pl);
        for (int c = 0; c < 3; ++c) nv[c] = u123[c] + 2.0 * u4 * x[c];
    }
    const double nl = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    for (int c = 0; c < 3; ++c) nv[c] /= nl;
    if (isnan(x[0]) || isnan(x[1]) || isnan(x[2])) return false;
    const double step = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (step > step_max)
        for (int c = 0; c < 3; ++c) x[c] *= step_max / step;
    for (int c = 0; c < 3; ++c) nrm[c] = float(nv[c]);
    return true;
}

// MODE: 0 = kNN APSS projection, 1 = ball APSS projection, 2 = kNN sets only.
template <int KTYPE, int MODE>
__global__ void __launch_bounds__(kGatherThreads, MODE == 0 ? kKnnMinBlocks : kGatherMinBlocks) gather_kernel(GatherArgs a)
{
    __shared__ GStack stacks[kGatherThreads / 32];
    __shared__ KnnCarry carries[kGatherThreads / 32];
    const int lane = threadIdx.x & 31;
    GStack& st = stacks[threadIdx.x >> 5];
    KnnCarry& carry = carries[threadIdx.x >> 5];
    if (MODE == 0 && lane == 0) carry.searches = 0;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const int k = a.k;
    const double r2ball = double(a.ball_r) * double(a.ball_r);
    const int n_iter = MODE == 2 ? 1 : a.n_iter;
    int64_t overflows = 0;

    for (;;) {
        unsigned int qs = 0;
        if (lane == 0) qs = atomicAdd(a.counter, 1u);
        qs = __shfl_sync(kFull, qs, 0);
        if (int64_t(qs) >= a.nq) break;
        const int64_t qi = qs;
        const float q0[3] = {a.q_in[3 * qi], a.q_in[3 * qi + 1], a.q_in[3 * qi + 2]};
        double xd[3] = {double(q0[0]) - a.o0, double(q0[1]) - a.o1, double(q0[2]) - a.o2};
        float nrm[3] = {0.f, 0.f, 0.f};
        bool failed = false, empty = false, overflow = false;
        float best_d = INFINITY;
        uint32_t best_o = 0xFFFFFFFFu, best_p = 0xFFFFFFFFu;
        for (int it = 0; it < n_iter && !failed; ++it) {
            // the reference keeps the iterate as a float glm::vec3
            const float wx = it == 0 ? q0[0] : float(xd[0] + a.o0);
            const float wy = it == 0 ? q0[1] : float(xd[1] + a.o1);
            const float wz = it == 0 ? q0[2] : float(xd[2] + a.o2);
            const float lx = float(double(wx) - a.o0), ly = float(double(wy) - a.o1), lz = float(double(wz) - a.o2);
            float acc[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) acc[c] = 0.f;
            int found = 0;
            int64_t w0 = 0, w1 = 0;  // Morton window already in the best list
            // squared search radius: for the kNN projection an upper bound on
            // the (k+1)-th distance, so that the search also bounds the points
            // it leaves out; for the kNN sets the k-th
            float bound = INFINITY;
            bool search = true;
            float warm = INFINITY;  // kNN projection, iteration > 0: the search's starting bound
            if (MODE == 0 && it > 0) {
                const double ddx = double(wx) - double(carry.px), ddy = double(wy) - double(carry.py),
                             ddz = double(wz) - double(carry.pz);
                const double step = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
                const double out_lo = carry.out_lo, out_hi = carry.out_hi;
                __syncwarp();  // every lane has read the carry before lane 0 updates it
                // the previous (k+1)-th nearest point is at most out_hi + step away
                const double r = (out_hi + step) * (1.0 + 1e-5) + 1e-30;
                warm = __double2float_ru(r * r);
                if (__shfl_sync(kFull, best_p, k - 1) != 0xFFFFFFFFu) {
                    // the kept points' distances from the new iterate
                    if (lane < k) {
                        best_d = kd_dist2(__ldg(a.wspts + best_p), wx, wy, wz);
                    } else {
                        best_d = INFINITY;
                        best_o = best_p = 0xFFFFFFFFu;
                    }
                    const float dmax = warp_max_f(lane < k ? best_d : 0.f);
                    // Every other point is at least out_lo - step away: if all
                    // kept points are nearer (margins of 1e-5 cover the float
                    // distances), a search would return the same k points, so
                    // they are only ranked again.
                    if (sqrt(double(dmax)) * (1.0 + 1e-5) < (out_lo - step) * (1.0 - 1e-5)) {
                        search = false;
                        // after a short step they are mostly still in order
                        const float dn = __shfl_down_sync(kFull, best_d, 1);
                        const uint32_t on = __shfl_down_sync(kFull, best_o, 1);
                        if (__any_sync(kFull, lane < k - 1 && key_less(dn, on, best_d, best_o)))
                            warp_sort(best_d, best_o, best_p, false);
                        if (lane == 0) {
                            carry.out_lo = out_lo - step;
                            carry.out_hi = out_hi + step;
                        }
                    } else if (a.n_pts > k) {
                        // the kept k and one other point bound the (k+1)-th
                        // distance: the first sorted position after the
                        // nearest kept point's that none of them holds
                        uint32_t c = __shfl_sync(kFull, best_p, 0), xp = 0xFFFFFFFFu;
                        for (int t = 0; t <= k; ++t) {
                            c = c + 1u == uint32_t(a.n_pts) ? 0u : c + 1u;
                            if (!__any_sync(kFull, lane < k && best_p == c)) {
                                xp = c;
                                break;
                            }
                        }
                        if (xp != 0xFFFFFFFFu)
                            warm = fminf(warm, fmaxf(dmax, kd_dist2(__ldg(a.wspts + xp), wx, wy, wz)));
                    }
                }
            }
            if (search) {
                best_d = INFINITY;
                best_o = best_p = 0xFFFFFFFFu;
                if (MODE == 0 && it > 0 && warm < INFINITY) {
                    bound = warm;
                } else if (MODE != 1) {
                    const uint64_t qc = lattice_code(a, wx, wy, wz);
                    const int64_t pos = warp_upper_bound(a.codes, a.n_pts, qc);
                    w0 = pos - 16 < 0 ? 0 : pos - 16;
                    w1 = w0 + 32 > a.n_pts ? a.n_pts : w0 + 32;
                    w0 = w1 - 32 < 0 ? 0 : w1 - 32;
                    const int64_t j = w0 + lane;
                    if (j < w1) {
                        const float4 p = __ldg(a.wspts + j);
                        best_d = kd_dist2(p, wx, wy, wz);
                        best_o = __float_as_uint(p.w);
                        best_p = uint32_t(j);
                    }
                    warp_sort(best_d, best_o, best_p, false);
                    if (MODE == 0 && k == 32) {
                        // a 33rd point beside the window bounds the 33rd distance
                        const int64_t xp = w1 < a.n_pts ? w1 : w0 - 1;
                        const float xd2 = xp >= 0 ? kd_dist2(__ldg(a.wspts + xp), wx, wy, wz) : INFINITY;
                        bound = fmaxf(__shfl_sync(kFull, best_d, 31), xd2);
                    } else {
                        bound = __shfl_sync(kFull, best_d, MODE == 0 ? k : k - 1);
                    }
                } else {
                    bound = float(r2ball) * (1.f + 1e-6f);
                }
            }
            // ---- octree walk
            int top = search ? 1 : 0;
            if (lane == 0 && search) {
                st.first[0] = 0;
                st.cnt[0] = 1u;
            }
            __syncwarp();
            while (top > 0) {
                uint32_t e_first = 0, e_cnt = 0;
                int c = 0;
                if (lane < top) {
                    e_first = st.first[top - 1 - lane];
                    e_cnt = st.cnt[top - 1 - lane];
                    c = int(e_cnt & kGCount);
                }
                const int incl = warp_incl_scan_i(c);
                const int pop_lanes = top > kBatchPopLimit ? 1 : top;  // depth-first near the cap
                const uint32_t fit = __ballot_sync(kFull, lane < pop_lanes && incl <= 32);
                int npop = __popc(fit);
                const bool partial = npop == 0;
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
                const int r_start = partial ? 0 : __shfl_sync(kFull, incl - c, e);
                if (partial) {
                    if (lane == 0) {
                        st.first[top - 1] = e_first + 32u;
                        st.cnt[top - 1] = e_cnt - 32u;
                    }
                } else {
                    top -= npop;
                }
                const uint32_t idx = r_first + uint32_t(lane - r_start);
                // candidate point of this lane (sorted position), if any
                int64_t cpos = -1;
                bool push = false;
                uint32_t p_first = 0, p_cnt = 0;
                if (active) {
                    if (r_cnt & kGPoints) {
                        cpos = idx;
                    } else {
                        const float4 g4 = __ldg(a.nodes.geom + idx);
                        const float4 x4 = __ldg(a.nodes.aux + idx);
                        const uint32_t info = __float_as_uint(x4.z);
                        if (info & kLeafBit) {
                            const int cnt = int(node_count(info));
                            const int64_t head = __ldg(a.node_head + idx);
                            if (cnt == 1) {
                                cpos = head;
                            } else {
                                push = true;
                                p_first = uint32_t(head);
                                p_cnt = uint32_t(cnt) | kGPoints;
                            }
                        } else {
                            const float cx = g4.x - lx, cy = g4.y - ly, cz = g4.z - lz;
                            const float dc = sqrtf(cx * cx + cy * cy + cz * cz);
                            const float lo = dc - g4.w - a.eps;
                            if (!(lo > 0.f && lo * lo > bound)) {
                                push = true;
                                p_first = __float_as_uint(x4.y);
                                p_cnt = node_count(info);
                            }
                        }
                    }
                }
                float cd = INFINITY;
                uint32_t co = 0xFFFFFFFFu, cp = 0xFFFFFFFFu;
                if (cpos >= 0 && !(MODE != 1 && cpos >= w0 && cpos < w1)) {
                    const float4 p = __ldg(a.wspts + cpos);
                    const float d2 = kd_dist2(p, wx, wy, wz);
                    if (MODE == 1) {
                        if (double(d2) <= r2ball) {
                            const float4 pl = __ldg(a.spts + cpos);
                            const float4 nn = __ldg(a.snrm + cpos);
                            const float dx = pl.x - lx, dy = pl.y - ly, dz = pl.z - lz;
                            const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            const float w = weight_cpu<KTYPE>(a.kc, dd);
                            acc[0] += w;
                            acc[1] = fmaf(w, nn.x, acc[1]);
                            acc[2] = fmaf(w, nn.y, acc[2]);
                            acc[3] = fmaf(w, nn.z, acc[3]);
                            acc[4] = fmaf(w, dx, acc[4]);
                            acc[5] = fmaf(w, dy, acc[5]);
                            acc[6] = fmaf(w, dz, acc[6]);
                            acc[7] = fmaf(w, fmaf(dx, nn.x, fmaf(dy, nn.y, dz * nn.z)), acc[7]);
                            acc[8] = fmaf(w, dd, acc[8]);
                            ++found;
                        }
                    } else if (d2 <= bound) {
                        cd = d2;
                        co = __float_as_uint(p.w);
                        cp = uint32_t(cpos);
                    }
                }
                if (MODE != 1) {
                    if (__any_sync(kFull, cd <= bound && cd < INFINITY)) {
                        float lost = INFINITY;
                        warp_merge(best_d, best_o, best_p, cd, co, cp, lost);
                        // the (k+1)-th (kNN projection) or k-th distance so far
                        if (MODE == 0 && k == 32)
                            bound = fminf(bound, warp_min_f(lost));
                        else
                            bound = fminf(bound, __shfl_sync(kFull, best_d, MODE == 0 ? k : k - 1));
                    }
                }
                const uint32_t pm = __ballot_sync(kFull, push);
                const int npush = __popc(pm);
                if (top + npush > kGatherCap) {
                    overflow = true;
                } else {
                    if (push) {
                        const int pos = top + __popc(pm & lt_mask);
                        st.first[pos] = p_first;
                        st.cnt[pos] = p_cnt;
                    }
                    top += npush;
                }
                __syncwarp();
            }
            if (overflow) {
                failed = true;
                break;
            }
            if (MODE == 2) break;
            if (MODE == 0) {
                if (lane == 0) {
                    carry.px = wx;
                    carry.py = wy;
                    carry.pz = wz;
                    if (search) {
                        // every point left out is at least sqrt(bound) away
                        // (it was pruned, rejected or ranked beyond the k-th
                        // against a bound no smaller than the final one), and
                        // the (k+1)-th nearest at most: bound never fell below it
                        const double lb = sqrt(double(bound));
                        carry.out_lo = lb * (1.0 - 1e-5);
                        carry.out_hi = lb * (1.0 + 1e-5);
                        ++carry.searches;
                    }
                }
                __syncwarp();
                if (lane < k && best_p != 0xFFFFFFFFu) {
                    const float4 pl = __ldg(a.spts + best_p);
                    const float4 nn = __ldg(a.snrm + best_p);
                    const float dx = pl.x - lx, dy = pl.y - ly, dz = pl.z - lz;
                    const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    const float w = weight_cpu<KTYPE>(a.kc, dd);
                    acc[0] = w;
                    acc[1] = w * nn.x;
                    acc[2] = w * nn.y;
                    acc[3] = w * nn.z;
                    acc[4] = w * dx;
                    acc[5] = w * dy;
                    acc[6] = w * dz;
                    acc[7] = w * fmaf(dx, nn.x, fmaf(dy, nn.y, dz * nn.z));
                    acc[8] = w * dd;
                }
            } else {
                // CPUUtils.cpp:711-716: an empty ball returns the start point, normal 0
                const int tot = __reduce_add_sync(kFull, found);
                if (tot == 0) {
                    empty = true;
                    failed = true;
                    break;
                }
            }
            float s[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) s[c] = warp_sum_f(acc[c]);
            double x[3];
            if (!fit_cpu(s, double(a.step_max), x, nrm)) {
                // NaN: the iterate stays, normal 0 (CPUUtils.cpp:770-776)
                nrm[0] = nrm[1] = nrm[2] = 0.f;
                xd[0] = double(wx) - a.o0;
                xd[1] = double(wy) - a.o1;
                xd[2] = double(wz) - a.o2;
                continue;
            }
            xd[0] = double(lx) + x[0];
            xd[1] = double(ly) + x[1];
            xd[2] = double(lz) + x[2];
        }
        if (MODE == 2) {
            if (lane < k) {
                const bool ok = best_p != 0xFFFFFFFFu && !overflow;
                a.out_idx[qi * k + lane] = ok ? int32_t(best_o) : -1;
                a.out_d2[qi * k + lane] = ok ? best_d : -1.f;
            }
        } else if (lane == 0) {
            float* op = a.out_p + 3 * qi;
            float* on = a.out_n + 3 * qi;
            if (empty || overflow) {
                op[0] = q0[0];
                op[1] = q0[1];
                op[2] = q0[2];
                on[0] = on[1] = on[2] = 0.f;
            } else {
                op[0] = float(xd[0] + a.o0);
                op[1] = float(xd[1] + a.o1);
                op[2] = float(xd[2] + a.o2);
                on[0] = nrm[0];
                on[1] = nrm[1];
                on[2] = nrm[2];
            }
        }
        if (overflow) ++overflows;
    }
    if (lane == 0 && a.stats && overflows)
        atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[2]), (unsigned long long)overflows);
    if (MODE == 0 && lane == 0 && a.stats && carry.searches)
        atomicAdd(reinterpret_cast<unsigned long long*>(&a.stats[5]), (unsigned long long)carry.searches);
}

// ---------------------------------------------------------------- global APSS

#ifndef MLODS_GLOBAL_MIN_BLOCKS
#define MLODS_GLOBAL_MIN_BLOCKS 0
#endif
constexpr int kGlobalThreads = 128;
#if MLODS_GLOBAL_MIN_BLOCKS > 0
#define MLODS_GLOBAL_BOUNDS __launch_bounds__(kGlobalThreads, MLODS_GLOBAL_MIN_BLOCKS)
#else
#define MLODS_GLOBAL_BOUNDS __launch_bounds__(kGlobalThreads)
#endif
constexpr int kGlobalTile = 256;  // points per shared-memory tile
constexpr int kGlobalQpt = 2;     // queries per thread: each point read from shared memory serves two

// Weight of the CPU path (Kernel::w, Kernel.cpp:51-76) with the number of
// multi-Gaussian terms fixed at compile time when NSIG > 0.
template <int KTYPE, int NSIG>
__device__ __forceinline__ float global_weight(const KernelConsts& kc, float d2)
{
    float w;
    if (KTYPE == MLODS_GAUSSIAN_MULTIPLE && NSIG > 0) {
        w = 0.f;
#pragma unroll
        for (int i = 0; i < NSIG; ++i) w = fmaf(exp2f(d2 * kc.ms_scale[i]), kc.ms_w[i], w);
    } else {
        w = kernel_weight<KTYPE>(kc, d2);
    }
    if (KTYPE == MLODS_GAUSSIAN_MULTIPLE && w == 0.f) w = kc.shift;  // Kernel.cpp:70-74
    return w;
}

// Sums over the points [p_begin, p_end) for the kGlobalQpt = 2 queries of a
// thread (local-frame float positions lx, ly, lz): every point contributes
// w(p_i, q) a_i {1, n_i, p_i - q, (p_i - q).n_i, |p_i - q|^2}
// (APSSOctree::APSSStats, CPUUtils.cpp:515-528).  Points stream through
// shared memory in tiles, each value stored twice ({v, v}), so that one
// packed f32x2 instruction (sm_100) does the arithmetic of both queries:
// the same roundings, in the same order, as two scalar instructions.  Per-
// tile float partial sums are added to `tot` in double.  Every thread of the
// block calls it (it synchronises the block).
template <int KTYPE, int NSIG>
__device__ __forceinline__ void global_pair_sums(const GlobalArgs& a, int64_t p_begin, int64_t p_end,
                                                 const float (&lx)[kGlobalQpt], const float (&ly)[kGlobalQpt],
                                                 const float (&lz)[kGlobalQpt], double (&tot)[kGlobalQpt][9],
                                                 float4* s_pd, float4* s_nd)
{
    static_assert(kGlobalQpt == 2, "the packed pair sums serve two queries per thread");
    // p - q as p + (-q): the same rounding as the subtraction
    const float2 mqx = make_float2(-lx[0], -lx[1]), mqy = make_float2(-ly[0], -ly[1]),
                 mqz = make_float2(-lz[0], -lz[1]);
    for (int64_t base = p_begin; base < p_end; base += kGlobalTile) {
        __syncthreads();
        for (int j = threadIdx.x; j < kGlobalTile; j += kGlobalThreads) {
            const int64_t g = base + j;
            if (g < p_end) {
                const float4 p = __ldg(a.spts + g);
                const float4 nn = __ldg(a.snrm + g);
                const float ar = __ldg(a.area + __float_as_uint(p.w));
                s_pd[2 * j] = make_float4(p.x, p.x, p.y, p.y);
                s_pd[2 * j + 1] = make_float4(p.z, p.z, ar, ar);
                s_nd[2 * j] = make_float4(nn.x, nn.x, nn.y, nn.y);
                s_nd[2 * j + 1] = make_float4(nn.z, nn.z, 0.f, 0.f);
            } else {  // zero area: no contribution
                s_pd[2 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
                s_pd[2 * j + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
                s_nd[2 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
                s_nd[2 * j + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        __syncthreads();
        float2 acc[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) acc[c] = make_float2(0.f, 0.f);
#pragma unroll 2
        for (int j = 0; j < kGlobalTile; ++j) {
            const float4 pa = s_pd[2 * j], pb = s_pd[2 * j + 1];
            const float4 na = s_nd[2 * j], nb = s_nd[2 * j + 1];
            const float2 nx = make_float2(na.x, na.y), ny = make_float2(na.z, na.w), nz = make_float2(nb.x, nb.y);
            const float2 dx = __fadd2_rn(make_float2(pa.x, pa.y), mqx);
            const float2 dy = __fadd2_rn(make_float2(pa.z, pa.w), mqy);
            const float2 dz = __fadd2_rn(make_float2(pb.x, pb.y), mqz);
            const float2 dd = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            float2 w;
            if (KTYPE == MLODS_GAUSSIAN_MULTIPLE && NSIG > 0) {
                w = make_float2(0.f, 0.f);
#pragma unroll
                for (int i = 0; i < NSIG; ++i) {
                    const float2 t = __fmul2_rn(dd, make_float2(a.kc.ms_scale[i], a.kc.ms_scale[i]));
                    const float2 e = make_float2(exp2f(t.x), exp2f(t.y));
                    w = __ffma2_rn(e, make_float2(a.kc.ms_w[i], a.kc.ms_w[i]), w);
                }
                if (w.x == 0.f) w.x = a.kc.shift;  // Kernel.cpp:70-74
                if (w.y == 0.f) w.y = a.kc.shift;
            } else {
                w = make_float2(global_weight<KTYPE, NSIG>(a.kc, dd.x), global_weight<KTYPE, NSIG>(a.kc, dd.y));
            }
            w = __fmul2_rn(w, make_float2(pb.z, pb.w));
            acc[0] = __fadd2_rn(acc[0], w);
            acc[1] = __ffma2_rn(w, nx, acc[1]);
            acc[2] = __ffma2_rn(w, ny, acc[2]);
            acc[3] = __ffma2_rn(w, nz, acc[3]);
            acc[4] = __ffma2_rn(w, dx, acc[4]);
            acc[5] = __ffma2_rn(w, dy, acc[5]);
            acc[6] = __ffma2_rn(w, dz, acc[6]);
            acc[7] = __ffma2_rn(w, __ffma2_rn(dx, nx, __ffma2_rn(dy, ny, __fmul2_rn(dz, nz))), acc[7]);
            acc[8] = __ffma2_rn(w, dd, acc[8]);
        }
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            tot[0][c] += double(acc[c].x);
            tot[1][c] += double(acc[c].y);
        }
    }
}

// One fit step of a query from its sums: false (iterate kept, normal 0) when
// the fit is NaN (CPUUtils.cpp:770-776).
__device__ __forceinline__ bool global_step(const GlobalArgs& a, const double (&tot)[9], float lx, float ly, float lz,
                                            double xd[3], float nrm[3])
{
    float s[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) s[c] = float(tot[c]);
    double x[3];
    if (!fit_cpu(s, double(a.step_max), x, nrm)) {
        nrm[0] = nrm[1] = nrm[2] = 0.f;
        return false;
    }
    xd[0] = double(lx) + x[0];
    xd[1] = double(ly) + x[1];
    xd[2] = double(lz) + x[2];
    return true;
}

// All iterations of kGlobalQpt queries per thread in one launch, every point
// per iteration: the form for query counts that fill the GPU.
template <int KTYPE, int NSIG>
__global__ void MLODS_GLOBAL_BOUNDS global_apss_kernel(GlobalArgs a)
{
    constexpr int Q = kGlobalQpt;
    __shared__ float4 s_pd[2 * kGlobalTile];
    __shared__ float4 s_nd[2 * kGlobalTile];
    const int64_t q_first = int64_t(blockIdx.x) * kGlobalThreads * Q + threadIdx.x;
    double xd[Q][3];
    float nrm[Q][3];
    bool valid[Q], failed[Q];
#pragma unroll
    for (int u = 0; u < Q; ++u) {
        const int64_t qi = q_first + int64_t(u) * kGlobalThreads;
        valid[u] = qi < a.nq;
        failed[u] = false;
        const double o[3] = {a.o0, a.o1, a.o2};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            xd[u][c] = valid[u] ? double(a.q_in[3 * qi + c]) - o[c] : 0.0;
            nrm[u][c] = 0.f;
        }
    }
    for (int it = 0; it < a.n_iter; ++it) {
        float lx[Q], ly[Q], lz[Q];
        double tot[Q][9];
#pragma unroll
        for (int u = 0; u < Q; ++u) {
            lx[u] = float(xd[u][0]);
            ly[u] = float(xd[u][1]);
            lz[u] = float(xd[u][2]);
#pragma unroll
            for (int c = 0; c < 9; ++c) tot[u][c] = 0.0;
        }
        global_pair_sums<KTYPE, NSIG>(a, 0, a.n_pts, lx, ly, lz, tot, s_pd, s_nd);
#pragma unroll
        for (int u = 0; u < Q; ++u) {
            if (!valid[u] || failed[u]) continue;
            if (!global_step(a, tot[u], lx[u], ly[u], lz[u], xd[u], nrm[u])) failed[u] = true;
        }
    }
#pragma unroll
    for (int u = 0; u < Q; ++u) {
        if (!valid[u]) continue;
        const int64_t qi = q_first + int64_t(u) * kGlobalThreads;
        a.out_p[3 * qi] = float(xd[u][0] + a.o0);
        a.out_p[3 * qi + 1] = float(xd[u][1] + a.o1);
        a.out_p[3 * qi + 2] = float(xd[u][2] + a.o2);
        a.out_n[3 * qi] = nrm[u][0];
        a.out_n[3 * qi + 1] = nrm[u][1];
        a.out_n[3 * qi + 2] = nrm[u][2];
    }
}

// The split form, for query counts too small to fill the GPU: the points are
// cut into `chunks` ranges, block (x, y) sums query tile x against range y
// and writes its double sums to part[(y * nq + q) * 9 + c]; then one thread
// per query adds the ranges in order, fits, and moves the iterate.  One such
// pair of launches per iteration.
struct GlobalSplit {
    double* part;     // chunks * nq * 9
    double* xd;       // nq * 3, the iterate in the local frame
    float* nrm;       // nq * 3
    uint32_t* failed; // nq
    int chunks;
    int64_t chunk_pts;
};

__global__ void global_split_init_kernel(GlobalArgs a, GlobalSplit g)
{
    const int64_t qi = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (qi >= a.nq) return;
    const double o[3] = {a.o0, a.o1, a.o2};
    for (int c = 0; c < 3; ++c) {
        g.xd[3 * qi + c] = double(a.q_in[3 * qi + c]) - o[c];
        g.nrm[3 * qi + c] = 0.f;
    }
    g.failed[qi] = 0u;
}

template <int KTYPE, int NSIG>
__global__ void MLODS_GLOBAL_BOUNDS global_split_sums_kernel(GlobalArgs a, GlobalSplit g)
{
    constexpr int Q = kGlobalQpt;
    __shared__ float4 s_pd[2 * kGlobalTile];
    __shared__ float4 s_nd[2 * kGlobalTile];
    const int64_t q_first = int64_t(blockIdx.x) * kGlobalThreads * Q + threadIdx.x;
    const int64_t p_begin = int64_t(blockIdx.y) * g.chunk_pts;
    const int64_t p_end = p_begin + g.chunk_pts < a.n_pts ? p_begin + g.chunk_pts : a.n_pts;
    float lx[Q], ly[Q], lz[Q];
    double tot[Q][9];
#pragma unroll
    for (int u = 0; u < Q; ++u) {
        const int64_t qi = q_first + int64_t(u) * kGlobalThreads;
        const bool valid = qi < a.nq;
        lx[u] = valid ? float(g.xd[3 * qi]) : 0.f;
        ly[u] = valid ? float(g.xd[3 * qi + 1]) : 0.f;
        lz[u] = valid ? float(g.xd[3 * qi + 2]) : 0.f;
#pragma unroll
        for (int c = 0; c < 9; ++c) tot[u][c] = 0.0;
    }
    global_pair_sums<KTYPE, NSIG>(a, p_begin, p_end, lx, ly, lz, tot, s_pd, s_nd);
#pragma unroll
    for (int u = 0; u < Q; ++u) {
        const int64_t qi = q_first + int64_t(u) * kGlobalThreads;
        if (qi >= a.nq) continue;
        double* dst = g.part + (int64_t(blockIdx.y) * a.nq + qi) * 9;
#pragma unroll
        for (int c = 0; c < 9; ++c) dst[c] = tot[u][c];
    }
}

__global__ void global_split_step_kernel(GlobalArgs a, GlobalSplit g, bool last)
{
    const int64_t qi = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (qi >= a.nq) return;
    double xd[3] = {g.xd[3 * qi], g.xd[3 * qi + 1], g.xd[3 * qi + 2]};
    float nrm[3] = {g.nrm[3 * qi], g.nrm[3 * qi + 1], g.nrm[3 * qi + 2]};
    if (!g.failed[qi]) {
        double tot[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < g.chunks; ++k) {
            const double* src = g.part + (int64_t(k) * a.nq + qi) * 9;
#pragma unroll
            for (int c = 0; c < 9; ++c) tot[c] += src[c];
        }
        const float lx = float(xd[0]), ly = float(xd[1]), lz = float(xd[2]);
        if (!global_step(a, tot, lx, ly, lz, xd, nrm)) g.failed[qi] = 1u;
        for (int c = 0; c < 3; ++c) {
            g.xd[3 * qi + c] = xd[c];
            g.nrm[3 * qi + c] = nrm[c];
        }
    }
    if (last) {
        a.out_p[3 * qi] = float(xd[0] + a.o0);
        a.out_p[3 * qi + 1] = float(xd[1] + a.o1);
        a.out_p[3 * qi + 2] = float(xd[2] + a.o2);
        a.out_n[3 * qi] = nrm[0];
        a.out_n[3 * qi + 1] = nrm[1];
        a.out_n[3 * qi + 2] = nrm[2];
    }
}

// Launches the global projection of one kernel specialisation: the fused
// kernel when the query tiles fill the GPU about four times over, else the
// split form over as many point ranges as bring it there.
template <int KTYPE, int NSIG>
cudaError_t launch_global_typed(const GlobalArgs& a, int sm_count, cudaStream_t s)
{
    const int64_t per_block = int64_t(kGlobalThreads) * kGlobalQpt;
    const int64_t qblocks = (a.nq + per_block - 1) / per_block;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, global_apss_kernel<KTYPE, NSIG>,
                                                                  kGlobalThreads, 0);
    if (e != cudaSuccess) return e;
    const int64_t target = 4 * int64_t(per_sm < 1 ? 1 : per_sm) * sm_count;
    int64_t chunks = (target + qblocks - 1) / qblocks;
    const int64_t max_chunks = a.n_pts / (8 * kGlobalTile);  // ranges of at least 2048 points
    if (chunks > max_chunks) chunks = max_chunks;
    if (chunks > 64) chunks = 64;
    if (chunks <= 1 || a.n_iter < 1) {
        global_apss_kernel<KTYPE, NSIG><<<unsigned(qblocks), kGlobalThreads, 0, s>>>(a);
        note_launch();
        return cudaGetLastError();
    }
    GlobalSplit g;
    g.chunks = int(chunks);
    g.chunk_pts = (a.n_pts + chunks - 1) / chunks;
    const size_t part_bytes = size_t(chunks) * size_t(a.nq) * 9 * sizeof(double);
    const size_t state_bytes = size_t(a.nq) * (3 * sizeof(double) + 3 * sizeof(float) + sizeof(uint32_t));
    void* mem = nullptr;
    e = scratch_alloc(&mem, part_bytes + state_bytes + 256, s);
    if (e != cudaSuccess) return e;
    char* m = static_cast<char*>(mem);
    g.part = reinterpret_cast<double*>(m);
    g.xd = reinterpret_cast<double*>(m + part_bytes);
    g.nrm = reinterpret_cast<float*>(m + part_bytes + size_t(a.nq) * 3 * sizeof(double));
    g.failed = reinterpret_cast<uint32_t*>(m + part_bytes + size_t(a.nq) * (3 * sizeof(double) + 3 * sizeof(float)));
    const unsigned q_threads = 256;
    const unsigned q_grid = unsigned((a.nq + q_threads - 1) / q_threads);
    global_split_init_kernel<<<q_grid, q_threads, 0, s>>>(a, g);
    note_launch();
    for (int it = 0; it < a.n_iter && e == cudaSuccess; ++it) {
        global_split_sums_kernel<KTYPE, NSIG><<<dim3(unsigned(qblocks), unsigned(chunks)), kGlobalThreads, 0, s>>>(a, g);
        global_split_step_kernel<<<q_grid, q_threads, 0, s>>>(a, g, it + 1 == a.n_iter);
        note_launch(2);
        e = cudaGetLastError();
    }
    const cudaError_t ef = scratch_free(mem, s);
    return e != cudaSuccess ? e : ef;
}

template <int KTYPE, int MODE>
cudaError_t launch_gather_typed(const GatherArgs& a, int sm_count, cudaStream_t s)
{
    auto kern = gather_kernel<KTYPE, MODE>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGatherThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int64_t want = (a.nq + kGatherThreads / 32 - 1) / (kGatherThreads / 32);
    int64_t grid = int64_t(per_sm) * sm_count;
    if (grid > want) grid = want;
    if (grid < 1) grid = 1;
    kern<<<unsigned(grid), kGatherThreads, 0, s>>>(a);
    note_launch();
    return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_gather_mode(const GatherArgs& a, int ktype, int sm_count, cudaStream_t s)
{
    switch (ktype) {
    case MLODS_GAUSSIAN: return launch_gather_typed<MLODS_GAUSSIAN, MODE>(a, sm_count, s);
    case MLODS_SINGULAR: return launch_gather_typed<MLODS_SINGULAR, MODE>(a, sm_count, s);
    default: return launch_gather_typed<MLODS_GAUSSIAN_MULTIPLE, MODE>(a, sm_count, s);
    }
}

}  // namespace

cudaError_t launch_gather(const GatherArgs& a, int mode, int ktype, int sm_count, cudaStream_t s)
{
    if (mode == kGatherKnnApss) return launch_gather_mode<0>(a, ktype, sm_count, s);
    if (mode == kGatherBallApss) return launch_gather_mode<1>(a, ktype, sm_count, s);
    return launch_gather_mode<2>(a, ktype, sm_count, s);
}

cudaError_t launch_global_apss(const GlobalArgs& a, int ktype, cudaStream_t s)
{
    const int sm = sm_count_for_current_device();
    switch (ktype) {
    case MLODS_GAUSSIAN: return launch_global_typed<MLODS_GAUSSIAN, 0>(a, sm, s);
    case MLODS_SINGULAR: return launch_global_typed<MLODS_SINGULAR, 0>(a, sm, s);
    default:
        switch (a.kc.nsig) {
        case 1: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 1>(a, sm, s);
        case 2: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 2>(a, sm, s);
        case 3: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 3>(a, sm, s);
        case 4: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 4>(a, sm, s);
        case 5: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 5>(a, sm, s);
        case 6: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 6>(a, sm, s);
        case 8: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 8>(a, sm, s);
        default: return launch_global_typed<MLODS_GAUSSIAN_MULTIPLE, 0>(a, sm, s);
        }
    }
}

}  // namespace mlods
