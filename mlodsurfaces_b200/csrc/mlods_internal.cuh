// mlods_internal.cuh -- device data layout and helpers shared by the kernels.
//
// Layout in HBM (one tree):
//   DNode nodes[n_nodes + n_extra]   64-byte records, breadth-first order of the
//                                    reference octree (CPUUtils.cpp:601-619),
//                                    followed by one record per point of every
//                                    multi-point leaf (leaves at max depth).
//   Everything is stored in a cloud-local frame: world = origin + local, with
//   origin (double) the centre of the root box.  Far-from-origin clouds keep
//   full float precision this way.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mlods.h"

namespace mlods
{

// Node info word: bits 0-19 child (or point) count, bits 20-24 depth,
// bit 28 leaf, bit 29 multi-point leaf.
constexpr uint32_t kCountMask = 0xFFFFFu;
constexpr int kDepthShift = 20;
constexpr uint32_t kDepthMask = 0x1Fu;
constexpr uint32_t kLeafBit = 1u << 28;
constexpr uint32_t kMultiBit = 1u << 29;
constexpr int kMaxTreeDepth = 12;  // MAX_DEPTH, CPUUtils.h:20

// One octree node (or one point of a multi-point leaf).  Moments are centred
// on the node centroid pbar:
//   m0  = sum a_i                      n   = sum a_i n_i
//   cpn = sum a_i (p_i - pbar).n_i     cpp = sum a_i |p_i - pbar|^2
// which is the reference's {s_ai, s_ai_ni, s_ai_pi, s_ai_pi_ni, s_ai_pi_pi}
// (CPUUtils.h:29-49) rewritten so that no term grows with the distance to the
// origin: s_ai_pi = m0 pbar, s_ai_pi_ni = cpn + pbar.n, s_ai_pi_pi = cpp + m0 |pbar|^2.
struct __align__(16) DNode {
    float cx, cy, cz, r;       // box centre, half box diagonal (BBOX::radius, CPUUtils.h:85)
    float px, py, pz, m0;      // centroid, mass
    float nx, ny, nz, cpn;     // weighted normal sum, centred p.n moment
    float cpp;                 // centred |p|^2 moment
    uint32_t first;            // first child / first point record
    uint32_t info;             // count, depth, flags
    uint32_t parent;           // parent index (0xFFFFFFFF for the root)
};
static_assert(sizeof(DNode) == 64, "DNode must stay 64 bytes");

// The nodes live in HBM as four float4 arrays (structure of arrays), so that
// the loads of one sibling range are contiguous per array:
//   geom[i] = {cx, cy, cz, r}      pm[i] = {px, py, pz, m0}
//   nc[i]   = {nx, ny, nz, cpn}    aux[i] = {cpp, first, info, parent}
struct NodeArrays {
    float4* geom;
    float4* pm;
    float4* nc;
    float4* aux;
};

__device__ inline void store_node(const NodeArrays& a, int64_t i, const DNode& n)
{
    a.geom[i] = make_float4(n.cx, n.cy, n.cz, n.r);
    a.pm[i] = make_float4(n.px, n.py, n.pz, n.m0);
    a.nc[i] = make_float4(n.nx, n.ny, n.nz, n.cpn);
    float4 x;
    x.x = n.cpp;
    x.y = __uint_as_float(n.first);
    x.z = __uint_as_float(n.info);
    x.w = __uint_as_float(n.parent);
    a.aux[i] = x;
}

__device__ inline DNode load_node_all(const NodeArrays& a, int64_t i)
{
    const float4 g = a.geom[i], p = a.pm[i], c = a.nc[i], x = a.aux[i];
    DNode n;
    n.cx = g.x; n.cy = g.y; n.cz = g.z; n.r = g.w;
    n.px = p.x; n.py = p.y; n.pz = p.z; n.m0 = p.w;
    n.nx = c.x; n.ny = c.y; n.nz = c.z; n.cpn = c.w;
    n.cpp = x.x;
    n.first = __float_as_uint(x.y);
    n.info = __float_as_uint(x.z);
    n.parent = __float_as_uint(x.w);
    return n;
}

__host__ __device__ inline uint32_t node_count(uint32_t info) { return info & kCountMask; }
__host__ __device__ inline int node_depth(uint32_t info) { return int((info >> kDepthShift) & kDepthMask); }

// Weight kernel constants, derived on the host from mlods_kernel.
struct KernelConsts {
    int type;          // MLODS_GAUSSIAN, MLODS_SINGULAR, MLODS_GAUSSIAN_MULTIPLE
    int nsig;
    float shift;       // constant_shift
    float exponent;
    float g_scale;     // gaussian: -log2(e) / (2 sigma^2)
    float num;         // singular: max(shift, 1e-4)^exponent
    float ms_scale[MLODS_INLINE_SIGMAS];  // multi: -log2(e) / (2 sigma_i^2)
    float ms_w[MLODS_INLINE_SIGMAS];      // multi: 1 / sigma_i^3
    // multi-Gaussian kernels with more than MLODS_INLINE_SIGMAS terms: all
    // nsig pairs {ms_scale_i, ms_w_i} in device memory (a table the library
    // keeps for the life of the process, shared by every kernel with the
    // same sigmas); nullptr otherwise
    const float2* ms_ext;
};

// Fills the constants of a validated kernel.  A multi-Gaussian kernel with
// more than MLODS_INLINE_SIGMAS terms gets its device table on the current
// device (allocated on first use of that sigma list).
int make_kernel_consts(const mlods_kernel& k, KernelConsts* out);
// Checks a kernel as mlods_set_kernel does; sets the error message.
int validate_kernel(const mlods_kernel* k);

// Weight as a function of the squared distance (Kernel::w, Kernel.cpp:64-83;
// KernelGPU::w, GPUUtils.cu:243-257).
template <int KTYPE>
__device__ __forceinline__ float kernel_weight(const KernelConsts& kc, float d2)
{
    if (KTYPE == MLODS_GAUSSIAN) {
        return exp2f(d2 * kc.g_scale) + kc.shift;
    } else if (KTYPE == MLODS_GAUSSIAN_MULTIPLE) {
        float s = 0.f;
        if (kc.nsig <= MLODS_INLINE_SIGMAS) {
            for (int i = 0; i < kc.nsig; ++i) s = fmaf(exp2f(d2 * kc.ms_scale[i]), kc.ms_w[i], s);
        } else {
            for (int i = 0; i < kc.nsig; ++i) {
                const float2 t = __ldg(kc.ms_ext + i);
                s = fmaf(exp2f(d2 * t.x), t.y, s);
            }
        }
        return s;
    } else {
        return kc.num * exp2f(-kc.exponent * __log2f(d2 + kc.shift));
    }
}

// Counts kernel launches made by the library (mlods_kernel_launches).
void note_launch(int n = 1);
// Kernel launches so far (all threads); graphs add their kernel count per replay.
int64_t launches_so_far();
// Multiprocessor count of the current device (cached per device).
int sm_count_for_current_device();
// Stream-ordered scratch memory from the library's pool on the current device.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s);
cudaError_t scratch_free(void* p, cudaStream_t s);

// Makes `dev` the calling thread's current device for the life of the guard
// and restores the previous one afterwards (a tree, batch or server holds
// memory of the device it was made on; dev < 0 leaves the device alone).
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev)
    {
        if (dev < 0) return;
        int cur = 0;
        err = cudaGetDevice(&cur);
        if (err != cudaSuccess || cur == dev) return;
        err = cudaSetDevice(dev);
        if (err == cudaSuccess) prev = cur;
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Error-reporting helpers (host).
void set_last_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define MLODS_CUDA(call)                                                              \
    do {                                                                              \
        cudaError_t _e = (call);                                                      \
        if (_e != cudaSuccess) return ::mlods::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

// Opens an entry point that works on memory of device `dev`: makes it current
// until the function returns, or fails with MLODS_ERR_CUDA.
#define MLODS_ON_DEVICE(dev)                                                              \
    ::mlods::DeviceGuard _mlods_device_guard(dev);                                        \
    if (_mlods_device_guard.err != cudaSuccess)                                           \
        return ::mlods::cuda_fail(_mlods_device_guard.err, "select device", __FILE__, __LINE__)

}  // namespace mlods
