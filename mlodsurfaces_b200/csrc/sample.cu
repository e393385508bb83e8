// sample.cu -- query generation in octree cells on the device
// (scene::generateFromOctree, scene.cpp:733-756).
//
// Each output point picks a cell (depth, x, y, z) of the [-1, 1]^3 octree
// uniformly, then moves from the cell's centre by an offset uniform in
// [-0.5, 0.5)^3 times 4 / 2^depth (twice the cell side); its normal is the
// point itself.  The reference draws from a std::mt19937 seeded by
// std::random_device; here every draw is a counter-based hash of
// (seed, output index, draw index), so a seed gives the same points on any
// device and launch shape, and the points are written straight into HBM for
// the projection that follows.
#include <cstdint>

#include "mlods.h"
#include "mlods_internal.cuh"

namespace mlods
{
namespace
{
constexpr int kSampleThreads = 256;

// splitmix64 finaliser (Steele, Lea, Flood: "Fast splittable pseudorandom
// number generators", OOPSLA 2014).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Draw k of output i: four draws per point (cell, x, y, z).
__device__ __forceinline__ uint64_t draw(uint64_t seed, int64_t i, int k)
{
    return mix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t(i) * 4u + uint64_t(k) + 1u));
}

// Uniform in [-0.5, 0.5) with 24 bits: exact in float.
__device__ __forceinline__ float centred_unit(uint64_t r)
{
    return float(uint32_t(r >> 40)) * (1.0f / 16777216.0f) - 0.5f;
}

__global__ void __launch_bounds__(kSampleThreads)
    sample_cells_kernel(const int32_t* __restrict__ cells, int64_t n_cells, int64_t n_out, uint64_t seed,
                        float* __restrict__ out_p, float* __restrict__ out_n)
{
    for (int64_t i = int64_t(blockIdx.x) * kSampleThreads + threadIdx.x; i < n_out;
         i += int64_t(gridDim.x) * kSampleThreads) {
        const uint64_t pick = __umul64hi(draw(seed, i, 0), uint64_t(n_cells));  // in [0, n_cells)
        const int4 c = reinterpret_cast<const int4*>(cells)[pick];
        const int depth = c.x;
        if (depth < 0 || depth > 30) {  // not a cell: NaN point
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                out_p[3 * i + a] = __int_as_float(0x7fc00000);
                if (out_n) out_n[3 * i + a] = __int_as_float(0x7fc00000);
            }
            continue;
        }
        // aabb_octree::bounds / center over [-1, 1]^3 (octree.h:939-955), float
        const float w = __fdiv_rn(2.0f, float(1 << depth));
        const float move = __fdiv_rn(4.0f, float(1 << depth));
        const int pos[3] = {c.y, c.z, c.w};
        float p[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float lo = __fadd_rn(-1.0f, __fmul_rn(w, float(pos[a])));
            const float hi = __fadd_rn(-1.0f, __fmul_rn(w, float(pos[a] + 1)));
            const float centre = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
            p[a] = __fadd_rn(centre, __fmul_rn(centred_unit(draw(seed, i, a + 1)), move));
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            out_p[3 * i + a] = p[a];
            if (out_n) out_n[3 * i + a] = p[a];
        }
    }
}
}  // namespace
}  // namespace mlods

using namespace mlods;

extern "C" int mlods_sample_cells_device(const int32_t* d_cells, int64_t n_cells, int64_t n_out, uint64_t seed,
                                         float* d_out_pts, float* d_out_nrm, void* stream)
{
    if (n_out < 0 || (n_out > 0 && (!d_cells || n_cells <= 0 || !d_out_pts))) {
        set_last_error("sample cells: bad arguments");
        return MLODS_ERR_INVALID;
    }
    if (reinterpret_cast<uintptr_t>(d_cells) % 16 != 0) {
        set_last_error("sample cells: the cell array must be 16-byte aligned");
        return MLODS_ERR_INVALID;
    }
    if (n_out == 0) return MLODS_OK;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t want = (n_out + kSampleThreads - 1) / kSampleThreads;
    const int64_t cap = int64_t(sm_count_for_current_device()) * 8;
    const unsigned grid = unsigned(want < cap ? want : cap);
    sample_cells_kernel<<<grid, kSampleThreads, 0, s>>>(d_cells, n_cells, n_out, seed, d_out_pts, d_out_nrm);
    note_launch();
    MLODS_CUDA(cudaGetLastError());
    return MLODS_OK;
}
