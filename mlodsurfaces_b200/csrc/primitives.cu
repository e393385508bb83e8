// primitives.cu -- device exclusive scan and stable LSD radix sort.
//
// Both are plain HBM-bound passes: tiles of 2048 (scan) or 4096 (sort) items
// per 256-thread block, grids sized by the input.
#include "primitives.cuh"
#include "mlods_internal.cuh"

namespace mlods
{
namespace
{
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;
constexpr int kSortWarps = kSortThreads / 32;

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x == kScanThreads).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* block_total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_scan(v);
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
        uint32_t wi = warp_incl_scan(w);
        if (lane < kScanThreads / 32) s_warp[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) s_warp[kScanThreads / 32] = wi;
    }
    __syncthreads();
    const uint32_t r = s_warp[warp] + incl - v;
    *block_total = s_warp[kScanThreads / 32];
    __syncthreads();
    return r;
}

__global__ void scan_reduce_kernel(const uint32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ block_sums)
{
    __shared__ uint32_t s_warp[kScanThreads / 32 + 1];
    const int64_t base = int64_t(blockIdx.x) * kScanTile;
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + int64_t(k) * kScanThreads + threadIdx.x;
        if (i < n) sum += in[i];
    }
    uint32_t total;
    block_excl_scan(sum, s_warp, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void scan_apply_kernel(const uint32_t* in, uint32_t* out, int64_t n, const uint32_t* __restrict__ block_offs,
                                  uint32_t* total_out)
{
    __shared__ uint32_t s_warp[kScanThreads / 32 + 1];
    const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        sum += v[k];
    }
    uint32_t total;
    uint32_t run = block_excl_scan(sum, s_warp, &total);
    const uint32_t off = block_offs ? block_offs[blockIdx.x] : 0u;
    run += off;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total_out = off + total;
}

// ---------------------------------------------------------------- radix sort

__global__ void radix_hist_kernel(const uint64_t* __restrict__ keys, int64_t n, int shift, int nblocks,
                                  uint32_t* __restrict__ counts)
{
    __shared__ uint32_t hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
#pragma unroll 4
    for (int k = 0; k < kSortRounds; ++k) {
        int64_t i = base + int64_t(k) * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[int64_t(threadIdx.x) * nblocks + blockIdx.x] = hist[threadIdx.x];
}

__global__ void radix_scatter_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals, int64_t n,
                                     int shift, int nblocks, const uint32_t* __restrict__ offs,
                                     uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out)
{
    __shared__ uint32_t s_off[256];
    __shared__ uint32_t s_wcnt[kSortWarps][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s_off[threadIdx.x] = offs[int64_t(threadIdx.x) * nblocks + blockIdx.x];
    const uint32_t lt_mask = (1u << lane) - 1u;
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
    for (int k = 0; k < kSortRounds; ++k) {
        if (base + int64_t(k) * kSortThreads >= n) break;  // uniform across the block
        const int64_t i = base + int64_t(k) * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        const uint64_t key = valid ? keys[i] : 0ull;
        const uint32_t val = (valid && vals) ? vals[i] : 0u;  // vals == nullptr: keys only
        const uint32_t d = valid ? uint32_t((key >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lt_mask);
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) s_wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        if (valid && rank == 0) s_wcnt[warp][d] = __popc(peers);
        __syncthreads();
        uint32_t pos = 0;
        if (valid) {
            pos = s_off[d] + rank;
            for (int w = 0; w < warp; ++w) pos += s_wcnt[w][d];
        }
        __syncthreads();
        {
            uint32_t add = 0;
#pragma unroll
            for (int w = 0; w < kSortWarps; ++w) add += s_wcnt[w][threadIdx.x];
            s_off[threadIdx.x] += add;
        }
        if (valid) {
            keys_out[pos] = key;
            if (vals_out) vals_out[pos] = val;
        }
        __syncthreads();
    }
}

}  // namespace

size_t scan_temp_bytes(int64_t n)
{
    if (n <= kScanTile) return 256;
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    return align_up(size_t(nb) * 4, 256) + scan_temp_bytes(nb);
}

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, void* temp,
                               cudaStream_t s)
{
    if (n <= 0) {
        if (total) return cudaMemsetAsync(total, 0, sizeof(uint32_t), s);
        return cudaSuccess;
    }
    if (n <= kScanTile) {
        scan_apply_kernel<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total);
        note_launch();
        return cudaGetLastError();
    }
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    uint32_t* sums = static_cast<uint32_t*>(temp);
    void* sub = static_cast<char*>(temp) + align_up(size_t(nb) * 4, 256);
    scan_reduce_kernel<<<unsigned(nb), kScanThreads, 0, s>>>(in, n, sums);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = exclusive_scan_u32(sums, sums, nb, nullptr, sub, s);
    if (e != cudaSuccess) return e;
    scan_apply_kernel<<<unsigned(nb), kScanThreads, 0, s>>>(in, out, n, sums, total);
    note_launch();
    return cudaGetLastError();
}

size_t radix_temp_bytes(int64_t n)
{
    const int64_t nb = (n + kSortTile - 1) / kSortTile;
    const int64_t nc = nb * 256;
    return align_up(size_t(nc) * 4, 256) + scan_temp_bytes(nc);
}

cudaError_t radix_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, int64_t n,
                                 int nbits, bool* result_in_alt, void* temp, cudaStream_t s)
{
    *result_in_alt = false;
    if (n <= 1 || nbits <= 0) return cudaSuccess;
    const int64_t nb = (n + kSortTile - 1) / kSortTile;
    const int64_t nc = nb * 256;
    uint32_t* counts = static_cast<uint32_t*>(temp);
    void* scan_tmp = static_cast<char*>(temp) + align_up(size_t(nc) * 4, 256);
    uint64_t* kin = keys;
    uint32_t* vin = vals;
    uint64_t* kout = keys_alt;
    uint32_t* vout = vals_alt;
    bool alt = false;
    for (int shift = 0; shift < nbits; shift += 8) {
        radix_hist_kernel<<<unsigned(nb), kSortThreads, 0, s>>>(kin, n, shift, int(nb), counts);
        note_launch();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        e = exclusive_scan_u32(counts, counts, nc, nullptr, scan_tmp, s);
        if (e != cudaSuccess) return e;
        radix_scatter_kernel<<<unsigned(nb), kSortThreads, 0, s>>>(kin, vin, n, shift, int(nb), counts, kout, vout);
        note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        uint64_t* tk = kin;
        kin = kout;
        kout = tk;
        uint32_t* tv = vin;
        vin = vout;
        vout = tv;
        alt = !alt;
    }
    *result_in_alt = alt;
    return cudaSuccess;
}

}  // namespace mlods
