// project.cuh -- launch interface of the MLoD projection kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "mlods_internal.cuh"

namespace mlods
{

#ifndef MLODS_PROJECT_MIN_BLOCKS
#define MLODS_PROJECT_MIN_BLOCKS 10
#endif
#ifndef MLODS_PROJECT_STACK_CAP
#define MLODS_PROJECT_STACK_CAP 160
#endif
#ifndef MLODS_PROJECT_PAIR_MIN_BLOCKS
#define MLODS_PROJECT_PAIR_MIN_BLOCKS 7
#endif
#ifndef MLODS_PROJECT_PAIR_STACK_CAP
#define MLODS_PROJECT_PAIR_STACK_CAP 128
#endif
constexpr int kProjectThreads = 128;                          // 4 warps per block, one walk per warp at a time
constexpr int kProjectMinBlocks = MLODS_PROJECT_MIN_BLOCKS;  // 10 -> 40 warps per SM, <= 48 registers
constexpr int kProjectStackCap = MLODS_PROJECT_STACK_CAP;    // sibling ranges per warp (28 bytes each)
// the paired walk (two queries per warp): more registers and a wider stack entry
constexpr int kProjectPairMinBlocks = MLODS_PROJECT_PAIR_MIN_BLOCKS;
constexpr int kProjectPairStackCap = MLODS_PROJECT_PAIR_STACK_CAP;

// One tree and its projection settings, plus the query buffers it serves.
struct CloudArgs {
    NodeArrays nodes;
    double o0, o1, o2;      // local frame origin
    KernelConsts kc;
    float cutoff;
    int min_depth;
    float step_max;
    int rule;               // MLODS_BLEND_*
    int n_iter;
    int conv_mode;          // MLODS_CONVERGE_*
    float conv_tol;
    const float* q_in;      // world xyz
    float* out_p;           // world xyz (may alias q_in), or relative to the origin with local_out
    float* out_n;
    int local_out;          // 1: out_p holds the result relative to (o0, o1, o2)
    int qpw;                // the tree's walk schedule (queries per warp) for launches of its own
    float prune_thr;        // > 0: kernel-weight pruning threshold (prune_tol * w(0) * mean sample area)
};

struct ProjectArgs {
    CloudArgs cloud;
    const uint32_t* order;  // processing order (Morton), or nullptr
    int64_t nq;
    unsigned int* counter;  // work counter, zero before launch
    int64_t* stats;         // [0] query-node visits, [1] max stack, [2] overflows, [3] counter, [4] rounds,
                            // [5] query-iterations, [6] lane visits (a node shared by a warp's queries once)
    int queries_per_warp = 1;  // 1, or 2: consecutive queries of `order` share one walk
    uint32_t order_base = 0;   // subtracted from every entry of `order` (a tree's slice of a batch order)
};

// Many trees in ONE persistent launch.  The queries of cloud c occupy the
// global range [base[c], base[c] + len[c]) of the concatenated buffers, and
// the same range of slots of the batch order: order[slot] is the global
// index of the query processed at that slot (nullptr: slot = query index).
// The warps of the queue kernel take queries_per_warp consecutive slots of
// one cloud at a time from a device counter, as the single-tree kernel does
// over one cloud.
struct QueueArgs {
    const CloudArgs* clouds;   // host array: each cloud's q_in / out_p / out_n address its own range
    const int64_t* base;       // host array: first global query of each cloud
    const int64_t* len;        // host array: its query count
    int n_clouds;
    const uint32_t* order;     // device
    unsigned long long* counters;  // device: one 64-bit slot counter per launch group, zero before launch
    int64_t* stats;            // device, as ProjectArgs::stats
    int line_order = 0;        // kQueueMostWorkFirst or kQueueBySpecialisation
};

// The order of the clouds along a launch's slot line: the clouds with the
// most work (queries x iterations) first, or grouped by walk specialisation
// (kernel family, terms, blend rule; the groups with the most work first,
// the clouds inside each group likewise), so that the warps working at any
// moment run the same code.
constexpr int kQueueMostWorkFirst = 0;
constexpr int kQueueBySpecialisation = 1;

// Clouds per launch of the queue kernel: their launch arguments travel by
// value in the kernel's parameters (within the 32 KB parameter limit); a
// batch of more clouds runs as consecutive launches of up to this many.
constexpr int kQueueMaxClouds = 80;
inline int queue_groups(int n_clouds) { return (n_clouds + kQueueMaxClouds - 1) / kQueueMaxClouds; }

// The queue kernel over every group of clouds (usually one launch); every
// cloud is walked queries_per_warp (1 or 2) queries at a time, the pairs
// aligned to the cloud's first slot, so that results equal per-tree
// launches with the same schedule bit for bit.
cudaError_t launch_mlod_queue(const QueueArgs& a, int queries_per_warp, int sm_count, int grid_pct, cudaStream_t s);

// Queries the single-tree walk holds in flight when every SM runs its
// blocks (resident warps x queries per warp).
int64_t project_resident_queries(int queries_per_warp, int sm_count);

// Per-cloud frame used to key queries: the cloud's rank in the batch order
// (clouds of a batch keep their own rank: their slots are their query range)
// and its Morton frame.
struct BatchFrame {
    double o0, o1, o2;
    float inv_ext;
    uint32_t rank;
};

cudaError_t launch_mlod_project(const ProjectArgs& a, int ktype, int rule, int sm_count, cudaStream_t s);

// Swaps query points invalid[i] and end_valid-1-i (GPUUtils.cu:413-424).
cudaError_t launch_reorganize(float* d_q, const uint32_t* d_invalid, int64_t n_invalid, uint32_t end_valid,
                              cudaStream_t s);

// Morton order of queries on a 1024^3 grid over the root box (the reference
// orders its queries on a 64^3 grid, Pn.cpp:388-445).  d_order receives the
// query indices in processing order.
size_t query_order_temp_bytes(int64_t n);
cudaError_t compute_query_order(const float* d_q, int64_t n, const double origin[3], float extent, uint32_t* d_order,
                                void* temp, cudaStream_t s);
// Same for a batch: grouped by cloud rank, Morton order inside each cloud
// (input order when morton is false).
cudaError_t compute_batch_order(const float* d_q, int64_t n, const int64_t* d_q_offsets, int n_clouds,
                                const BatchFrame* d_frames, bool morton, uint32_t* d_order, void* temp,
                                cudaStream_t s);

}  // namespace mlods
