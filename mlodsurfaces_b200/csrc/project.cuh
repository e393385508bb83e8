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
#ifndef MLODS_BATCH_MIN_BLOCKS
#define MLODS_BATCH_MIN_BLOCKS 8
#endif
#ifndef MLODS_PROJECT_STACK_CAP
#define MLODS_PROJECT_STACK_CAP 160
#endif
#ifndef MLODS_PROJECT_PAIR_MIN_BLOCKS
#define MLODS_PROJECT_PAIR_MIN_BLOCKS 8
#endif
#ifndef MLODS_PROJECT_PAIR_STACK_CAP
#define MLODS_PROJECT_PAIR_STACK_CAP 128
#endif
constexpr int kProjectThreads = 128;                          // 4 warps per block, one walk per warp at a time
constexpr int kProjectMinBlocks = MLODS_PROJECT_MIN_BLOCKS;  // 10 -> 40 warps per SM, <= 48 registers
constexpr int kProjectStackCap = MLODS_PROJECT_STACK_CAP;    // sibling ranges per warp (28 bytes each)
constexpr int kBatchMinBlocks = MLODS_BATCH_MIN_BLOCKS;      // the batch kernel keeps more registers (64)
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
};

// Many trees in one launch: clouds[c] serves the global query range
// [q_offsets[c], q_offsets[c+1]) of the concatenated buffers (each cloud's
// q_in/out_p/out_n point at the start of its own range).  order[slot] is the
// global index of the query processed at each slot; clouds that share a
// kernel specialisation occupy consecutive slots, and each such group runs
// as one launch of its specialised kernel over its slot range.
struct BatchArgs {
    const CloudArgs* clouds;
    const int64_t* q_offsets;  // n_clouds + 1 entries
    int n_clouds;
    int64_t total;
    const uint32_t* order;     // slot -> global query index (grouped, Morton order inside each cloud)
    const int64_t* rank_slot;  // n_clouds + 1 entries: first slot of the cloud of each rank
    const int32_t* rank_cloud; // n_clouds entries: cloud of each rank
    unsigned int* counters;    // one work counter per group, zero before launch
    int64_t* stats;            // [0] visits, [1] max stack, [2] overflows, [4] rounds, [5] iterations
};

constexpr int kMaxBatchGroups = 256;
constexpr int kMaxSoloClouds = 128;  // clouds launched on their own, at most

// One launch of a batch and its slot range: either a kernel specialisation
// shared by several clouds (solo < 0), run by the batched kernel, or one
// large cloud (solo = its index) run by the single-tree kernel with the
// cloud's arguments in the constant bank; solo_args then addresses the whole
// concatenated buffers, so that the global indices of `order` apply.
struct BatchGroup {
    int ktype, nsig, rule;
    int64_t slot_begin, slot_end;
    int solo = -1;
    CloudArgs solo_args;
    int queries_per_warp = 1;  // the solo cloud's walk schedule
};

// Per-cloud frame used to key queries: the group-ordered rank of the cloud
// and its Morton frame.
struct BatchFrame {
    double o0, o1, o2;
    float inv_ext;
    uint32_t rank;
};

// Ranks the clouds so that those of one kernel specialisation (weight type,
// number of sigmas, blend rule) are consecutive and fills frames[i].rank,
// rank_slot (n_clouds + 1 entries) and rank_cloud (n_clouds); groups receive
// the slot ranges.  Host only.
// Clouds with at least solo_min queries (0: none) get their own launch,
// up to kMaxSoloClouds of them, largest first.
void plan_batch_groups(const CloudArgs* clouds, const int64_t* q_offsets, int n_clouds, BatchFrame* frames,
                       int64_t* rank_slot, int32_t* rank_cloud, std::vector<BatchGroup>& groups,
                       int64_t solo_min);
// Query count from which a cloud of a batch runs in a launch of its own:
// eight queries per resident warp of the single-tree kernel.
int64_t batch_solo_min_queries(int sm_count);

cudaError_t launch_mlod_project(const ProjectArgs& a, int ktype, int rule, int sm_count, cudaStream_t s);
cudaError_t launch_mlod_batch(const BatchArgs& b, const std::vector<BatchGroup>& groups, int sm_count,
                              int grid_scale_pct, cudaStream_t s);

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
