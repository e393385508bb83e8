// gather.cuh -- launch interface of the neighbour gathers and the global APSS.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mlods_internal.cuh"

namespace mlods
{

constexpr int kGatherThreads = 128;
constexpr int kGatherKnnApss = 0;
constexpr int kGatherBallApss = 1;
constexpr int kGatherKnnOnly = 2;

struct GatherArgs {
    NodeArrays nodes;
    const int32_t* node_head;  // sorted position of each node's first point
    const uint64_t* codes;     // sorted Morton codes
    const float4* wspts;       // sorted points, world frame, w = original index bits
    const float4* spts;        // sorted points, local frame
    const float4* snrm;        // sorted normals
    const float* bounds;       // per-axis float bound tables
    int64_t bounds_stride;
    int max_depth;
    int64_t n_pts;
    const float* q_in;         // world xyz
    int64_t nq;
    float* out_p;
    float* out_n;
    int32_t* out_idx;          // kNN sets (k per query)
    float* out_d2;
    int k;
    float ball_r;
    float eps;                 // pruning margin for the float local frame
    int n_iter;
    float step_max;
    double o0, o1, o2;
    KernelConsts kc;
    unsigned int* counter;
    int64_t* stats;
};

struct GlobalArgs {
    const float4* spts;
    const float4* snrm;
    const float* area;  // per original point
    int64_t n_pts;
    const float* q_in;
    int64_t nq;
    float* out_p;
    float* out_n;
    int n_iter;
    float step_max;
    double o0, o1, o2;
    KernelConsts kc;
};

cudaError_t launch_gather(const GatherArgs& a, int mode, int ktype, int sm_count, cudaStream_t s);
cudaError_t launch_global_apss(const GlobalArgs& a, int ktype, cudaStream_t s);

}  // namespace mlods
