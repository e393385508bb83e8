// project.cuh -- launch interface of the MLoD projection kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mlods_internal.cuh"

namespace mlods
{

constexpr int kProjectThreads = 128;   // 4 warps per block, one query per warp at a time
constexpr int kProjectStackCap = 192;  // sibling ranges per warp (24 bytes each)

struct ProjectArgs {
    const DNode* nodes;
    const float* q_in;       // world xyz
    float* out_p;            // world xyz (may alias q_in)
    float* out_n;
    const uint32_t* order;   // processing order (Morton), or nullptr
    int64_t nq;
    int n_iter;
    float cutoff;
    int min_depth;
    float step_max;
    double o0, o1, o2;       // local frame origin
    KernelConsts kc;
    unsigned int* counter;   // work counter, zero before launch
    int64_t* stats;          // [0] node visits, [1] max stack, [2] overflows, [3] work counter, [4] rounds
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

}  // namespace mlods
