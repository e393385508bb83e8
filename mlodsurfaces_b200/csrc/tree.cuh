// tree.cuh -- the tree handle behind mlods_tree.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "mlods_internal.cuh"

struct mlods_tree_s {
    int device = 0;
    int64_t n_pts = 0;
    int max_depth = 0;
    int depth = 0;
    int64_t n_nodes = 0;   // reference nodes
    int64_t n_extra = 0;   // point records of multi-point leaves
    int64_t n_ties = 0;
    float bb[3] = {0, 0, 0};
    float BB[3] = {0, 0, 0};
    double origin[3] = {0, 0, 0};
    float root_radius = 0.f;  // BBOX::radius of the root box, float as the reference
    float root_mass = 0.f;    // sum of the sample areas (the root's m0)

    // device data
    mlods::NodeArrays nodes{};             // n_nodes + n_extra records (one allocation at nodes.geom)
    int32_t* d_node_head = nullptr;        // sorted position of each node's first point
    uint64_t* d_codes = nullptr;           // Morton codes in sorted order
    uint32_t* d_perm = nullptr;            // sorted position -> original point index
    float* d_area = nullptr;               // per original point (float, as the reference)
    float4* d_spts = nullptr;              // sorted points, local frame: xyz, w = original index bits
    float4* d_snrm = nullptr;              // sorted normals
    float4* d_wspts = nullptr;             // sorted points, world frame (exact neighbour distances)
    float* d_bounds = nullptr;             // per-axis float bound tables (3 x table size)
    int64_t bounds_stride = 0;

    // configuration
    mlods_kernel kernel{};                 // sigmas_ext is always null here
    std::vector<float> sigmas_long;        // the sigmas when there are more than MLODS_INLINE_SIGMAS
    mlods::KernelConsts kc{};
    mlods_params params{};
    bool kernel_set = false;

    // reusable scratch for projection (grown on demand)
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    int64_t* d_stats = nullptr;  // [0] visits, [1] max stack, [2] overflows, [3] work counter
    int64_t last_visits = 0;
    int32_t last_max_stack = 0;
    int64_t last_overflows = 0;

    int64_t device_bytes = 0;

    // CUDA events bracketing the last projection kernel (created on first use)
    cudaEvent_t ev_start = nullptr;
    cudaEvent_t ev_stop = nullptr;
    bool timed = false;
};

// Device query buffer of the copyPointsToGPU / project protocol, owned by the
// projection object (APSS::m_outPts, m_outNmls, GPUUtils.h:56-57).
struct mlods_queries_s {
    float* d_q = nullptr;
    float* d_qn = nullptr;
    int64_t n = 0;    // uploaded queries
    int64_t cap = 0;  // allocated queries
};

// Dual-contouring cell grid: (depth, x, y, z) per cell in sorted_octree order.
struct mlods_dcgrid_s {
    std::vector<int32_t> cells;
    int max_depth = 0;
    // rows 0-2 of the 4x4 map from the grid's unit frame to the tree's frame
    // (new2bbox, scene.cpp:1311)
    float xform[12] = {2.f, 0.f, 0.f, -1.f, 0.f, 2.f, 0.f, -1.f, 0.f, 0.f, 2.f, -1.f};
    int64_t n_projected = 0;  // centre projections made while generating it
};

namespace mlods
{
// Builds the tree from device arrays (xyz float triples).
int build_tree(mlods_tree_s* T, const float* d_pts, const float* d_nrm, int64_t n, int max_depth, cudaStream_t s);
void free_tree_device(mlods_tree_s* T);
// Scratch of one projection call that must not share the tree's: a
// zero-initialised-by-the-callee statistics block of 8 int64 (visits, max
// stack, overflows, work counter, ...) and `bytes` bytes of device memory at
// `base` (at least project_call_bytes).
struct CallScratch {
    int64_t* stats;
    char* base;
    size_t bytes;
};
// Device scratch bytes (beyond the statistics block) one projection call of n
// queries needs with the tree's current options.
size_t project_call_bytes(const mlods_tree_s* T, int64_t n);
// Projects n device queries through the tree with its current kernel and
// options (the mode selects MLoD, global, kNN or ball APSS).  Asynchronous.
// Without `cs` the call uses the tree's own scratch, statistics and timing
// events (calls on one tree must then be ordered); with `cs` it touches none of
// them, so calls from several host threads may overlap.
int project_buffers(mlods_tree_s* T, int64_t n, const float* d_q, float* d_out_p, float* d_out_n, int iters,
                    float step_max, cudaStream_t s, int rule_override = -1, const CallScratch* cs = nullptr);
struct CloudArgs;
// Fills the per-tree part of a projection launch.
void fill_cloud_args(const mlods_tree_s* T, CloudArgs& c, const float* d_q, float* d_out_p, float* d_out_n,
                     int iters, float step_max, int rule);
int export_tree(mlods_tree_s* T, int32_t* depth, int32_t* parent, int32_t* first_child, int32_t* n_children,
                int32_t* next_brother, int32_t* leaf_off, int32_t* leaf_cnt, int32_t* perm, float* bmin, float* bmax,
                double* mom, float* area);
}  // namespace mlods
