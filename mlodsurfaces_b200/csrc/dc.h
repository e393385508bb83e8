// dc.h -- dual-contouring grid (host) and corner-field / vertex evaluation (device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

struct mlods_tree_s;

namespace mlods
{
// Cells as (depth, x, y, z) quadruples in sorted_octree order; depth_out is the
// deepest cell depth.
int dcgrid_from_points(const float* pts, int64_t n, int max_depth, const float box_min[3], const float box_max[3],
                       std::vector<int32_t>& cells_out, int& depth_out);

// Field at the 8 corners of every cell (unique corners projected once) and
// the per-cell vertex; host arrays in and out.
int dc_evaluate(mlods_tree_s* T, int64_t n_cells, const int32_t* cells, int max_depth, const float* xform,
                int use_normals, float* corner_f, float* vertex, int32_t* n_cross, int64_t* n_unique, cudaStream_t s);
}  // namespace mlods
