// dc.h -- dual contouring: cell grids (host), corner field / vertex
// evaluation (device), mesh extraction and refinement.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

struct mlods_tree_s;

namespace mlods
{
namespace dcg
{
// One octree cell: octree_id (sources/dual-contouring/octree.h:18-44).
struct Cell {
    int depth, x, y, z;
    bool operator==(const Cell& o) const { return depth == o.depth && x == o.x && y == o.y && z == o.z; }
};

// node_comparator, octree.h:147-154: depth, then z, y, x
inline bool cell_less(const Cell& a, const Cell& b)
{
    if (a.depth != b.depth) return a.depth < b.depth;
    if (a.z != b.z) return a.z < b.z;
    if (a.y != b.y) return a.y < b.y;
    return a.x < b.x;
}

// octree_id::parent / ancestor_at_depth, octree.h:547-572 (division rounded
// towards -infinity)
inline int floor_half(int v) { return (v < 0 && (v % 2) != 0) ? v / 2 - 1 : v / 2; }
inline Cell parent(const Cell& c) { return Cell{c.depth - 1, floor_half(c.x), floor_half(c.y), floor_half(c.z)}; }
inline Cell ancestor_at(Cell c, int d)
{
    while (c.depth > d) c = parent(c);
    return c;
}
// octree_id::child, octree.h:574-582
inline Cell child(const Cell& c, int k)
{
    return Cell{c.depth + 1, 2 * c.x + (k & 1), 2 * c.y + ((k >> 1) & 1), 2 * c.z + ((k >> 2) & 1)};
}
// octree_id::neighbor, octree.h:591-602 (n = 0..26, 13 is the cell itself)
inline Cell neighbor(const Cell& c, int n)
{
    const int z = n / 9, y = (n - 9 * z) / 3, x = n - 9 * z - 3 * y;
    return Cell{c.depth, c.x + x - 1, c.y + y - 1, c.z + z - 1};
}

void remove_duplicates(std::vector<Cell>& v);
void grade(std::vector<Cell>& nodes);
void regularize_up(std::vector<Cell>& nodes);
void regularize_siblings(std::vector<Cell>& nodes);
// all 26 neighbours of the cells at `depth` (every cell when depth < 0),
// then sorted and de-duplicated (upsample.cpp:404-414)
void expand(std::vector<Cell>& nodes, int depth);
void cells_to_ints(const std::vector<Cell>& nodes, std::vector<int32_t>& out, int& max_depth);
}  // namespace dcg

// Cells as (depth, x, y, z) quadruples in sorted_octree order; depth_out is the
// deepest cell depth.
int dcgrid_from_points(const float* pts, int64_t n, int max_depth, const float box_min[3], const float box_max[3],
                       std::vector<int32_t>& cells_out, int& depth_out);

// dcgrid_from_points with the set work on the device; *handled is false when
// the inputs need the host version (depth or coordinates beyond the keys).
int dcgrid_from_points_device(const float* pts, int64_t n, int max_depth, const float box_min[3],
                              const float box_max[3], cudaStream_t s, std::vector<int32_t>& cells_out, int& depth_out,
                              bool* handled);

// The projection-driven grid (OctreeGenerator::generate + uniformize,
// upsample.cpp:228-251, :262-273): cells, their depth and the 3x4 map from the
// grid's unit frame to the tree's frame (new2bbox, scene.cpp:1311).
int dcgrid_adaptive(mlods_tree_s* T, int max_depth, bool cut, cudaStream_t s, std::vector<int32_t>& cells_out,
                    int& depth_out, float xform[12], int64_t* n_projected);

// A triangle mesh in device memory and the refinement steps on it
// (mesh_dev.cu); each returns an MLODS_* status.
struct DeviceMesh;
DeviceMesh* dmesh_create();
void dmesh_destroy(DeviceMesh* m);
int dmesh_upload(DeviceMesh& m, const float* pos, int64_t nv, const uint32_t* tri, int64_t nt, cudaStream_t s);
int dmesh_download(const DeviceMesh& m, std::vector<float>& pos, std::vector<float>& nrm, std::vector<uint32_t>& tri,
                   cudaStream_t s);
int dmesh_transform(DeviceMesh& m, const float* xform, cudaStream_t s);
int dmesh_project(mlods_tree_s* T, DeviceMesh& m, int iters, cudaStream_t s);
int dmesh_smooth(DeviceMesh& m, cudaStream_t s);
int dmesh_subdivide(DeviceMesh& m, cudaStream_t s);

// The corner field of a grid kept in device memory: cells (int4), 8 corner
// values, vertex and crossing count per cell, in one allocation.
struct DcField {
    void* base = nullptr;   // scratch of the library pool, freed in stream order
    void* base2 = nullptr;  // unique-corner buffers
    cudaStream_t stream = nullptr;
    const int4* cells = nullptr;
    float* cf = nullptr;
    float* vert = nullptr;
    int32_t* ncross = nullptr;
    int64_t n = 0, n_unique = 0;
};
int dc_field_device(mlods_tree_s* T, int64_t n_cells, const int32_t* cells, bool cells_on_device, int max_depth,
                    const float* xform, int use_normals, DcField& out, cudaStream_t s);
void dc_field_free(DcField& f);

// Extraction on the device (dc_extract_dev.cu) from a device field; the mesh
// goes to `out` (unit-frame vertices).  *used_device is false when the grid
// is too deep for the device path (the caller then extracts on the host).
int dc_extract_device(const int4* d_cells, int64_t n_cells, const int64_t* h_depth_begin, int max_depth,
                      const float* d_cf, const float* d_cell_vertex, DeviceMesh& out, bool* used_device,
                      cudaStream_t s);
int dmesh_reserve(DeviceMesh& m, int64_t nv, int64_t nt);
int64_t dmesh_nv(const DeviceMesh& m);
int64_t dmesh_nt(const DeviceMesh& m);
// Copies the mesh into caller buffers (any may be null) and waits for it.
int dmesh_get(const DeviceMesh& m, float* pos, float* nrm, uint32_t* tri, cudaStream_t s);
float* dmesh_pos(DeviceMesh& m);
float* dmesh_nrm(DeviceMesh& m);
uint32_t* dmesh_tri(DeviceMesh& m);

// Field at the 8 corners of every cell (unique corners projected once) and
// the per-cell vertex; cells in host or device memory, outputs in host or
// device memory (told apart by address).
int dc_evaluate(mlods_tree_s* T, int64_t n_cells, const int32_t* cells, bool cells_on_device, int max_depth,
                const float* xform, int use_normals, float* corner_f, float* vertex, int32_t* n_cross,
                int64_t* n_unique, cudaStream_t s);
}  // namespace mlods
