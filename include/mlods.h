/*
 * mlods.h -- C ABI of libmlods.so, a B200 (sm_100a) implementation of the
 * point-set surface projection path of "Moving Level-of-Detail Surfaces"
 * (reference project: CorentinMercier/MlodSurfaces).
 *
 * Plain pointers and sizes only.  Every entry point returns an int status
 * (MLODS_OK on success); mlods_last_error() gives the message of the last
 * failure on the calling thread.  `stream` is a cudaStream_t passed as void*
 * (NULL = the legacy default stream).  Host pointers are ordinary (pageable or
 * pinned) memory; arguments named d_* are device pointers.
 *
 * Coordinates are float xyz triples (the layout of std::vector<glm::vec3>).
 */
#ifndef MLODS_H
#define MLODS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define MLODS_OK 0
#define MLODS_ERR_INVALID 1   /* bad argument (null handle, n == 0, unknown enum, ...) */
#define MLODS_ERR_CUDA 2      /* a CUDA call failed; see mlods_last_error() */
#define MLODS_ERR_STATE 3     /* call out of protocol order (e.g. project before upload) */
#define MLODS_ERR_CAPACITY 4  /* a request exceeds a fixed capacity */
#define MLODS_ERR_TIMEOUT 5   /* a bounded wait ran out (the operation may still finish) */

/* ---- weight kernels (Kernel.h:37, Kernel.cpp:64-83) ------------------- */
#define MLODS_GAUSSIAN 0
#define MLODS_SINGULAR 1          /* the reference's "rational" kernel */
#define MLODS_GAUSSIAN_MULTIPLE 2
/* sigmas held in mlods_kernel itself; longer lists go through sigmas_ext */
#define MLODS_INLINE_SIGMAS 16

/* ---- projection modes (APSS subclasses and APSSOctree modes) ----------- */
#define MLODS_MODE_MLOD 0    /* Fastapss::project (Fastapss.cu:439-455) */
#define MLODS_MODE_GLOBAL 1  /* GlobalAPSS::project (GlobalAPSS.cu:203-235) */
#define MLODS_MODE_KNN 2     /* APSSOctree::knnMode + projectAPSSCPU (CPUUtils.cpp:674-737) */
#define MLODS_MODE_BALL 3    /* APSSOctree::ballMode + projectAPSSCPU (CPUUtils.cpp:682-737) */

/* ---- blend rules of the MLoD traversal --------------------------------- */
#define MLODS_BLEND_GPU 0  /* parent weight w * a_child / a_node, |u4| < 1e-6 (Fastapss.cu:244, :362) */
#define MLODS_BLEND_CPU 1  /* parent weight w / #children, |u4| < 1e-12 (CPUUtils.cpp:485, :751) */

/* Kernel value type; mirrors class Kernel (Kernel.h:24-60).  sigma and sigmas
 * are absolute lengths (already multiplied by the box radius, as
 * scene::setNewKernel does, scene.cpp:1025-1033).  Like the reference's
 * Kernel::sigmas (a std::vector, Kernel.cpp:110-128, copied to a device array
 * of its size by GPUUtils.cu:262-272) the list has no fixed length: up to
 * MLODS_INLINE_SIGMAS sigmas sit in sigmas[]; a longer list is read from
 * sigmas_ext (n_sigmas host floats; sigmas[] is then ignored).  The library
 * copies the list when the kernel is set or a request is submitted, so
 * sigmas_ext need only live for that call.  The reference's own parameter
 * files use up to 30 terms (data/rhino-holes.params). */
typedef struct mlods_kernel {
    int32_t type;            /* MLODS_GAUSSIAN / _SINGULAR / _GAUSSIAN_MULTIPLE */
    float sigma;             /* Kernel::sigma */
    float exponent;          /* Kernel::exponent */
    float constant_shift;    /* Kernel::constant_shift */
    int32_t n_sigmas;        /* Kernel::sigmas.size() */
    float sigmas[MLODS_INLINE_SIGMAS];
    const float* sigmas_ext; /* n_sigmas sigmas when n_sigmas > MLODS_INLINE_SIGMAS, else unused (NULL) */
} mlods_kernel;

/* Projection options; mirror APSS::setScalingProtectionSphere / setMinDepth
 * (GPUUtils.h:40-43) and APSSOctree::knnMode / ballMode (CPUUtils.h:191-192). */
/* ---- convergence modes (extension; the reference always runs n_iterations) ---- */
#define MLODS_CONVERGE_OFF 0    /* run every iteration (reference behaviour) */
#define MLODS_CONVERGE_EXACT 1  /* stop a query once its float iterate repeats: the remaining iterations
                                   would return the same result, so outputs are bit-identical */
#define MLODS_CONVERGE_TOL 2    /* stop a query once its step is shorter than converge_tol */

typedef struct mlods_params {
    float cutoff;        /* scalingProtectionSphere: a node is an aggregate when |q-c| > cutoff*r (default 2) */
    int32_t min_depth;   /* nodes shallower than this are always opened (default 0) */
    int32_t mode;        /* MLODS_MODE_* */
    int32_t knn;         /* k for MLODS_MODE_KNN (default 20) */
    float ball_radius;   /* radius for MLODS_MODE_BALL; < 0 uses 3 * sigmas[0] (default 0.1) */
    int32_t blend_rule;  /* MLODS_BLEND_GPU (default) or MLODS_BLEND_CPU */
    int32_t reorder;     /* 1: process queries in Morton order (results are identical) */
    float prune_tol;     /* extension, default 0 (off: the reference's walk).  > 0: kernel-weight
                            pruning of the MLoD walk -- a node the walk would open is taken as an
                            aggregate instead when a bound on what its whole subtree can weigh,
                            f * w(distance to the node's bounding sphere) * its area (the kernel
                            decreases with distance), is below prune_tol times the weight of one
                            average sample at the query, w(0) * mean area.  Fewer node visits;
                            results move by at most what the dropped subtrees could weigh.
                            Applies to projections of one tree (queries_per_warp 1 or 2, which
                            it requires); batched and served projections walk without it. */
    int32_t converge;    /* MLODS_CONVERGE_* (default MLODS_CONVERGE_OFF) */
    float converge_tol;  /* step length for MLODS_CONVERGE_TOL (absolute units) */
    int32_t local_output; /* extension, default 0.  1: MLoD results are written relative to the
                             tree's origin (mlods_tree_info.origin) instead of in world
                             coordinates, so a cloud far from the world origin keeps full
                             float precision in its output.  Ignored when the output buffer
                             is the input buffer (the in-place query-buffer protocol). */
    int32_t queries_per_warp; /* extension: the MLoD walk schedule.  1 (default): one query per warp.
                                 2 or 4: that many queries that are neighbours in processing order
                                 share one walk of the tree (node loads and traversal bookkeeping
                                 paid once); each query's arithmetic is unchanged, only the order
                                 of its float sums differs, so results agree with 1 to float
                                 rounding.  mlods_tune_schedule picks it by timing. */
} mlods_params;

typedef struct mlods_tree_s* mlods_tree;

/* Tree statistics. */
typedef struct mlods_tree_info {
    int64_t n_points;
    int64_t n_nodes;       /* reference node count (APSSOctree nbOfNodes, CPUUtils.cpp:177-184) */
    int64_t n_extra;       /* point records of multi-point leaves */
    int32_t depth;         /* octreeNode::computeDepth of the root (CPUUtils.cpp:254-261) */
    int32_t max_depth;
    int64_t n_ties;        /* points lying exactly on a split they were classified by (sent low) */
    float bbox_min[3];     /* root box, BBOX (CPUUtils.h:70-99) */
    float bbox_max[3];
    double origin[3];      /* local frame origin (centre of the root box) */
    int64_t device_bytes;  /* device memory held by the tree */
} mlods_tree_info;

/* ---- library ------------------------------------------------------------ */
const char* mlods_last_error(void);
int mlods_version(void);

/* ---- tree (APSSOctree::build, CPUUtils.cpp:540-569) ----------------------
 * Builds the octree on the device: Morton codes on the reference's split
 * lattice, radix sort, level-wise node creation, area weights and bottom-up
 * moments.  Topology and breadth-first order equal the reference's (points
 * exactly on a split go to the low child).  max_depth <= 12 (MAX_DEPTH).
 * mlods_tree_build takes host arrays (copied in); mlods_tree_build_device
 * takes device arrays (read, not kept). */
int mlods_tree_build(const float* pts, const float* nrm, int64_t n, int32_t max_depth, void* stream,
                     mlods_tree* out);
int mlods_tree_build_device(const float* d_pts, const float* d_nrm, int64_t n, int32_t max_depth, void* stream,
                            mlods_tree* out);
/* Frees everything the tree holds (Fastapss::eraseFromGPU + APSS::erasePointsFromGPU,
 * Fastapss.cu:486-511, GPUUtils.cu:452-464). */
int mlods_tree_free(mlods_tree t);
int mlods_tree_get_info(mlods_tree t, mlods_tree_info* info);

/* Downloads the topology in breadth-first order for parity checks.  Arrays
 * are n_nodes long (perm: n_points): father/firstChild/nextBrother as
 * octreeNode::getRelations (CPUUtils.cpp:213-234); leaf_off/leaf_cnt index
 * into perm, which lists each leaf's original point indices in ascending
 * order; bmin/bmax are the float boxes (3 per node); mom holds 9 doubles per
 * node {m0, pbar[3] (world), n[3], cpn, cpp}.  Any pointer may be NULL. */
int mlods_tree_export(mlods_tree t, int32_t* depth, int32_t* parent, int32_t* first_child, int32_t* n_children,
                      int32_t* next_brother, int32_t* leaf_off, int32_t* leaf_cnt, int32_t* perm, float* bmin,
                      float* bmax, double* mom, float* area);

/* ---- kernel and options ---------------------------------------------------
 * mlods_set_kernel replaces the device kernel (APSS::updateKernel,
 * GPUUtils.cu:466-472, without its leak).  mlods_set_params replaces all
 * options at once; mlods_default_params fills the reference defaults. */
int mlods_set_kernel(mlods_tree t, const mlods_kernel* k);
void mlods_default_params(mlods_params* p);
int mlods_set_params(mlods_tree t, const mlods_params* p);

/* ---- query buffer protocol (Fastapss::copyToGPU/project, APSS::copyPointsToGPU) ----
 * A query buffer is owned by its projection object, as APSS owns m_outPts and
 * m_outNmls (GPUUtils.h:56-57); a tree can serve several buffers.
 * mlods_queries_upload copies n host points into the buffer's device memory
 * (APSS::copyPointsToGPU, GPUUtils.cu:406-411; an earlier upload is replaced,
 * not leaked).  mlods_project runs n_iterations projection steps in place on
 * that buffer, so repeated calls continue from the last positions, and
 * copies positions/normals back when the host pointers are non-NULL
 * (Fastapss::project, Fastapss.cu:439-455).  step_max < 0 selects the root
 * box radius.  n must not exceed the uploaded count.  mlods_queries_free
 * releases the device memory (APSS::erasePointsFromGPU) and keeps the handle;
 * mlods_queries_destroy releases both. */
typedef struct mlods_queries_s* mlods_queries;
int mlods_queries_create(mlods_queries* out);
int mlods_queries_destroy(mlods_queries q);
int mlods_queries_upload(mlods_queries q, int64_t n, const float* pts, void* stream);
int mlods_queries_free(mlods_queries q);
int mlods_project(mlods_tree t, mlods_queries q, int64_t n, int32_t n_iterations, float step_max, float* out_pts,
                  float* out_nrm, void* stream);

/* Swaps the queries listed in invalid[0..n_invalid) with the tail of the first
 * end_valid queries of the buffer, so that the valid ones come first
 * (APSS::reorganizePoints and the reorganizePts kernel, GPUUtils.cu:413-424,
 * :503-517).  invalid is a host array. */
int mlods_queries_reorganize(mlods_queries q, int64_t n_invalid, const uint32_t* invalid, uint32_t end_valid,
                             void* stream);

/* ---- one-off host projection ---------------------------------------------
 * Projects n host queries into host outputs without touching the query
 * buffer (synchronous).  blend_rule overrides the tree's rule (-1 keeps it);
 * the C++ mirror's projectCPU uses MLODS_BLEND_CPU here, the reference's CPU
 * semantics (APSSOctree::projectCPU, CPUUtils.cpp:621-636), evaluated on the
 * device. */
int mlods_project_host(mlods_tree t, int64_t n, const float* q, float* out_pts, float* out_nrm, int32_t n_iterations,
                       float step_max, int32_t blend_rule, void* stream);

/* ---- device-buffer projection (no host traffic) ---------------------------
 * Projects n queries d_q (device, xyz) into d_out_pts / d_out_nrm (device).
 * d_out_pts may equal d_q (in place).  Asynchronous on `stream`. */
int mlods_project_device(mlods_tree t, int64_t n, const float* d_q, float* d_out_pts, float* d_out_nrm,
                         int32_t n_iterations, float step_max, void* stream);

/* ---- walk schedule autotuner (extension) -----------------------------------
 * Times the MLoD projection of the n device queries d_q (n_iterations steps,
 * the tree's kernel and options, outputs to scratch) with each walk schedule
 * -- 1, 2 and 4 queries per warp (4 is skipped under pruning) -- after one
 * untimed run of each, and keeps the fastest in the tree's options
 * (mlods_params.queries_per_warp), which every later single-tree projection
 * uses.  *chosen receives it; ms (may be NULL) the three device times in
 * milliseconds (-1 for a skipped one).  The results of the schedules agree to
 * float rounding.  Synchronises. */
int mlods_tune_schedule(mlods_tree t, int64_t n, const float* d_q, int32_t n_iterations, void* stream,
                        int32_t* chosen, float* ms);
/* The same on n host queries (xyz floats), staged in library scratch memory. */
int mlods_tune_schedule_host(mlods_tree t, int64_t n, const float* q, int32_t n_iterations, int32_t* chosen,
                             float* ms);

/* ---- neighbour gathers -----------------------------------------------------
 * k nearest neighbours of n device query points (world xyz), as the
 * reference kd-tree's knearest (kdTreeNN.h:416-461, :590-600) which
 * APSSOctree::knnMode uses: squared distances evaluated in float exactly as
 * the kd-tree does, so the sets are equal except at exact distance ties at
 * the k-th place (resolved here to the lower point index).  Rows are sorted
 * by (distance, index); d_idx holds original point indices (-1 past the
 * point count).  k <= MLODS_MAX_KNN.  Asynchronous. */
#define MLODS_MAX_KNN 32
int mlods_knn(mlods_tree t, int64_t n, const float* d_q, int32_t k, int32_t* d_idx, float* d_d2, void* stream);
/* The same with host arrays (APSSOctree::getKnn / cpuSphere, CPUUtils.cpp:638-672);
 * synchronous. */
int mlods_knn_host(mlods_tree t, int64_t n, const float* q, int32_t k, int32_t* idx, float* d2);

/* ---- dual contouring --------------------------------------------------------
 * Cells are octree nodes (depth, x, y, z) as octree_id (octree.h:18-44) over
 * the unit cube; their corners sit on the integer lattice of the deepest
 * level, max_depth.
 *
 * mlods_dcgrid_from_points builds the DC grid of the reference's `-b` path:
 * OctreeGenerator::generateFromPoints (upsample.cpp:128-144: the cells at
 * max_depth enclosing the points inside [box_min, box_max], the reference uses
 * [-1,1]^3) followed by uniformizeFromPoints (upsample.cpp:253-260: grade,
 * regularize_up, regularize_siblings), cells in sorted_octree order
 * (node_comparator, octree.h:147-154).  Host code. */
typedef struct mlods_dcgrid_s* mlods_dcgrid;
int mlods_dcgrid_from_points(const float* pts, int64_t n, int32_t max_depth, const float* box_min,
                             const float* box_max, mlods_dcgrid* out);
/* The same grid with its set work on the device (keys, radix sort, unique,
 * the grade and regularize steps level by level); pts may be in host or
 * device memory.  Falls back to the host code for max_depth > 15 or points
 * whose cells lie beyond 2^19 cells from the box.  Synchronous on `stream`. */
int mlods_dcgrid_from_points_device(const float* pts, int64_t n, int32_t max_depth, const float* box_min,
                                    const float* box_max, void* stream, mlods_dcgrid* out);
int mlods_dcgrid_info(mlods_dcgrid g, int64_t* n_cells, int32_t* max_depth);
int mlods_dcgrid_cells(mlods_dcgrid g, int32_t* cells);  /* 4 int32 per cell */
int mlods_dcgrid_free(mlods_dcgrid g);
/* The projection-driven grid of the reference's default mode
 * (OctreeGenerator::generate + uniformize, upsample.cpp:228-273): cell
 * centres projected level by level with the tree's projection (one step, no
 * step limit), kept where the projection lands, refined with their
 * neighbours, then graded and regularised; cut != 0 drops cells deeper than
 * max_depth.  The grid's unit frame maps to the tree's frame by the 3x4
 * matrix mlods_dcgrid_xform returns (new2bbox, scene.cpp:1311); for
 * mlods_dcgrid_from_points it is the map of the given box. */
int mlods_dcgrid_adaptive(mlods_tree t, int32_t max_depth, int32_t cut, void* stream, mlods_dcgrid* out);
int mlods_dcgrid_xform(mlods_dcgrid g, float* xform, int64_t* n_projected);

/* Signed field at the 8 corners of every cell and the per-cell vertex
 * (scene.cpp:1346-1394, dual_contouring.h:124-176).  xform is the 3x4
 * row-major map from the unit cube to the tree's frame (the top rows of
 * new2bbox, scene.cpp:1313).  Every unique corner is projected once (one MLoD
 * iteration with the tree's kernel and options); corner_f[8 c + k] =
 * (corner - projection).normal, NaN when the projection failed.  vertex[3 c]
 * is the cell's vertex in the unit cube and n_cross[c] its number of edge
 * crossings: with use_normals = 0 the reference's zero normal field, i.e. the
 * mass point of the crossings (the cell centre without crossings); with
 * use_normals = 1 a full QEF on the interpolated projected normals, solved in
 * double (extension).  Host arrays in and out; synchronous. */
int mlods_dc_evaluate(mlods_tree t, int64_t n_cells, const int32_t* cells, int32_t max_depth, const float* xform,
                      int32_t use_normals, float* corner_f, float* vertex, int32_t* n_cross,
                      int64_t* n_unique_corners, void* stream);
/* The same with the cells and the three outputs in device memory (xform stays
 * a host array): nothing crosses the host link but the 12-float map and the
 * unique-corner count.  Returns when the outputs are written. */
int mlods_dc_evaluate_device(mlods_tree t, int64_t n_cells, const int32_t* d_cells, int32_t max_depth,
                             const float* xform, int32_t use_normals, float* d_corner_f, float* d_vertex,
                             int32_t* d_n_cross, int64_t* n_unique_corners, void* stream);

/* ---- mesh extraction and refinement (dual_contouring.h:59-87, scene.cpp:1396-1452) ----
 * mlods_dc_extract builds the dual-contouring mesh of a grid (cells sorted as
 * mlods_dcgrid_cells gives them) from its corner values and per-cell vertices
 * (as mlods_dc_evaluate returns them): minimal edges enumerated in the
 * reference's order (minimal_edges::traverse, octree.h:400-540), two
 * triangles per sign-changing edge, vertices numbered on first use, vertex
 * positions in the grid's unit frame.  Runs on the host, no GPU needed.
 * mlods_mesh_transform applies a 3x4 map, mlods_mesh_smooth and
 * mlods_mesh_subdivide are mesh::smoothMesh / mesh::subdivideMesh
 * (upsample.h:55-133), mlods_mesh_project projects the vertices in place
 * (positions and normals).  mlods_dc_mesh runs the whole reference pipeline
 * on a grid: corner field, extraction, transform to the tree's frame,
 * projection (3 iterations), then refine_rounds x (smooth, subdivide,
 * project 3 iterations); the reference uses 2 rounds.
 * A mesh from mlods_dc_extract lives in host memory; one from mlods_dc_mesh
 * stays in device memory: the mesh functions then run on the device (the
 * same results in the same order), mlods_mesh_get copies it into the
 * caller's buffers (pinned buffers copy fastest), and
 * mlods_mesh_device_arrays gives its device arrays (float3 positions and
 * normals, uint3 triangles), valid until the mesh is changed or freed. */
typedef struct mlods_mesh_s* mlods_mesh;
int mlods_dc_extract(int64_t n_cells, const int32_t* cells, const float* corner_f, const float* cell_vertex,
                     mlods_mesh* out);
int mlods_mesh_info(mlods_mesh m, int64_t* n_vertices, int64_t* n_triangles);
int mlods_mesh_get(mlods_mesh m, float* vertices, float* normals, uint32_t* indices);
int mlods_mesh_device_arrays(mlods_mesh m, const float** vertices, const float** normals, const uint32_t** indices);
int mlods_mesh_transform(mlods_mesh m, const float* xform);
int mlods_mesh_smooth(mlods_mesh m);
int mlods_mesh_subdivide(mlods_mesh m);
int mlods_mesh_project(mlods_tree t, mlods_mesh m, int32_t n_iterations, void* stream);
int mlods_mesh_free(mlods_mesh m);
/* Host wall time (ms) of mlods_dc_mesh's 7 stages: corner field, extraction,
 * upload + transform, projections, smoothing, subdivision, download (0: the
 * mesh stays in device memory); zeros for meshes built otherwise. */
int mlods_mesh_stage_ms(mlods_mesh m, double* ms);
int mlods_dc_mesh(mlods_tree t, mlods_dcgrid g, int32_t use_normals, int32_t refine_rounds, void* stream,
                  mlods_mesh* out);

/* ---- per-launch statistics of the last projection on this tree ------------
 * node visits summed over queries and iterations, warp rounds (32 lanes each)
 * that evaluated them, largest traversal stack, queries whose traversal stack
 * overflowed (their result is the input point with a zero normal), and the
 * device time of the projection kernel itself in milliseconds (CUDA events on
 * the launching stream).  Any pointer may be NULL.  Synchronises. */
int mlods_last_stats(mlods_tree t, int64_t* node_visits, int64_t* rounds, int32_t* max_stack, int64_t* overflows,
                     float* kernel_ms);
/* Iterations the last MLoD projection on this tree ran, summed over its
 * queries: n x n_iterations, fewer under a convergence mode (each query
 * counts the iterations it evaluated).  After a kNN projection: the
 * iterations that searched the octree for their neighbours; the others kept
 * the previous iteration's k points, which the step provably left the k
 * nearest, and only ranked them again.  0 after a global or ball
 * projection.  Extension; synchronises. */
int mlods_last_iterations(mlods_tree t, int64_t* iterations);
/* Counters of the last MLoD projection on this tree.  lane_visits: node
 * evaluations, where a node that the queries of one warp's shared walk
 * (queries_per_warp = 2 or 4) all need is evaluated, and counted, once (equals
 * node_visits of mlods_last_stats with one query per warp).  pruned: nodes
 * that kernel-weight pruning (mlods_params.prune_tol) took as aggregates
 * instead of opening, per query.  Either pointer may be NULL.  Extension;
 * synchronises. */
int mlods_last_walk_counts(mlods_tree t, int64_t* lane_visits, int64_t* pruned);

/* ---- batched projection over many resident trees (extension) ---------------
 * No counterpart in the reference, which projects one tree per launch
 * (Fastapss::project, Fastapss.cu:439-455).  A batch holds a fixed list of
 * trees; mlods_batch_project projects, in ONE persistent kernel launch on one
 * stream (after the Morton ordering of the queries), the device query buffer
 * d_q (float xyz, concatenated per tree: tree i owns queries
 * [offsets[i], offsets[i+1]), offsets is a HOST array of n_trees + 1 entries
 * starting at 0) onto their trees, writing d_out_pts/d_out_nrm in the same
 * layout.  The launch's warps take a tree's queries one or two at a time from
 * a device counter, the trees with the most work first, and walk them with
 * the tree's own specialisation of the walk (kernel family and terms, blend
 * rule, queries per warp), so trees of any size and kernel share the launch.
 * Every tree must be in MLODS_MODE_MLOD with a kernel set; each tree's own
 * cutoff, min_depth, blend rule and convergence mode apply (pruning does not),
 * and the step clamp is each tree's root box radius.  Every tree is walked
 * with its own queries_per_warp (4 runs as 2) unless the schedule sets one
 * for all; results equal per-tree mlods_project_device calls with the same
 * schedule bit for bit.  With use_graph != 0 the work is captured once in a
 * CUDA graph and replayed while buffers, offsets, tree settings, schedule and
 * n_iterations stay the same (the stream must not be capturing).
 * mlods_batch_tune (the batch's autotuner) times, on the given buffers, a set
 * of schedules -- one or two queries per warp for every tree, Morton or input
 * order, the share of the resident grid, the order of the trees in the
 * launch, and launches of their own for the largest trees -- each run once
 * untimed and once timed, and keeps the fastest for later calls.  The trees
 * must outlive the batch and must not be rebuilt while it exists. */
typedef struct mlods_batch_s* mlods_batch;
/* The launch shape of a batch. */
typedef struct {
    int32_t queries_per_warp; /* 0: each tree's own setting (the largest of them, at most 2); else 1 or 2 for every tree */
    int32_t reorder;          /* 1: Morton order inside each tree; 0: input order */
    int32_t grid_pct;         /* share of the resident grid launched, 1-100 */
    int32_t line_order;       /* 0: the trees with the most work first; 1: grouped by walk specialisation */
    int64_t solo_min_queries; /* > 0: a tree with at least this many queries runs in a launch of its own
                                 (the single-tree kernel) before the shared launch of the others; 0: none */
} mlods_batch_schedule;
int mlods_batch_create(const mlods_tree* trees, int32_t n_trees, mlods_batch* out);
int mlods_batch_free(mlods_batch b);
int mlods_batch_project(mlods_batch b, const int64_t* offsets, const float* d_q, float* d_out_pts, float* d_out_nrm,
                        int32_t n_iterations, int32_t use_graph, void* stream);
int mlods_batch_tune(mlods_batch b, const int64_t* offsets, const float* d_q, float* d_out_pts, float* d_out_nrm,
                     int32_t n_iterations, void* stream);
/* Statistics of the last batch call (synchronises): query-node visits,
 * rounds, overflows, device time (ordering and kernels), node evaluations
 * (lane_visits, see mlods_last_walk_counts) and the kernel launches it made.
 * Any pointer may be NULL. */
int mlods_batch_stats(mlods_batch b, int64_t* node_visits, int64_t* rounds, int64_t* overflows, float* kernel_ms,
                      int64_t* lane_visits, int32_t* walk_launches);
/* The schedule in use / sets one without tuning. */
int mlods_batch_get_schedule(mlods_batch b, mlods_batch_schedule* out);
int mlods_batch_set_schedule(mlods_batch b, const mlods_batch_schedule* sched);
/* The candidates of the last mlods_batch_tune and the device time of each:
 * *n_candidates = their number; the first max_candidates are written to
 * cands and ms (either may be NULL). */
int mlods_batch_tune_results(mlods_batch b, int32_t max_candidates, mlods_batch_schedule* cands, float* ms,
                             int32_t* n_candidates);

/* ---- projection without device allocation (extension) ----------------------
 * No counterpart in the reference.  Same computation and results as
 * mlods_project_device (MLoD mode only; the tree's kernel, cutoff, min depth,
 * blend rule, query ordering and convergence mode apply), but the call
 * allocates no device memory: its scratch (query order, sort buffers, work
 * counter) lives in one fixed array of about 13 MB that the library's module
 * holds on each device, instead of the tree's lazily grown cudaMalloc buffer.
 * For callers that must not allocate at call time (fixed memory budget, an
 * allocator that owns the free memory, start-up-only footprint).
 *   - n is at most MLODS_NOALLOC_MAX_QUERIES per call; larger n returns
 *     MLODS_ERR_CAPACITY (split the batch).
 *   - The first call on a device does a one-time setup (it looks up the
 *     array's address; with CUDA's lazy module loading this is also when the
 *     array becomes resident); make it outside any stream capture.
 *   - All calls on a device share the array: calls that overlap in time
 *     (several streams or host threads) race and must be serialised.
 *   - mlods_last_stats does not report these calls. */
#define MLODS_NOALLOC_MAX_QUERIES 524288
int mlods_project_device_noalloc(mlods_tree t, int64_t n, const float* d_q, float* d_out_pts, float* d_out_nrm,
                                 int32_t n_iterations, float step_max, void* stream);

/* ---- projection server (extension) -----------------------------------------
 * No counterpart in the reference (one synchronous request at a time).  A
 * server keeps a fixed list of resident trees (MLoD mode, kernel set; their
 * settings must not change while it runs) and answers requests from any
 * host thread: mlods_server_submit queues n host query points for one tree
 * (optionally with their own weight kernel) and returns a ticket at once;
 * worker threads, one per CUDA stream, take what is queued whenever they
 * are free (up to max_batch_queries / max_batch_requests, optionally waiting
 * max_wait_us for more; in arrival order, passing over a request that only a
 * later batch can hold, and cutting one larger than a batch into pieces) and
 * project it with one launch of the queue kernel (every request or piece
 * walked with its own tree, kernel and iteration count); results are written
 * to out_pts / out_nrm (either may be NULL), identical to mlods_project_host
 * on the same tree and kernel (with two queries per warp a request cut into
 * pieces pairs its queries within each piece: equal to float rounding).  The
 * query and output arrays must stay valid until the ticket is waited for.
 * Memory admission, by device footprint: a batch in flight holds, in the
 * library's stream-ordered pool, 36 bytes of query / result buffers and
 * about 24 bytes of ordering scratch per query plus its per-request
 * arguments (mlods_server_batch_bytes gives the exact figure), and returns
 * them when it finishes; a worker forms its next batch only from what fits
 * max_device_bytes minus the batches already in flight, so requests are
 * taken up as batches finish and their memory frees up.  A submit whose
 * footprint (its device bytes when run, plus 36 bytes of pinned staging per
 * query) would take the queued work beyond max_pending_bytes returns
 * MLODS_ERR_CAPACITY.  mlods_server_wait blocks at most timeout_ms
 * (MLODS_ERR_TIMEOUT after that; wait again later), returns the request's
 * status and its latency from submit to results on the host, and retires the
 * ticket.  mlods_server_free cancels queued requests, lets running batches
 * finish and joins the workers. */
typedef struct mlods_server_config {
    int32_t n_streams;            /* worker threads / CUDA streams (default 2) */
    int32_t max_batch_requests;   /* requests per launch (default 4096) */
    int64_t max_batch_queries;    /* queries per batch at most (default 2^18; larger requests run in pieces) */
    int64_t max_device_bytes;     /* device memory the batches in flight may hold together; 0 (default):
                                     half the device memory free when the server is created */
    int64_t max_pending_bytes;    /* admission bound on the footprint of queued requests; 0 (default):
                                     eight times max_device_bytes */
    int32_t max_wait_us;          /* batching window when less than a batch is queued (default 0) */
    int32_t reserved;
} mlods_server_config;
typedef struct mlods_server_s* mlods_server;
void mlods_server_default_config(mlods_server_config* c);
int mlods_server_create(const mlods_tree* trees, int32_t n_trees, const mlods_server_config* cfg, mlods_server* out);
int mlods_server_submit(mlods_server s, int32_t tree, int64_t n, const float* q, float* out_pts, float* out_nrm,
                        int32_t n_iterations, const mlods_kernel* kernel, uint64_t* ticket);
int mlods_server_wait(mlods_server s, uint64_t ticket, int32_t timeout_ms, double* latency_ms);
int mlods_server_stats(mlods_server s, int64_t* completed, int64_t* batches, int64_t* queries, int64_t* queued,
                       double* busy_ms);
/* Device bytes the batches in flight hold now and at most so far, the
 * footprint of the queued requests, and the two budgets in force (after the
 * defaults are resolved).  Any pointer may be NULL. */
int mlods_server_memory(mlods_server s, int64_t* in_flight_bytes, int64_t* peak_in_flight_bytes,
                        int64_t* pending_bytes, int64_t* max_device_bytes, int64_t* max_pending_bytes);
/* Device bytes one batch of n_queries queries from n_requests requests (or
 * pieces) holds while in flight. */
int64_t mlods_server_batch_bytes(int64_t n_queries, int64_t n_requests);
int mlods_server_free(mlods_server s);

/* ---- point-set and parameter files (Pn.cpp:102-290, scene.cpp:1183-1250) --
 * mlods_cloud_load reads a .pn (raw float32 x y z nx ny nz records) or .ply
 * file (the vertex element's x, y, z and, when present, nx, ny, nz; ascii or
 * binary, any scalar type) and, with do_normalize, applies Pn::normalize:
 * positions become (p - offset) / norme with offset the mean point and norme
 * the largest coordinate of the box widened by 0.5% of its diagonal.
 * mlods_cloud_save writes p * norme + offset (offset may be NULL) as a
 * binary little-endian .ply (normals optional) or a .pn (normals required),
 * as Pn::save does.  mlods_cloud_normalize applies Pn::normalize to an
 * array.  The .params functions read and write the reference's parameter
 * file, a packed 134-byte sequence of the fields below in this order. */
typedef struct mlods_cloud_s* mlods_cloud;
int mlods_cloud_load(const char* path, int32_t do_normalize, mlods_cloud* out);
int mlods_cloud_info(mlods_cloud c, int64_t* n_points, int32_t* has_normals, float* offset, float* norme);
int mlods_cloud_get(mlods_cloud c, float* pts, float* nrm);
int mlods_cloud_free(mlods_cloud c);
int mlods_cloud_save(const char* path, const float* pts, const float* nrm, int64_t n, const float* offset,
                     float norme);
int mlods_cloud_normalize(const float* pts, int64_t n, float* out_pts, float* offset, float* norme);

/* Pn::order (Pn.cpp:388-440): perm receives the point indices sorted by
 * their Morton code on a grid^3 lattice over the points' cube (grid 64 in
 * the reference); equal codes keep their input order.
 * Pn::initialize(n, pointSetToFit, factor) (Pn.cpp:324-357): n_out queries,
 * each an input point moved inside the disk of radius meanGap of its tangent
 * plane, with the point's normal; seeded (the reference's draws are not). */
int mlods_cloud_morton_order(const float* pts, int64_t n, int32_t grid, uint32_t* perm);
int mlods_cloud_sample_around(const float* pts, const float* nrm, int64_t n_pts, int64_t n_out, float factor,
                              uint64_t seed, float* out_pts, float* out_nrm);

/* scene::generateFromOctree (scene.cpp:733-756), on the device: n_out points,
 * each in a cell drawn uniformly from d_cells (n_cells rows of int32
 * {depth, x, y, z} of the [-1, 1]^3 octree, 16-byte aligned), at the cell
 * centre plus an offset uniform in [-0.5, 0.5)^3 times 4 / 2^depth; the
 * normal is the point itself (d_out_nrm may be NULL).  Draws are a
 * counter-based hash of (seed, index), so a seed fixes the output.  A row
 * whose depth is outside [0, 30] yields a NaN point.  Asynchronous on
 * `stream`. */
int mlods_sample_cells_device(const int32_t* d_cells, int64_t n_cells, int64_t n_out, uint64_t seed,
                              float* d_out_pts, float* d_out_nrm, void* stream);

#define MLODS_PARAMS_FILE_BYTES 134
typedef struct mlods_scene_params {
    float cam_quat[4];          /* viewer camera (not used by the projection) */
    float cam_translation[3];
    float cam_dist;
    float sigma;                /* Kernel::sigma, in units of the box radius */
    float fixed_sigmas[5];      /* Kernel::fixedSigmas */
    float beginning_sigma;      /* Kernel::beginningSigma */
    float factor;               /* Kernel::factor */
    float constant_shift;       /* Kernel::constant_shift */
    float exponent;             /* Kernel::exponent */
    float cutoff;               /* scalingProtectionSphere */
    uint32_t n_computed_sigmas; /* Kernel::nbOfComputedSigmas */
    uint32_t max_iterations;    /* projection iterations */
    uint32_t max_depth;         /* DC / upsampling octree depth */
    uint32_t min_depth;         /* MLoD minimum depth */
    uint32_t fast_method;       /* 1: Fastapss (MLoD), 0: GlobalAPSS */
    int32_t kernel_type;        /* MLODS_GAUSSIAN / _SINGULAR / _GAUSSIAN_MULTIPLE */
    uint8_t computed_sigma;     /* 1: sigmas from beginning_sigma * factor^i, 0: fixed_sigmas */
    uint8_t cut;                /* uniformize's cut */
    uint32_t n_points;          /* queries per upsampling round */
    uint32_t max_upsamples;
    float offset[6];
} mlods_scene_params;
int mlods_params_file_load(const char* path, mlods_scene_params* p);
int mlods_params_file_save(const char* path, const mlods_scene_params* p);

/* Number of kernels this library has launched in this process (diagnostics). */
int64_t mlods_kernel_launches(void);

/* Per-call scratch (DC corner fields, grid generation, split global APSS)
 * comes from a stream-ordered memory pool owned by the library, one per
 * device, which keeps up to 8 GiB of freed scratch for the next calls.
 * mlods_release_scratch returns the current device's unused pooled memory to
 * the system (extension; synchronises the device first). */
int mlods_release_scratch(void);

#ifdef __cplusplus
}
#endif

#endif /* MLODS_H */
