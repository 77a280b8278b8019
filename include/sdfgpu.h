/*
 * sdfgpu.h -- C ABI of libsdfgpu.so, the B200 (sm_100a) implementation of the SignedDistances
 * hot path of stl2sdf.jl: the truncated unsigned distance from every grid node to a triangle
 * mesh and the ray-cast inside/outside sign.
 *
 * Reference interfaces replaced (paths relative to the stl2sdf.jl project):
 *   evalDistancesOnTriMesh(mesh, grid, points) -> (dist, xp)
 *       src/SignedDistances/dfOnTriangularMesh.jl:19        -> sdfgpu_distances
 *   raycast_sign_detection(mesh, grid, points; min_rays=6, max_rays=30,
 *                          confidence_threshold=0.6, use_winding_fallback=true)
 *       src/SignedDistances/RaycastingSignDetection.jl:337  -> sdfgpu_signs
 *   sdf_dists = dists .* signs
 *       src/stl_to_sdf.jl:119                              -> sdfgpu_sdf (fused)
 *   TriangularMesh(X, IEN)
 *       src/MeshGrid/MeshInformations.jl:68                -> sdfgpu_set_mesh
 *   Grid(AABB_min, AABB_max, N_max, margineCells)
 *       src/MeshGrid/Grid.jl:9                             -> sdfgpu_grid_setup
 *   noninteractive_sdf_grid_setup(mesh, B)
 *       src/MeshGrid/Grid_setup.jl:104                     -> sdfgpu_grid_from_cell_size
 *   analyze_mesh(calculate_edge_distances(mesh))
 *       src/MeshGrid/Grid_setup.jl:28,64                   -> sdfgpu_mesh_edge_stats
 *   process_stl_mesh(vertices, triangles)
 *       src/DataImport/ImportStlData.jl:198                -> sdfgpu_stl_dedupe
 *   remove_sdf_artifacts!(sdf, grid; threshold, min_component_ratio)
 *       src/SignedDistances/SdfArtifactRemoval.jl:134      -> sdfgpu_remove_artifacts
 *   analyze_sdf_components(sdf, grid; threshold)
 *       src/SignedDistances/SdfArtifactRemoval.jl:259      -> sdfgpu_sdf_components
 *   RBFs_smoothing(dist, grid, is_interpolation, smooth, threshold)
 *       src/SdfSmoothing/RBFs4Smoothing.jl:275              -> sdfgpu_rbf_smoothing
 *
 * Conventions
 *   - Grid nodes are implicit: node (i, j, k), 0 <= i <= N[0] etc., sits at
 *     origin + h * [i, j, k] (one multiply and one add per component, no FMA, as Grid.jl:90),
 *     and its linear index is i + (N[0]+1) * (j + (N[1]+1) * k) (x fastest, Grid.jl:87-89).
 *     origin is the padded AABB_min of the reference Grid and h its cell_size.
 *   - X is the reference's 3 x nnp column-major Float64 matrix (vertex-major: x,y,z of vertex
 *     1, then vertex 2, ...).  IEN is the 3 x nel column-major Int64 matrix of 1-based indices.
 *   - The caller owns every host buffer passed in or out; the library owns the device memory
 *     held by a context.  Output buffers hold ngp = prod(N+1) doubles (xp: 3*ngp).
 *   - Every entry point returns an sdfgpu_status; 0 is success.  sdfgpu_last_error() gives the
 *     message of the last failure on that context.
 *   - A context is bound to one CUDA device and is not thread safe: use one host thread per
 *     context.  Host-buffer calls return after the results are in the host buffers.
 *   - Sign convention of the reference: +1 inside, -1 outside.
 */
#ifndef SDFGPU_H
#define SDFGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDFGPU_ABI_VERSION 1

typedef struct sdfgpu_ctx sdfgpu_ctx;

typedef enum sdfgpu_status {
  SDFGPU_OK = 0,
  SDFGPU_ERR_INVALID_ARGUMENT = 1,
  SDFGPU_ERR_NO_DEVICE = 2,
  SDFGPU_ERR_CUDA = 3,
  SDFGPU_ERR_OUT_OF_MEMORY = 4,
  SDFGPU_ERR_NO_MESH = 5,
  SDFGPU_ERR_CAPACITY = 6, /* a bounded per-thread buffer or traversal stack overflowed */
  SDFGPU_ERR_IO = 7
} sdfgpu_status;

typedef enum sdfgpu_distance_mode {
  /* The reference's rule (dfOnTriangularMesh.jl:79-177): candidates are the triangles whose
   * centroid lies within 2.5*cell_size (else the triangles of the 3 nearest vertices), folded in
   * ascending triangle index with the reference's vertex-skip rule, then clamped to cell_size. */
  SDFGPU_MODE_REF_RULE = 0,
  /* True point-triangle minimum over all triangles, clamped to cell_size. */
  SDFGPU_MODE_EXACT = 1,
  /* True point-triangle minimum over all triangles, not clamped (a full unsigned distance). */
  SDFGPU_MODE_UNBOUNDED = 2,
  /* SDFGPU_MODE_UNBOUNDED searched with the learned radius of the current mesh (train it first with
   * sdfgpu_train_radius): the same bits as SDFGPU_MODE_UNBOUNDED.  No reference counterpart. */
  SDFGPU_MODE_LEARNED = 3
} sdfgpu_distance_mode;

typedef struct sdfgpu_opts {
  int32_t device;  /* CUDA device ordinal */
  int32_t tile[3]; /* nodes per distance tile along x, y, z; 0 = default / autotuned */
} sdfgpu_opts;

/* Counters of the last sdfgpu_distances / sdfgpu_signs / sdfgpu_sdf call. */
typedef struct sdfgpu_stats {
  int64_t ngp;                    /* grid nodes of the call */
  int64_t nel;                    /* triangles of the mesh */
  int64_t tile_pairs;             /* (tile, triangle) candidate pairs */
  int64_t active_tiles;           /* tiles with at least one candidate */
  int64_t candidate_nodes;        /* nodes whose candidate set was non-empty */
  int64_t fp64_evals;             /* FP64 point-triangle evaluations (near-tie band) */
  int64_t knn_fallback_nodes;     /* nodes resolved by the 3-nearest-vertex fallback */
  int64_t band_nodes;             /* nodes flagged within cell_size by the band scatter */
  int64_t row_hits;               /* axis-ray (row, triangle) hits */
  int64_t undecided_nodes;        /* nodes whose 6 axis rays disagreed */
  int64_t extra_rays;             /* rays cast beyond the 6 axis rays */
  int64_t winding_nodes;          /* nodes that took the winding-number fallback */
  int64_t winding_ambiguous;      /* winding nodes with | |w| - 0.5 | < 1e-9 */
  int64_t unbounded_fallbacks;    /* learned-radius nodes that fell back to unbounded search */
  double rho_max;                 /* max vertex distance from a triangle centroid */
  double ms_distance;             /* device time of the distance stage (ms) */
  double ms_sign;                 /* device time of the sign stage (ms) */
  double ms_mesh;                 /* device time of the last set_mesh up to the triangle records (ms); the LBVH
                                     build runs beside the next call's distance stage */
  int64_t launches;               /* kernels of this library launched by the last call (CUB excluded) */
  int64_t mesh_launches;          /* same, for the last set_mesh */
  double ms_tiles;                /* (tile, triangle) pair build + sort */
  double ms_fold;                 /* tile fold kernel (the distance hot loop) */
  double ms_rows;                 /* axis-row hit lists (count, fill, sort) */
  double ms_parity;               /* the three axis-parity kernels */
  double ms_vote;                 /* vote + adaptive rays + winding */
  int64_t certified_nodes;        /* learned radius: nodes whose bounded search certified the result */
  double radius_loss;             /* final training loss of the radius network */
  int64_t bvh_visits;             /* LBVH nodes visited by the unbounded search (one per warp and node) */
  double ms_train;                /* device time of the last sdfgpu_train_radius (coarse grid + training) */
  int64_t train_launches;         /* kernels of this library launched by the last sdfgpu_train_radius */
  int64_t sign_band_reruns;       /* axis-row ray-triangle tests decided in FP64 (FP32 result inside its error band) */
} sdfgpu_stats;

/* Context lifetime.  opts may be NULL (device 0, default tiles). */
int sdfgpu_create(const sdfgpu_opts* opts, sdfgpu_ctx** out);
int sdfgpu_destroy(sdfgpu_ctx* ctx);
/* Message of the last failure on ctx, or of the last failed sdfgpu_create when ctx is NULL. */
const char* sdfgpu_last_error(const sdfgpu_ctx* ctx);
int sdfgpu_abi_version(void);

/* Grid constructor (Grid.jl:9-32).  Writes the padded origin (AABB_min), the adjusted AABB_max,
 * N (cells per axis), cell_size and ngp = prod(N+1).  Host arithmetic only; no device needed. */
int sdfgpu_grid_setup(const double xmin[3], const double xmax[3], int64_t n_max, int64_t margin,
                      double origin[3], double aabb_max[3], int64_t N[3], double* cell_size,
                      int64_t* ngp);
/* noninteractive_sdf_grid_setup (Grid_setup.jl:104-124): N_new = floor(max extent / B),
 * margin 3, over the vertex bounding box of X (3 x nnp). */
int sdfgpu_grid_from_cell_size(const double* X, int64_t nnp, double B, double origin[3],
                               double aabb_max[3], int64_t N[3], double* cell_size, int64_t* ngp);

/* TriangularMesh (MeshInformations.jl:68-83): uploads X (3 x nnp) and IEN (3 x nel, 1-based),
 * validates the indices, prepares the per-triangle data (dfOnTriangularMesh.jl:329-368) and
 * builds the LBVH.  The mesh stays resident until the next set_mesh or destroy. */
int sdfgpu_set_mesh(sdfgpu_ctx* ctx, const double* X, int64_t nnp, const int64_t* IEN, int64_t nel);
/* Same, with X and IEN already in device memory of the context's device. */
int sdfgpu_set_mesh_device(sdfgpu_ctx* ctx, const double* d_X, int64_t nnp, const int64_t* d_IEN,
                           int64_t nel);

/* evalDistancesOnTriMesh (dfOnTriangularMesh.jl:19-209) over the implicit grid.
 * dist_out: ngp doubles; xp_out: 3*ngp doubles (closest points, vertex-major) or NULL.
 * mode: sdfgpu_distance_mode.  use_learned_radius: only with SDFGPU_MODE_UNBOUNDED (0 or 1). */
int sdfgpu_distances(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3],
                     double* dist_out, double* xp_out, int32_t mode, int32_t use_learned_radius);

/* raycast_sign_detection (RaycastingSignDetection.jl:337-404) over the implicit grid.
 * sign_out: ngp doubles (+1 inside, -1 outside); conf_out: ngp doubles or NULL. */
int sdfgpu_signs(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3],
                 int32_t min_rays, int32_t max_rays, double confidence_threshold,
                 int32_t use_winding_fallback, double* sign_out, double* conf_out);

/* Fused stl_to_sdf.jl:105-119: distances, signs and sdf = dist .* sign in one call.  Any output
 * pointer may be NULL except sdf_out. */
int sdfgpu_sdf(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int32_t mode,
               int32_t min_rays, int32_t max_rays, double confidence_threshold,
               int32_t use_winding_fallback, double* sdf_out, double* dist_out, double* sign_out,
               double* conf_out);
/* Same as sdfgpu_sdf with every output pointer in device memory; returns once the work is
 * enqueued on the context's stream (see sdfgpu_get_stream) and the bounded host-side sizing
 * reads are done.  The outputs are valid after that stream synchronizes. */
int sdfgpu_sdf_device(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3],
                      int32_t mode, int32_t min_rays, int32_t max_rays,
                      double confidence_threshold, int32_t use_winding_fallback, double* d_sdf,
                      double* d_dist, double* d_sign, double* d_conf);

/* z-slab of sdfgpu_sdf: only the z layers k0..k1 (0 <= k0 <= k1 <= N[2]) of the grid
 * (origin, h, N), written as an (N[0]+1) x (N[1]+1) x (k1-k0+1) block, x fastest.  Every value
 * equals the value of the same node in the full-grid call (nodes stay origin + h * global index),
 * so slabs computed on different GPUs concatenate along z into the full field.  This is how a grid
 * of more than 2^31-1 nodes is computed, and how z-slab sharding splits one grid across ranks. */
int sdfgpu_sdf_slab(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int64_t k0,
                    int64_t k1, int32_t mode, int32_t min_rays, int32_t max_rays,
                    double confidence_threshold, int32_t use_winding_fallback, double* sdf_out,
                    double* dist_out, double* sign_out, double* conf_out);
/* Same with device output pointers, as sdfgpu_sdf_device. */
int sdfgpu_sdf_slab_device(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3],
                           int64_t k0, int64_t k1, int32_t mode, int32_t min_rays, int32_t max_rays,
                           double confidence_threshold, int32_t use_winding_fallback, double* d_sdf,
                           double* d_dist, double* d_sign, double* d_conf);

/* Allocation-free distances.  No counterpart in the reference: it exists for callers that must
 * not allocate GPU memory -- code running inside a host callback or an allocator hook, processes
 * whose device memory belongs to another framework's pool, or real-time loops that cannot take the
 * allocator's locks.  Every other entry point allocates its scratch on first use; this one keeps
 * its only scratch (the per-triangle records) in a fixed device array of about 5.8 MB that every
 * GPU loading the library holds until the process exits, and calls no allocator.
 *   d_X (3 x nnp), d_IEN (3 x nel, 1-based) and d_dist_out (ngp doubles) are device memory of the
 *   current device; mode is SDFGPU_MODE_EXACT or SDFGPU_MODE_UNBOUNDED; stream may be NULL.
 *   At most 16384 triangles, and at most 2^36 (node, triangle) pairs: the work is one FP64 step
 *   per pair (SDFGPU_ERR_CAPACITY beyond either).  The result equals sdfgpu_distances in the same
 *   mode.  The call synchronizes `stream` before it returns, so it must not be made while that
 *   stream is being captured.  Errors go to sdfgpu_last_error(NULL); when IEN holds an index
 *   outside 1..nnp, d_dist_out is left as it was.  Every call reuses the same array: calls that
 *   overlap on the GPU race, so serialise them. */
int sdfgpu_distances_noalloc(const double* d_X, int64_t nnp, const int64_t* d_IEN, int64_t nel,
                             const double origin[3], double h, const int64_t N[3], int32_t mode,
                             double* d_dist_out, void* stream);

/* One mesh of a batch: the mesh (host X 3 x nnp, IEN 3 x nel 1-based), its grid (origin, h, N) and
 * the host output buffer sdf (ngp doubles; dist/sign/conf optional, NULL to skip). */
typedef struct sdfgpu_batch_item {
  const double* X;
  int64_t nnp;
  const int64_t* IEN;
  int64_t nel;
  double origin[3];
  double h;
  int64_t N[3];
  double* sdf;
  double* dist;
  double* sign;
  double* conf;
} sdfgpu_batch_item;

/* stl_to_sdf's hot path (stl_to_sdf.jl:105-119) over many meshes, each with its own grid.  No
 * single reference call does this; it is the batched form of sdfgpu_set_mesh + sdfgpu_sdf.
 * `streams` worker contexts on the device of ctx (0 = 8), each with its own stream and host thread,
 * take meshes from a shared queue, largest estimated work (ngp * log2(nel)) first, so small and
 * large meshes overlap on the GPU.  With autotune = 1 each size class (log4 of ngp, log4 of nel)
 * gets its tile from sdfgpu_autotune the first time it appears; the choice is kept in ctx for later
 * calls.  Results equal per-mesh sdfgpu_sdf calls.  ctx's own mesh is left as it was; ctx's stats
 * become the sums over the items (rho_max: the maximum; ms_*: summed per-item device times).
 * Returns the first failure; its message names the item. */
int sdfgpu_sdf_batch(sdfgpu_ctx* ctx, sdfgpu_batch_item* items, int64_t count, int32_t mode, int32_t min_rays,
                     int32_t max_rays, double confidence_threshold, int32_t use_winding_fallback, int32_t streams,
                     int32_t autotune);

/* sdfgpu_sdf_batch with the choice of how the batch runs (results are the same either way).
 * persistent = 0: each item runs the whole per-mesh pipeline on one of the worker streams
 * (sdfgpu_sdf_batch does this).  persistent = 1: the workers first prepare every item (mesh, LBVH,
 * the sign stage, and the distance stage up to its last kernel: the tile lists of the reference-rule
 * and h-bounded modes; the search arguments and, in the learned mode, the radius network and the
 * radius of every warp brick of the unbounded and learned modes) in item-private buffers; then one
 * CUDA graph runs the distance kernels of all items in a single persistent launch -- the folds,
 * CTAs striding over the batch's (item, tile) work list, every item with its own tile; or the
 * searches, warps taking (item, brick) work items from one queue, with a second launch for the
 * bricks the learned radius did not certify -- followed by each item's nearest-vertex fallback and
 * combine on the worker streams side by side; then the fields are copied out.  Items go to the
 * workers by a fixed longest-processing-time assignment, so repeated batches reuse their buffers.
 * With mode = SDFGPU_MODE_LEARNED every mesh gets its own radius network, trained right after its
 * LBVH with the options of the last sdfgpu_train_radius on ctx (defaults: 50 steps, batch 2048,
 * learning rate 5e-3, seed 0) and ctx's search margin (sdfgpu_set_radius_margin) on a coarse grid of
 * min(24, K / 2) nodes on its longest axis (at least 16), K the nodes on the longest axis of the
 * mesh's own grid; results equal SDFGPU_MODE_UNBOUNDED. */
int sdfgpu_sdf_batch_ex(sdfgpu_ctx* ctx, sdfgpu_batch_item* items, int64_t count, int32_t mode, int32_t min_rays,
                        int32_t max_rays, double confidence_threshold, int32_t use_winding_fallback, int32_t streams,
                        int32_t autotune, int32_t persistent);

/* Tile autotuner for the distance stage (the reference has no counterpart).  Times the current mesh
 * on the grid (origin, h, N) in `mode` with each built-in tile shape (nodes per CTA along x, y, z:
 * 4x4x4, 8x4x2, 4x4x2, 8x4x4, 4x4x8, 8x8x4), keeps the fastest as ctx's tile and writes it to
 * tile_out and its device time to ms_out (either may be NULL).  In SDFGPU_MODE_UNBOUNDED, which
 * has no tiles, it times the warp bricks instead (the 32 nodes one warp searches together:
 * 4x2x4, 4x4x2, 2x4x4, 8x4x1, 4x8x1, 32x1x1) and keeps the fastest as ctx's brick.  Neither shape
 * changes a result, only how the work is split. */
int sdfgpu_autotune(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int32_t mode,
                    int32_t tile_out[3], double* ms_out);

/* Learned search radius for SDFGPU_MODE_UNBOUNDED (an extension of the reference's distance
 * search; no reference counterpart).  A 3 x 64 Fourier-feature MLP (FP16 weights, FP32
 * accumulate) is trained on the GPU on the exact unbounded distances of a coarse grid of the current
 * mesh (coarse_n - 1 cells on the longest axis of the mesh box, padded by one cell).  sdfgpu_distances
 * with use_learned_radius = 1 (or SDFGPU_MODE_LEARNED) then predicts a radius at the centre c of
 * every warp brick and starts the search of each node p of the brick from r(c) + |p - c|; a node
 * that finds a triangle inside that bound is certified exact, the bricks with other nodes are
 * searched again without it (stats: certified_nodes, unbounded_fallbacks).  Results are
 * bit-identical to the plain unbounded mode.  With the default margin, coarse_n = 24 and 50 Adam
 * steps of 2,048 samples at lr 5e-3 certify every node of 1.4M- and 5.7M-triangle meshes (3 ms of
 * training); longer training changes the search time by less than 1%. */
int sdfgpu_train_radius(sdfgpu_ctx* ctx, int32_t coarse_n, int32_t steps, int32_t batch, float lr, uint64_t seed,
                        float* final_loss);
/* Warp brick of the unbounded search: the nodes (brick[0] x brick[1] x brick[2] along x, y, z,
 * product 32) whose nearest triangles one warp searches together.  Default 4 x 2 x 4. */
int sdfgpu_set_brick(sdfgpu_ctx* ctx, const int32_t brick[3]);
/* Margin of the learned radius: r = (dhat (1 + alpha) + beta * coarse spacing / s) * s at a brick
 * centre, where dhat is the network's normalised distance and s its normalisation scale.  Defaults alpha = 0.5, beta = 4.
 * A smaller margin prunes more and certifies fewer nodes; results never change.  alpha = +inf makes
 * every radius infinite: the learned mode's search without the network's bound (to measure what the
 * network gains). */
int sdfgpu_set_radius_margin(sdfgpu_ctx* ctx, float alpha, float beta);
/* Number of FP32 parameters of the radius network (layout: W1 64x32, b1, W2 64x64, b2, W3 64x64,
 * b3, w4 64, b4). */
int sdfgpu_radius_param_count(void);
/* Read / replace the network: params (param_count floats, FP32 masters) and the normalisation
 * norm = {cx, cy, cz, s} of x = (p - c) / s. */
int sdfgpu_radius_params(sdfgpu_ctx* ctx, float* params, double norm[4]);
int sdfgpu_set_radius_params(sdfgpu_ctx* ctx, const float* params, const double norm[4]);
/* Network output dhat (normalised distance) at B normalised points xn (B x 3, host), evaluated by
 * the tensor-core inference kernel. */
int sdfgpu_radius_eval(sdfgpu_ctx* ctx, const float* xn, int64_t B, float* dhat);
/* The training forward and backward of the network at host params over B samples (host): dhat,
 * the loss and the FP32 parameter gradient (any output may be NULL).  Used to check the GPU
 * gradients against a CPU implementation. */
int sdfgpu_mlp_train_eval(sdfgpu_ctx* ctx, const float* params, const float* xn, const float* target, int64_t B,
                          float* dhat, float* loss, float* grad);

/* Edge-length statistics of the resident mesh, the analysis that calculate_edge_distances and
 * analyze_mesh (src/MeshGrid/Grid_setup.jl:28-102) print before the grid step is chosen.  Edge i of
 * a triangle runs from its vertex i to vertex i+1 (wrapping); lengths are FP64 norms of the vertex
 * differences.  out[0] shortest edge, out[1] longest edge, out[2] mean edge length, out[3] median
 * edge length (mean of the two middle values for an even count), out[4] / out[5] mean edge length
 * of the triangle with the smallest / largest sum of edge lengths; idx_out (may be NULL) receives
 * those two triangles' 0-based indices (the first one on ties, as Julia's argmin / argmax).
 * Returns after the results are in out. */
int sdfgpu_mesh_edge_stats(sdfgpu_ctx* ctx, double out[6], int64_t idx_out[2]);

/* Vertex deduplication of the STL import, process_stl_mesh (src/DataImport/ImportStlData.jl:198-309).
 * V holds the nv = 3 * nel vertices of the STL in stream order (x, y, z of each; triangle e is rows
 * 3e, 3e+1, 3e+2).  Writes the unique vertices to X_out (room for nv rows of 3 doubles; *nnp_out
 * rows used) in order of first appearance, and to IEN_out (nv entries) the 1-based index of every
 * stream vertex, i.e. the 3 x nel triangle matrix.  Equal vertices merge (-0.0 equals +0.0).
 * *near_out receives the number of ordered pairs of distinct unique vertices closer than 1e-10
 * (norm): when it is zero the result is the reference's; otherwise the reference's order-dependent
 * tolerance merge differs from exact deduplication and the caller must apply it.  Non-finite
 * vertices, or coordinates whose hash cell floor(x * 1e10) is not an Int64, are errors (the
 * reference throws for them too).  Returns after the results are in the host buffers. */
int sdfgpu_stl_dedupe(sdfgpu_ctx* ctx, const double* V, int64_t nv, double* X_out, int64_t* IEN_out,
                      int64_t* nnp_out, int64_t* near_out);

/* remove_sdf_artifacts!(sdf, grid; threshold, min_component_ratio)
 * (src/SignedDistances/SdfArtifactRemoval.jl:134-248), in place on the sdf of the grid with N cells
 * per axis (ngp = prod(N+1) doubles, x fastest).  Interior nodes are sdf >= threshold; their
 * 6-connected components smaller than max(1, round(min_component_ratio * largest)) (round to
 * nearest, ties to even, as Julia's round(Int, x)), other than the largest, get sdf = -|sdf|.
 * Writes the number of flipped nodes, of interior components and the size of the largest (any may
 * be NULL).  Ties for the largest component go to the one with the smallest node index (they matter
 * only for min_component_ratio > 1).  Needs no mesh.  sdf is host memory here and device memory of
 * the context's device in the _device form (which runs on the context's stream and returns after
 * it has finished). */
int sdfgpu_remove_artifacts(sdfgpu_ctx* ctx, const int64_t N[3], double* sdf, double threshold,
                            double min_component_ratio, int64_t* flipped, int64_t* components, int64_t* largest);
int sdfgpu_remove_artifacts_device(sdfgpu_ctx* ctx, const int64_t N[3], double* d_sdf, double threshold,
                                   double min_component_ratio, int64_t* flipped, int64_t* components,
                                   int64_t* largest);
/* analyze_sdf_components(sdf, grid; threshold) (SdfArtifactRemoval.jl:259-318): root_out (ngp
 * int32, may be NULL) receives for every interior node the smallest linear index of its component
 * (the component's label) and -1 for exterior nodes; also the component count and largest size. */
int sdfgpu_sdf_components(sdfgpu_ctx* ctx, const int64_t N[3], const double* sdf, double threshold, int32_t* root_out,
                          int64_t* components, int64_t* largest);

/* RBFs_smoothing(dist, grid, is_interpolation, smooth, threshold) (src/SdfSmoothing/RBFs4Smoothing.jl:275-320):
 * Gaussian RBFs of width cell_size, cut off where exp(-(r/cell_size)^2) <= threshold, centred on the
 * nodes of the grid (aabb_min, aabb_max, N), with weights from conjugate gradients on K w = dist
 * (interpolation = 1) or w = dist (interpolation = 0), evaluated on the grid refined `smooth` times
 * per axis (fine_out: prod(N*smooth+1) floats, x fastest, Float32 like the reference's result).
 * aabb_max is the grid's adjusted AABB_max (origin + N * cell_size).  weights_out (ngp floats),
 * cg_iterations and cg_residual (final |r|) may be NULL.  CG stops as IterativeSolvers.cg does, at
 * |r| <= sqrt(eps(Float32)) |dist|.  Needs no mesh. */
int sdfgpu_rbf_smoothing(sdfgpu_ctx* ctx, const double aabb_min[3], const double aabb_max[3], const int64_t N[3],
                         double cell_size, const double* dist, int32_t interpolation, int32_t smooth, double threshold,
                         float* fine_out, float* weights_out, int32_t* cg_iterations, double* cg_residual);

/* The cudaStream_t every kernel of the context runs on. */
int sdfgpu_get_stream(sdfgpu_ctx* ctx, void** stream);
int sdfgpu_get_stats(const sdfgpu_ctx* ctx, sdfgpu_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* SDFGPU_H */
