// common.cuh -- context, device buffers, error handling and shared launch helpers of libsdfgpu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "exact64.cuh"
#include "geom32.cuh"
#include "radius.cuh"
#include "sdfgpu.h"

namespace sdfgpu {

// LBVH node: the boxes of both children (mesh-local FP32, rounded outward) and their ids.
// A child id with the top bit set is a leaf: (id & 0x7fffffff) indexes the sorted primitives.
struct __align__(16) BNode {
  float4 a;  // lmin.x lmin.y lmin.z lmax.x
  float4 b;  // lmax.y lmax.z rmin.x rmin.y
  float4 c;  // rmin.z rmax.x rmax.y rmax.z
  int4 d;    // left, right, parent, unused
};
constexpr int32_t kLeafBit = (int32_t)0x80000000;
// Child subtrees of 2..kObbMaxLeaves leaves carry an oriented box (OBox, "obb" buffer) besides
// their axis-aligned one; above this size a patch is no longer flat and the box would not pay.
constexpr int kObbMaxLeaves = 4096;

// Device counters (int64) zeroed at the start of every grid call.
enum Counter : int {
  C_TILE_PAIRS = 0,
  C_ACTIVE_TILES,
  C_CAND_NODES,
  C_FP64,
  C_KNN,
  C_BAND,
  C_ROW_HITS,
  C_UNDECIDED,
  C_EXTRA_RAYS,
  C_WINDING,
  C_WIND_AMBIG,
  C_UNB_FALLBACK,
  C_ERR_CAPACITY,   // per-thread buffer overflow
  C_ERR_STACK,      // traversal stack overflow
  C_ERR_INDEX,      // mesh index out of range
  C_LIST_UNDECIDED, // length of the undecided-node list
  C_LIST_WINDING,   // length of the winding list
  C_CERTIFIED,      // learned radius: nodes certified by the bounded search
  C_VISITS,         // LBVH nodes visited by the unbounded search
  C_SIGN_BAND,      // ray-triangle decisions inside the FP32 band, replayed in FP64
  C_NUM = 32
};

// Grid of one call, with the FP32 error scale of the mesh-local frame.
struct GridP {
  double o[3];
  double h;
  int64_t N[3];
  int64_t n[3];     // nodes per axis (N + 1)
  int64_t ngp;
  double center[3]; // mesh-local frame origin
  double E;         // bound on |coordinate - center| for every vertex and node
  int32_t t[3];     // tile dims (nodes)
  int64_t nt[3];    // tiles per axis
  int64_t ntiles;
  int64_t k0 = 0;   // z index of local layer 0 in the full grid (a z-slab call), else 0
};

// Node (i, j, k) of the call in FP64, k local to the slab: origin + h * (global index), the
// reference's mul-then-add (Grid.jl:90).
__device__ __forceinline__ d3 gnode(const GridP& g, int64_t i, int64_t j, int64_t k) {
  return node_coord(g.o, g.h, i, j, k + g.k0);
}
// Centre of warp brick (bx, by, bz) of b[0] x b[1] x b[2] nodes, clipped to the grid: the midpoint of
// its first and last nodes (FP64).  The learned radius is predicted there, once per brick.
__device__ __forceinline__ d3 brick_center(const GridP& g, const int32_t b[3], int64_t bx, int64_t by, int64_t bz) {
  const d3 lo = gnode(g, bx * b[0], by * b[1], bz * b[2]);
  const d3 hi = gnode(g, min(bx * b[0] + b[0] - 1, g.N[0]), min(by * b[1] + b[1] - 1, g.N[1]),
                      min(bz * b[2] + b[2] - 1, g.N[2]));
  return {0.5 * (lo.x + hi.x), 0.5 * (lo.y + hi.y), 0.5 * (lo.z + hi.z)};
}
// Global index along axis a of local index idx.
__host__ __device__ __forceinline__ int64_t gidx(const GridP& g, int a, int64_t idx) {
  return a == 2 ? idx + g.k0 : idx;
}

struct MeshDev {
  int64_t nnp = 0, nel = 0;
  double center[3] = {0, 0, 0};
  double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
  double E = 0.0;        // max |vertex - center| (inf-norm)
  double rho_max = 0.0;  // max vertex distance from its triangle's centroid
  bool ine_ready = false;
};

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

}  // namespace sdfgpu

struct sdfgpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[6] = {};
  std::string err;
  int32_t tile[3] = {4, 4, 4};
  int32_t brick[3] = {4, 2, 4};  // nodes of one warp in the unbounded search (product 32)
  bool has_mesh = false;
  sdfgpu::MeshDev mesh;
  std::unordered_map<std::string, sdfgpu::DevBuf> bufs;
  int64_t* d_counters = nullptr;
  int64_t h_counters[sdfgpu::C_NUM] = {};
  sdfgpu_stats stats = {};
  sdfgpu::RadiusNorm radius;  // learned search radius (radius.cu)
  int64_t launches = 0;  // kernels of this library launched since the last reset
  cudaEvent_t tev[8] = {};  // stage timestamps, see sdfgpu::Stage
  cudaStream_t sign_stream = nullptr;    // the sign stage runs here, beside the distance stage
  cudaStream_t bvh_stream = nullptr;     // the LBVH build runs here, beside the distance stage
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_rows = nullptr;
  cudaEvent_t ev_mesh = nullptr;         // triangle records ready (on the context stream)
  cudaEvent_t ev_bvh = nullptr;          // LBVH of the current mesh complete (on bvh_stream)
  cudaEvent_t ev_obb = nullptr;          // its oriented child boxes complete too (on bvh_stream, after ev_bvh)
  int64_t* h_scalars = nullptr;          // page-locked host slots for sizing reads (see Scalar)
  std::string ns;                        // prefix of every scratch-buffer name (batch items keep their own)
  std::vector<sdfgpu_ctx*> workers;      // batch workers (batch.cu), created on first use
  std::map<int64_t, uint32_t> tuned;     // autotuner: (size class, mode) -> packed tile or brick (batch.cu)
};

namespace sdfgpu {

int fail(sdfgpu_ctx* ctx, int code, const std::string& msg);

#define SDF_CUDA(ctx, call)                                                                       \
  do {                                                                                            \
    cudaError_t e__ = (call);                                                                     \
    if (e__ != cudaSuccess) {                                                                     \
      return ::sdfgpu::fail((ctx), e__ == cudaErrorMemoryAllocation ? SDFGPU_ERR_OUT_OF_MEMORY     \
                                                                    : SDFGPU_ERR_CUDA,            \
                            std::string(#call) + ": " + cudaGetErrorString(e__));                 \
    }                                                                                             \
  } while (0)

// Checks a kernel launch and counts it.
#define SDF_KERNEL(ctx)                         \
  do {                                          \
    SDF_CUDA((ctx), cudaGetLastError());        \
    ++(ctx)->launches;                          \
  } while (0)

// Stage timestamps: the distance stage's on the context stream, the sign stage's on its stream.
enum Stage : int { T_DIST0 = 0, T_TILES, T_FOLD, T_DIST1, T_ROWS, T_PARITY, T_SIGN1, T_SIGN0, T_NUM };
#define SDF_MARK(ctx, i) SDF_CUDA((ctx), cudaEventRecord((ctx)->tev[(i)], (ctx)->stream))
#define SDF_MARK_ON(ctx, i, st) SDF_CUDA((ctx), cudaEventRecord((ctx)->tev[(i)], (st)))

// Slots of ctx->h_scalars: device counts read back to size the next stage.  Page-locked, so the
// read is an asynchronous copy the host waits for only when it needs the value.
enum Scalar : int { S_ROW_TOTAL = 0, S_UNDECIDED, S_WINDING, S_NUM = 8 };

#define SDF_TRY(expr)          \
  do {                         \
    int rc__ = (expr);         \
    if (rc__ != 0) return rc__; \
  } while (0)

// Grow-only named device buffer; *out receives a pointer to at least `bytes` bytes.
int scratch(sdfgpu_ctx* ctx, const char* name, size_t bytes, void** out);

template <class T>
inline int scratch_t(sdfgpu_ctx* ctx, const char* name, size_t count, T** out) {
  void* p = nullptr;
  int rc = scratch(ctx, name, count * sizeof(T) + 16, &p);
  *out = (T*)p;
  return rc;
}

template <class T>
inline T* buf(sdfgpu_ctx* ctx, const char* name) {
  auto it = ctx->ns.empty() ? ctx->bufs.find(name) : ctx->bufs.find(ctx->ns + name);
  return it == ctx->bufs.end() ? nullptr : (T*)it->second.p;
}

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline unsigned grid_for(int64_t n, int block, int64_t cap = 148 * 64) {
  int64_t g = cdiv(n, block);
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// Ordered integer encodings for atomic min/max of doubles.
__device__ __forceinline__ unsigned long long dbl_ord(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
}
__host__ __device__ inline double ord_dbl(unsigned long long u) {
  u = (u & 0x8000000000000000ULL) ? (u & 0x7fffffffffffffffULL) : ~u;
  double d;
  memcpy(&d, &u, sizeof(d));
  return d;
}

__device__ __forceinline__ void count_add(int64_t* counters, int idx, int64_t v) {
  atomicAdd((unsigned long long*)&counters[idx], (unsigned long long)v);
}

// Call scaffolding of the entry points (capi.cu).
int begin_call(sdfgpu_ctx* ctx);
int create_context(const sdfgpu_opts* opts, sdfgpu_ctx** out, bool stage_priority);
int need_mesh(sdfgpu_ctx* ctx);
int reset_counters(sdfgpu_ctx* ctx);
int finish_counters(sdfgpu_ctx* ctx, const GridP& g);
int check_sign_args(sdfgpu_ctx* ctx, int min_rays, int max_rays, double conf);
int check_mode(sdfgpu_ctx* ctx, int mode, int learned);
struct DistPlan;
// All stages of one grid call.  With `defer`, the distance stage stops after its tile lists (its
// fold, fallback and the combine are left to the caller, described by *defer).
int run_all(sdfgpu_ctx* ctx, const GridP& g, bool want_dist, bool want_sign, int mode, int learned, int min_rays,
            int max_rays, double conf, int use_winding, double* d_dist, double* d_xp, double* d_sign, double* d_conf,
            double* d_sdf, DistPlan* defer = nullptr);

// Fills GridP from (origin, h, N) and the current mesh frame; validates sizes.
// k0..k1 (inclusive, k1 >= 0) restricts the call to those z layers of the grid (a z-slab);
// k1 < 0 means all layers.
int make_grid(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], GridP& g, int64_t k0 = 0,
              int64_t k1 = -1);

// Stage entry points (implemented in mesh.cu / distance.cu / sign.cu).
int mesh_upload_and_build(sdfgpu_ctx* ctx, const double* X, int64_t nnp, const int64_t* IEN, int64_t nel,
                          bool device_ptrs);
int ensure_ine(sdfgpu_ctx* ctx);
int run_distances(sdfgpu_ctx* ctx, const GridP& g, int mode, int use_learned, double* d_dist, double* d_xp);
// Exact unbounded distances of a sparse grid's nodes, one thread per node (learned.cu).
int run_nearest_points(sdfgpu_ctx* ctx, const GridP& g, double* d_dist);

// The reference-rule / h-bounded distance stage in parts (distance.cu), so a batch can run the folds
// of many meshes in one launch: dist_prepare builds one mesh's tile lists and fold arguments,
// dist_fold runs one mesh's fold, dist_knn its 3-nearest-vertex fallback, dist_fold_multi the
// folds of many prepared meshes together.
struct DistPlan {
  alignas(16) unsigned char fold[448];      // the fold kernel's arguments
  alignas(16) unsigned char knn_args[448];  // the fallback kernel's arguments (when knn)
  alignas(16) unsigned char unb[512];       // unbounded / learned: the search's arguments (UnbArgs)
  bool unbounded = false;                   // the plan is an unbounded search (unb), not a fold
  bool unb_radius = false;                  // ... started from the learned radius
  int64_t nbricks = 0;                      // ... over this many warp bricks
  GridP g;
  int64_t ntiles = 0;
  int64_t nonempty = -1;  // tiles with candidates (they come first in the fold's order); -1: unknown
  int threads = 0;
  bool knn = false;                         // the fallback runs after the fold
  uint8_t* band = nullptr;                  // nodes within h of a triangle (NULL: every empty node)
  const float4* band_v32 = nullptr;
  const TriRec64* band_rec = nullptr;
  int64_t nel = 0;
  double hb = 0.0;
};
int dist_prepare(sdfgpu_ctx* ctx, const GridP& g, int mode, double* d_dist, double* d_xp, DistPlan& P,
                 int use_learned = 0);
int dist_fold(sdfgpu_ctx* ctx, const DistPlan& P);
int dist_knn(sdfgpu_ctx* ctx, const DistPlan& P, cudaStream_t st, bool wait_bvh);
int dist_fold_multi_grid(sdfgpu_ctx* ctx, int threads, int64_t total, int64_t* grid);
int dist_fold_multi(sdfgpu_ctx* ctx, const void* d_args, const int64_t* d_off, int count, int64_t total, int threads,
                    int64_t grid, cudaStream_t st);
size_t fold_args_size();
void plan_set_counters(DistPlan& P, int64_t* counters);
// The unbounded / learned counterparts for a batch (distance.cu): dist_prepare fills plan.unb when
// the mode is SDFGPU_MODE_UNBOUNDED; unb_multi runs the searches of many such plans in one
// persistent launch (two with the learned radius).
size_t unb_args_size();
void plan_set_redo(DistPlan& P, int64_t* redo, unsigned long long* redo_n, int64_t base);
int unb_multi_grid(sdfgpu_ctx* ctx, int64_t total, int64_t* grid);
int unb_multi(sdfgpu_ctx* ctx, const void* d_items, const int64_t* d_off, int count, bool radius, int64_t* redo,
              unsigned long long* heads, int64_t grid, cudaStream_t st);
int launch_combine(sdfgpu_ctx* ctx, int64_t ngp, const double* d_dist, const double* d_sign, double* d_sdf,
                   cudaStream_t st);
// The sign stage in two parts on ctx->sign_stream: sign_begin enqueues the axis-row counting and
// returns without waiting; sign_finish waits for that count and enqueues the rest (lists, parities,
// vote, adaptive rays, winding).  Between the two the caller can enqueue the distance stage, which
// then overlaps the sign stage on the GPU.  d_sign / d_conf receive the results.
struct SignPlan {
  int64_t Rx = 0, Ry = 0, Rz = 0, nrows = 0;
  int32_t *row_cnt = nullptr, *row_off = nullptr, *row_cur = nullptr;
};
int sign_begin(sdfgpu_ctx* ctx, const GridP& g, SignPlan& P);
int sign_finish(sdfgpu_ctx* ctx, const GridP& g, SignPlan& P, int min_rays, int max_rays, double conf_thresh,
                int use_winding, double* d_sign, double* d_conf);
int run_combine(sdfgpu_ctx* ctx, const GridP& g, const double* d_dist, const double* d_sign, double* d_sdf);
// Exclusive scan of n int32 on stream st (the context stream when NULL), CUB temp storage in the
// named scratch buffer (streams that may overlap use different names).
int cub_scan_i32(sdfgpu_ctx* ctx, const int32_t* in, int32_t* out, int64_t n, cudaStream_t st = nullptr,
                 const char* tmp_name = "cub_tmp_scan");
int train_radius(sdfgpu_ctx* ctx, int coarse_n, int steps, int batch, float lr, uint64_t seed, float* final_loss);
int set_radius_params(sdfgpu_ctx* ctx, const float* params, const double norm[4]);
int get_radius_params(sdfgpu_ctx* ctx, float* params, double norm[4]);
int run_radius(sdfgpu_ctx* ctx, const GridP* g, const float* d_pts, int64_t count, float alpha, float beta, float* d_out,
               const int32_t* brick = nullptr);
int mlp_eval_host(sdfgpu_ctx* ctx, const float* params, const float* xn, const float* target, int64_t B, float* yhat,
                  float* loss, float* grad);
int cub_scan_i64(sdfgpu_ctx* ctx, const int64_t* in, int64_t* out, int64_t n);

}  // namespace sdfgpu
