// stlimport.cu -- the vertex deduplication of the STL import, process_stl_mesh
// (src/DataImport/ImportStlData.jl:198-309), on the GPU.
//
// The reference walks the triangle stream vertex by vertex and merges a vertex into the first
// earlier unique vertex within norm < 1e-10 that it finds in its cell floor(v * 1e10) of a spatial
// hash or, failing that, in a neighbouring cell; unique vertices are numbered in order of first
// appearance.  Unless two DISTINCT vertices of the mesh lie within 1e-10 of each other, that is
// exact deduplication (a vertex merges only with copies of itself; -0.0 equals +0.0) with
// first-appearance numbering, which this file computes:
//   1. three stable radix sorts of the stream (by z, then y, then x) give the lexicographic order,
//      and stability keeps each group of equal vertices in stream order, so the head of a group
//      is its first appearance;
//   2. a scan of the group heads numbers the groups; a sort of the groups by first appearance
//      gives the reference's vertex numbering, and the triangle indices follow;
//   3. the same reference cells decide whether distinct vertices closer than 1e-10 exist: the
//      unique vertices are sorted by cell, and every vertex looks for another within norm < 1e-10
//      in its own and the 26 neighbouring cells (every such pair lies in adjacent cells).  Their
//      number is returned; when it is not zero the reference's order-dependent tolerance merge
//      applies instead, and the caller runs it.
#include <cub/cub.cuh>

#include <climits>
#include <cmath>

#include "common.cuh"

namespace sdfgpu {
namespace {

constexpr double kDedupeTol = 1e-10;
constexpr double kCellScale = 1e10;  // floor(Int, 1 / tol)

// Order-preserving key of a double; -0.0 is taken as +0.0 (the two compare equal).
__device__ __forceinline__ uint64_t dkey(double x) {
  if (x == 0.0) x = 0.0;
  const uint64_t u = (uint64_t)__double_as_longlong(x);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
// Order-preserving key of an int64.
__device__ __forceinline__ uint64_t ikey(int64_t c) { return (uint64_t)c ^ 0x8000000000000000ull; }

__global__ void k_dd_iota(int32_t* __restrict__ p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (int32_t)i;
}

// Sort key of coordinate `axis` of the vertices in the current order; also flags non-finite ones.
__global__ void k_dd_keys(const double* __restrict__ V, const int32_t* __restrict__ perm, int64_t n, int axis,
                          uint64_t* __restrict__ key, int32_t* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = V[3 * (int64_t)perm[i] + axis];
    if (!isfinite(x)) atomicExch(bad, 1);
    key[i] = dkey(x);
  }
}

__global__ void k_dd_heads(const double* __restrict__ V, const int32_t* __restrict__ perm, int64_t n,
                           int32_t* __restrict__ head) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t h = 1;
    if (i > 0) {
      const double* a = V + 3 * (int64_t)perm[i];
      const double* b = V + 3 * (int64_t)perm[i - 1];
      h = (a[0] != b[0] || a[1] != b[1] || a[2] != b[2]) ? 1 : 0;
    }
    head[i] = h;
  }
}

// gid1: inclusive scan of the heads (1-based group number).  Group g's first appearance is the
// stream index at its head.
__global__ void k_dd_first(const int32_t* __restrict__ perm, const int32_t* __restrict__ head,
                           const int32_t* __restrict__ gid1, int64_t n, int32_t* __restrict__ first,
                           int32_t* __restrict__ gidx) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (head[i]) {
      const int32_t g = gid1[i] - 1;
      first[g] = perm[i];
      gidx[g] = g;
    }
}

__global__ void k_dd_rank(const int32_t* __restrict__ g_sorted, int64_t nu, int32_t* __restrict__ rank) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nu; r += (int64_t)gridDim.x * blockDim.x)
    rank[g_sorted[r]] = (int32_t)r;
}

__global__ void k_dd_out(const double* __restrict__ V, const int32_t* __restrict__ first_sorted, int64_t nu,
                         double* __restrict__ X) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nu; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = first_sorted[r];
    X[3 * r] = V[3 * s];
    X[3 * r + 1] = V[3 * s + 1];
    X[3 * r + 2] = V[3 * s + 2];
  }
}

__global__ void k_dd_ien(const int32_t* __restrict__ perm, const int32_t* __restrict__ gid1,
                         const int32_t* __restrict__ rank, int64_t n, int64_t* __restrict__ IEN) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    IEN[perm[i]] = (int64_t)rank[gid1[i] - 1] + 1;
}

// The reference's hash cell of a coordinate, floor(Int, x * 1e10); *bad when it is not an Int64.
__device__ __forceinline__ int64_t cell_of(double x, int32_t* bad) {
  const double f = floor(x * kCellScale);
  if (!(f >= -9.2233720368547758e18 && f < 9.2233720368547758e18)) {
    atomicExch(bad, 2);
    return 0;
  }
  return (int64_t)f;
}

__global__ void k_dd_cell_keys(const double* __restrict__ X, const int32_t* __restrict__ perm, int64_t nu, int axis,
                               uint64_t* __restrict__ key, int32_t* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nu; i += (int64_t)gridDim.x * blockDim.x)
    key[i] = ikey(cell_of(X[3 * (int64_t)perm[i] + axis], bad));
}

__global__ void k_dd_cells(const double* __restrict__ X, const int32_t* __restrict__ perm, int64_t nu,
                           longlong4* __restrict__ cells, int32_t* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nu; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t u = perm[i];
    cells[i] = make_longlong4(cell_of(X[3 * u], bad), cell_of(X[3 * u + 1], bad), cell_of(X[3 * u + 2], bad), u);
  }
}

__device__ __forceinline__ bool cell_less(const longlong4& a, long long x, long long y, long long z) {
  return a.x < x || (a.x == x && (a.y < y || (a.y == y && a.z < z)));
}

// For every unique vertex, the other unique vertices with norm(v - w) < 1e-10 in its own and the 26
// neighbouring cells (cells sorted lexicographically).  Counts ordered pairs.
__global__ void k_dd_near(const double* __restrict__ X, const longlong4* __restrict__ cells, int64_t nu,
                          unsigned long long* __restrict__ near) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nu; i += (int64_t)gridDim.x * blockDim.x) {
    const longlong4 c = cells[i];
    const d3 v = {X[3 * c.w], X[3 * c.w + 1], X[3 * c.w + 2]};
    unsigned long long cnt = 0;
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          // cells[] is sorted and the neighbour cells are valid Int64 (the reference would have
          // thrown otherwise), but c.x + dx may still wrap at the Int64 limits: skip those
          if ((dx < 0 && c.x == LLONG_MIN) || (dx > 0 && c.x == LLONG_MAX) || (dy < 0 && c.y == LLONG_MIN) ||
              (dy > 0 && c.y == LLONG_MAX) || (dz < 0 && c.z == LLONG_MIN) || (dz > 0 && c.z == LLONG_MAX))
            continue;
          const long long tx = c.x + dx, ty = c.y + dy, tz = c.z + dz;
          int64_t lo = 0, hi = nu;  // first position not less than the target cell
          while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (cell_less(cells[mid], tx, ty, tz)) lo = mid + 1;
            else hi = mid;
          }
          for (int64_t j = lo; j < nu; ++j) {
            const longlong4 w = cells[j];
            if (w.x != tx || w.y != ty || w.z != tz) break;
            if (w.w == c.w) continue;
            const d3 q = {X[3 * w.w], X[3 * w.w + 1], X[3 * w.w + 2]};
            if (v_norm(v_sub(v, q)) < kDedupeTol) ++cnt;
          }
        }
    if (cnt) atomicAdd(near, cnt);
  }
}

// Three stable radix sorts of perm by the keys of coordinates z, y, x (LSD order).
int sort_lexicographic(sdfgpu_ctx* ctx, cudaStream_t st, int64_t n, int32_t*& perm, int32_t*& perm2, uint64_t* key,
                       uint64_t* key2, int32_t* bad, bool cells, const double* V) {
  for (int axis = 2; axis >= 0; --axis) {
    if (cells)
      k_dd_cell_keys<<<grid_for(n, 256), 256, 0, st>>>(V, perm, n, axis, key, bad);
    else
      k_dd_keys<<<grid_for(n, 256), 256, 0, st>>>(V, perm, n, axis, key, bad);
    SDF_KERNEL(ctx);
    size_t bytes = 0;
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, bytes, key, key2, perm, perm2, (int)n, 0, 64, st));
    void* tmp;
    SDF_TRY(scratch(ctx, "cub_tmp_dedupe", bytes, &tmp));
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, bytes, key, key2, perm, perm2, (int)n, 0, 64, st));
    std::swap(perm, perm2);
  }
  return 0;
}

}  // namespace
}  // namespace sdfgpu

using namespace sdfgpu;

extern "C" {

int sdfgpu_stl_dedupe(sdfgpu_ctx* ctx, const double* V, int64_t nv, double* X_out, int64_t* IEN_out,
                      int64_t* nnp_out, int64_t* near_out) {
  SDF_TRY(begin_call(ctx));
  if (!V || !X_out || !IEN_out || !nnp_out || !near_out)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "V, X_out, IEN_out, nnp_out and near_out must not be NULL");
  if (nv < 1) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "nv must be >= 1");
  if (nv > 0x7fffffffLL) return fail(ctx, SDFGPU_ERR_CAPACITY, "more than 2^31 - 1 stream vertices");
  cudaStream_t st = ctx->stream;
  const int64_t n = nv;
  double* dV;
  int32_t *perm, *perm2, *head, *gid1, *bad;
  uint64_t *key, *key2;
  SDF_TRY(scratch_t(ctx, "dd_v", (size_t)(3 * n), &dV));
  SDF_TRY(scratch_t(ctx, "dd_perm", (size_t)n, &perm));
  SDF_TRY(scratch_t(ctx, "dd_perm2", (size_t)n, &perm2));
  SDF_TRY(scratch_t(ctx, "dd_key", (size_t)n, &key));
  SDF_TRY(scratch_t(ctx, "dd_key2", (size_t)n, &key2));
  SDF_TRY(scratch_t(ctx, "dd_head", (size_t)n, &head));
  SDF_TRY(scratch_t(ctx, "dd_gid", (size_t)n, &gid1));
  SDF_TRY(scratch_t(ctx, "dd_bad", 4, &bad));
  SDF_CUDA(ctx, cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
  SDF_CUDA(ctx, cudaMemcpyAsync(dV, V, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
  // 1. lexicographic order of the stream, ties in stream order
  k_dd_iota<<<grid_for(n, 256), 256, 0, st>>>(perm, n);
  SDF_KERNEL(ctx);
  SDF_TRY(sort_lexicographic(ctx, st, n, perm, perm2, key, key2, bad, false, dV));
  // 2. groups of equal vertices and their numbering by first appearance
  k_dd_heads<<<grid_for(n, 256), 256, 0, st>>>(dV, perm, n, head);
  SDF_KERNEL(ctx);
  {
    size_t bytes = 0;
    SDF_CUDA(ctx, cub::DeviceScan::InclusiveSum(nullptr, bytes, head, gid1, (int)n, st));
    void* tmp;
    SDF_TRY(scratch(ctx, "cub_tmp_dedupe_scan", bytes, &tmp));
    SDF_CUDA(ctx, cub::DeviceScan::InclusiveSum(tmp, bytes, head, gid1, (int)n, st));
  }
  int32_t h_small[2] = {0, 0};  // {groups, bad}
  SDF_CUDA(ctx, cudaMemcpyAsync(&h_small[0], gid1 + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(&h_small[1], bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  if (h_small[1]) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "STL vertices must be finite");
  const int64_t nu = h_small[0];
  int32_t *first, *gidx, *first_s, *g_s, *rank;
  double* dX;
  int64_t* dIEN;
  SDF_TRY(scratch_t(ctx, "dd_first", (size_t)nu, &first));
  SDF_TRY(scratch_t(ctx, "dd_gidx", (size_t)nu, &gidx));
  SDF_TRY(scratch_t(ctx, "dd_first_s", (size_t)nu, &first_s));
  SDF_TRY(scratch_t(ctx, "dd_g_s", (size_t)nu, &g_s));
  SDF_TRY(scratch_t(ctx, "dd_rank", (size_t)nu, &rank));
  SDF_TRY(scratch_t(ctx, "dd_x", (size_t)(3 * nu), &dX));
  SDF_TRY(scratch_t(ctx, "dd_ien", (size_t)n, &dIEN));
  k_dd_first<<<grid_for(n, 256), 256, 0, st>>>(perm, head, gid1, n, first, gidx);
  SDF_KERNEL(ctx);
  {
    int bits = 1;
    while (bits < 31 && (1LL << bits) < n) ++bits;
    size_t bytes = 0;
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, bytes, first, first_s, gidx, g_s, (int)nu, 0, bits, st));
    void* tmp;
    SDF_TRY(scratch(ctx, "cub_tmp_dedupe", bytes, &tmp));
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, bytes, first, first_s, gidx, g_s, (int)nu, 0, bits, st));
  }
  k_dd_rank<<<grid_for(nu, 256), 256, 0, st>>>(g_s, nu, rank);
  SDF_KERNEL(ctx);
  k_dd_out<<<grid_for(nu, 256), 256, 0, st>>>(dV, first_s, nu, dX);
  SDF_KERNEL(ctx);
  k_dd_ien<<<grid_for(n, 256), 256, 0, st>>>(perm, gid1, rank, n, dIEN);
  SDF_KERNEL(ctx);
  // 3. distinct vertices closer than the tolerance, on the reference's hash cells
  int32_t *cperm = perm, *cperm2 = perm2;  // reused: the stream order is no longer needed
  longlong4* cells;
  unsigned long long* d_near;
  SDF_TRY(scratch_t(ctx, "dd_cells", (size_t)nu, &cells));
  SDF_TRY(scratch_t(ctx, "dd_near", 1, &d_near));
  SDF_CUDA(ctx, cudaMemsetAsync(d_near, 0, sizeof(unsigned long long), st));
  k_dd_iota<<<grid_for(nu, 256), 256, 0, st>>>(cperm, nu);
  SDF_KERNEL(ctx);
  SDF_TRY(sort_lexicographic(ctx, st, nu, cperm, cperm2, key, key2, bad, true, dX));
  k_dd_cells<<<grid_for(nu, 256), 256, 0, st>>>(dX, cperm, nu, cells, bad);
  SDF_KERNEL(ctx);
  k_dd_near<<<grid_for(nu, 128), 128, 0, st>>>(dX, cells, nu, d_near);
  SDF_KERNEL(ctx);
  unsigned long long h_near = 0;
  SDF_CUDA(ctx, cudaMemcpyAsync(&h_small[1], bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(&h_near, d_near, sizeof(h_near), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(X_out, dX, sizeof(double) * 3 * nu, cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(IEN_out, dIEN, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  if (h_small[1])
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "a vertex coordinate times 1e10 is outside the Int64 range");
  *nnp_out = nu;
  *near_out = (int64_t)h_near;
  return SDFGPU_OK;
}

}  // extern "C"
