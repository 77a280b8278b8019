// artifacts.cu -- remove_sdf_artifacts! / analyze_sdf_components
// (src/SignedDistances/SdfArtifactRemoval.jl:134-318) on the GPU.
//
// Interior nodes are sdf >= threshold (a NaN is exterior).  Their 6-connected components are found
// with a lock-free union-find over the grid (the hooking and pointer-jumping scheme of ECL-CC,
// Jaiganesh and Burtscher 2018): parent[i] <= i always holds, a union links the larger of the two
// roots under the smaller one with one compare-and-swap, and a find shortens the path it walks.
// So when every union has completed, the root of a component is its smallest linear node index,
// whatever order the unions ran in -- the labelling is deterministic, while the reference's
// union-by-rank inside @threads (:164-182) is racy.  Components smaller than
// max(1, round(ratio * largest)) that are not the largest one are flipped to -|sdf| (:201-230).
// Ties for the largest component are broken towards the smallest root; they change a result only
// when ratio > 1, where the reference's choice depends on its Dict's iteration order.
//
// Every loop walks strictly decreasing indices, so it ends within ngp steps; the loops still carry
// that bound and report SDFGPU_ERR_CAPACITY instead of spinning.
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace sdfgpu {
namespace {

__device__ __forceinline__ int32_t ld_parent(const int32_t* p, int64_t i) { return __ldcg(p + i); }

// Root of x.  kHalve: halve the path on the way (every store writes an ancestor, so parent[i] <= i
// and the ancestor relation survive concurrent unions).  Without it the walk only reads, which the
// final labelling pass needs: there each node's own thread must be the last writer of its entry,
// and a late halving store from another thread could put back a non-root ancestor.
template <bool kHalve>
__device__ __forceinline__ int32_t find_root(int32_t* p, int32_t x, int64_t cap, bool& bad) {
  int32_t cur = ld_parent(p, x);
  if (cur == x) return x;
  int32_t prev = x;
  int64_t steps = 0;
  int32_t nxt;
  while (cur > (nxt = ld_parent(p, cur))) {
    if (++steps > cap) { bad = true; break; }
    if (kHalve) __stcg(p + prev, nxt);
    prev = cur;
    cur = nxt;
  }
  return cur;
}

__device__ __forceinline__ void unite(int32_t* p, int32_t a, int32_t b, int64_t cap, bool& bad) {
  int32_t ra = find_root<true>(p, a, cap, bad), rb = find_root<true>(p, b, cap, bad);
  int64_t steps = 0;
  while (ra != rb && !bad) {
    if (++steps > cap) { bad = true; break; }
    if (ra < rb) {  // hook rb under ra
      const int32_t old = atomicCAS(p + rb, rb, ra);
      if (old == rb) break;
      rb = old;
    } else {
      const int32_t old = atomicCAS(p + ra, ra, rb);
      if (old == ra) break;
      ra = old;
    }
  }
}

__global__ void k_cc_init(const double* __restrict__ sdf, int64_t ngp, double thr, int32_t* __restrict__ parent,
                          int64_t* counters) {
  int64_t interior = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ngp; i += (int64_t)gridDim.x * blockDim.x) {
    const bool in = sdf[i] >= thr;
    parent[i] = in ? (int32_t)i : -1;
    interior += in;
  }
  for (int off = 16; off > 0; off >>= 1) interior += __shfl_down_sync(0xffffffffu, interior, off);
  if ((threadIdx.x & 31) == 0 && interior) count_add(counters, 0, interior);
}

// Unions of each interior node with its interior -x, -y and -z neighbours (the +x/+y/+z pairs are
// the same pairs seen from the other node).
__global__ void k_cc_union(int32_t* parent, int64_t nx, int64_t ny, int64_t nz, int64_t* counters) {
  const int64_t ngp = nx * ny * nz, nxy = nx * ny;
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ngp; i += (int64_t)gridDim.x * blockDim.x) {
    if (ld_parent(parent, i) < 0) continue;
    const int64_t x = i % nx, y = (i / nx) % ny, z = i / nxy;
    if (x > 0 && ld_parent(parent, i - 1) >= 0) unite(parent, (int32_t)i, (int32_t)(i - 1), ngp, bad);
    if (y > 0 && ld_parent(parent, i - nx) >= 0) unite(parent, (int32_t)i, (int32_t)(i - nx), ngp, bad);
    if (z > 0 && ld_parent(parent, i - nxy) >= 0) unite(parent, (int32_t)i, (int32_t)(i - nxy), ngp, bad);
  }
  if (bad) count_add(counters, 1, 1);
}

// Every interior node points at its root; sizes and the component count.  The unions have all
// completed, so the forest only changes here by each node's own store of its root (an ancestor of
// it): concurrent walks stay valid and every entry ends as its root.
__global__ void k_cc_flatten(int32_t* parent, int64_t ngp, int32_t* __restrict__ size, int64_t* counters) {
  bool bad = false;
  int64_t roots = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ngp; i += (int64_t)gridDim.x * blockDim.x) {
    if (ld_parent(parent, i) < 0) continue;
    const int32_t r = find_root<false>(parent, (int32_t)i, ngp, bad);
    __stcg(parent + i, r);
    atomicAdd(size + r, 1);
    roots += (r == (int32_t)i);
  }
  for (int off = 16; off > 0; off >>= 1) roots += __shfl_down_sync(0xffffffffu, roots, off);
  if ((threadIdx.x & 31) == 0 && roots) count_add(counters, 2, roots);
  if (bad) count_add(counters, 1, 1);
}

// Largest component: max of (size << 32 | 0x7fffffff - root), i.e. ties to the smallest root.
__global__ void k_cc_largest(const int32_t* __restrict__ parent, const int32_t* __restrict__ size, int64_t ngp,
                             unsigned long long* best) {
  unsigned long long b = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ngp; i += (int64_t)gridDim.x * blockDim.x) {
    if (parent[i] != (int32_t)i) continue;
    const unsigned long long key = ((unsigned long long)(uint32_t)size[i] << 32) | (uint32_t)(0x7fffffff - (int32_t)i);
    b = key > b ? key : b;
  }
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_down_sync(0xffffffffu, b, off);
    b = o > b ? o : b;
  }
  if ((threadIdx.x & 31) == 0 && b) atomicMax(best, b);
}

__global__ void k_cc_flip(double* __restrict__ sdf, const int32_t* __restrict__ parent, const int32_t* __restrict__ size,
                          int64_t ngp, int32_t keep_root, int64_t min_size, int64_t* counters) {
  int64_t flipped = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ngp; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = parent[i];
    if (r < 0 || r == keep_root || (int64_t)size[r] >= min_size) continue;
    sdf[i] = -fabs(sdf[i]);
    ++flipped;
  }
  for (int off = 16; off > 0; off >>= 1) flipped += __shfl_down_sync(0xffffffffu, flipped, off);
  if ((threadIdx.x & 31) == 0 && flipped) count_add(counters, 3, flipped);
}

struct CCResult {
  int64_t interior = 0, components = 0, largest = 0, flipped = 0;
  int32_t largest_root = -1;
};

// Labels the interior components of d_sdf (grid N); when ratio >= 0 also flips the small ones.
int run_components(sdfgpu_ctx* ctx, const int64_t N[3], double* d_sdf, double thr, double ratio, CCResult& R,
                   int32_t** d_parent_out) {
  if (!N) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "N must not be NULL");
  double cells = 1.0;
  for (int a = 0; a < 3; ++a) {
    if (N[a] < 0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "N must be >= 0");
    cells *= (double)(N[a] + 1);
  }
  if (cells > 2147483647.0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "grid has more than 2^31-1 nodes");
  const int64_t nx = N[0] + 1, ny = N[1] + 1, nz = N[2] + 1, ngp = nx * ny * nz;
  cudaStream_t st = ctx->stream;
  int32_t *parent, *size;
  unsigned long long* best;
  int64_t* cnt;
  SDF_TRY(scratch_t(ctx, "cc_parent", (size_t)ngp, &parent));
  SDF_TRY(scratch_t(ctx, "cc_size", (size_t)ngp, &size));
  SDF_TRY(scratch_t(ctx, "cc_best", 1, &best));
  SDF_TRY(scratch_t(ctx, "cc_counters", 4, &cnt));
  SDF_CUDA(ctx, cudaMemsetAsync(size, 0, sizeof(int32_t) * ngp, st));
  SDF_CUDA(ctx, cudaMemsetAsync(best, 0, sizeof(unsigned long long), st));
  SDF_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int64_t) * 4, st));
  const unsigned grid = grid_for(ngp, 256, 148 * 8);
  k_cc_init<<<grid, 256, 0, st>>>(d_sdf, ngp, thr, parent, cnt);
  SDF_KERNEL(ctx);
  k_cc_union<<<grid, 256, 0, st>>>(parent, nx, ny, nz, cnt);
  SDF_KERNEL(ctx);
  k_cc_flatten<<<grid, 256, 0, st>>>(parent, ngp, size, cnt);
  SDF_KERNEL(ctx);
  k_cc_largest<<<grid, 256, 0, st>>>(parent, size, ngp, best);
  SDF_KERNEL(ctx);
  int64_t h_cnt[4];
  unsigned long long h_best = 0;
  SDF_CUDA(ctx, cudaMemcpyAsync(h_cnt, cnt, sizeof(h_cnt), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(&h_best, best, sizeof(h_best), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  if (h_cnt[1]) return fail(ctx, SDFGPU_ERR_CAPACITY, "component labelling exceeded its step bound");
  R.interior = h_cnt[0];
  R.components = h_cnt[2];
  if (h_best) {
    R.largest = (int64_t)(h_best >> 32);
    R.largest_root = 0x7fffffff - (int32_t)(h_best & 0xffffffffULL);
  }
  if (ratio >= 0.0 && R.components > 0) {
    // max(1, round(Int, ratio * largest)): round to nearest, ties to even
    const double ms = std::nearbyint(ratio * (double)R.largest);
    const int64_t min_size = std::max<int64_t>(1, ms > 9.0e18 ? (int64_t)9e18 : (int64_t)ms);
    k_cc_flip<<<grid, 256, 0, st>>>(d_sdf, parent, size, ngp, R.largest_root, min_size, cnt);
    SDF_KERNEL(ctx);
    SDF_CUDA(ctx, cudaMemcpyAsync(&R.flipped, cnt + 3, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SDF_CUDA(ctx, cudaStreamSynchronize(st));
  }
  if (d_parent_out) *d_parent_out = parent;
  return 0;
}

void write_out(const CCResult& R, int64_t* flipped, int64_t* components, int64_t* largest) {
  if (flipped) *flipped = R.flipped;
  if (components) *components = R.components;
  if (largest) *largest = R.largest;
}

}  // namespace
}  // namespace sdfgpu

using namespace sdfgpu;

extern "C" {

int sdfgpu_remove_artifacts_device(sdfgpu_ctx* ctx, const int64_t N[3], double* d_sdf, double threshold,
                                   double min_component_ratio, int64_t* flipped, int64_t* components,
                                   int64_t* largest) {
  SDF_TRY(begin_call(ctx));
  if (!d_sdf) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "sdf must not be NULL");
  if (!(min_component_ratio >= 0.0) || !std::isfinite(min_component_ratio))
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "min_component_ratio must be finite and >= 0");
  CCResult R;
  SDF_TRY(run_components(ctx, N, d_sdf, threshold, min_component_ratio, R, nullptr));
  write_out(R, flipped, components, largest);
  return SDFGPU_OK;
}

int sdfgpu_remove_artifacts(sdfgpu_ctx* ctx, const int64_t N[3], double* sdf, double threshold,
                            double min_component_ratio, int64_t* flipped, int64_t* components, int64_t* largest) {
  SDF_TRY(begin_call(ctx));
  if (!sdf || !N) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "sdf and N must not be NULL");
  if (!(min_component_ratio >= 0.0) || !std::isfinite(min_component_ratio))
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "min_component_ratio must be finite and >= 0");
  double cells = 1.0;
  for (int a = 0; a < 3; ++a) cells *= (double)(std::max<int64_t>(N[a], -1) + 1);
  if (cells > 2147483647.0 || cells < 0.0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "bad grid size");
  const size_t ngp = (size_t)cells;
  double* d;
  SDF_TRY(scratch_t(ctx, "cc_sdf", ngp, &d));
  SDF_CUDA(ctx, cudaMemcpyAsync(d, sdf, sizeof(double) * ngp, cudaMemcpyHostToDevice, ctx->stream));
  CCResult R;
  SDF_TRY(run_components(ctx, N, d, threshold, min_component_ratio, R, nullptr));
  if (R.flipped) {
    SDF_CUDA(ctx, cudaMemcpyAsync(sdf, d, sizeof(double) * ngp, cudaMemcpyDeviceToHost, ctx->stream));
    SDF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  write_out(R, flipped, components, largest);
  return SDFGPU_OK;
}

int sdfgpu_sdf_components(sdfgpu_ctx* ctx, const int64_t N[3], const double* sdf, double threshold, int32_t* root_out,
                          int64_t* components, int64_t* largest) {
  SDF_TRY(begin_call(ctx));
  if (!sdf || !N) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "sdf and N must not be NULL");
  double cells = 1.0;
  for (int a = 0; a < 3; ++a) cells *= (double)(std::max<int64_t>(N[a], -1) + 1);
  if (cells > 2147483647.0 || cells < 0.0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "bad grid size");
  const size_t ngp = (size_t)cells;
  double* d;
  SDF_TRY(scratch_t(ctx, "cc_sdf", ngp, &d));
  SDF_CUDA(ctx, cudaMemcpyAsync(d, sdf, sizeof(double) * ngp, cudaMemcpyHostToDevice, ctx->stream));
  CCResult R;
  int32_t* parent = nullptr;
  SDF_TRY(run_components(ctx, N, d, threshold, -1.0, R, &parent));
  if (root_out) {
    SDF_CUDA(ctx, cudaMemcpyAsync(root_out, parent, sizeof(int32_t) * ngp, cudaMemcpyDeviceToHost, ctx->stream));
    SDF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  write_out(R, nullptr, components, largest);
  return SDFGPU_OK;
}

}  // extern "C"
