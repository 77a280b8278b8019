// meshstats.cu -- edge-length statistics of the resident mesh, the analysis the reference prints
// before it asks for a grid step (calculate_edge_distances + analyze_mesh,
// src/MeshGrid/Grid_setup.jl:28-102).
//
// Edge i of a triangle runs from its vertex i to vertex i+1 (wrapping), the same three edges as
// prepare_triangle_data's e1 = v2 - v1, e2 = v3 - v2, e3 = v1 - v3, whose FP64 lengths the triangle
// records already hold.  One pass over the records writes the 3 x nel lengths (for the median) and
// per block, in a fixed grid-stride order, the shortest / longest edge, the edge sum, and the
// triangles with the smallest / largest edge sum (Julia's argmin / argmax: the first index on
// ties).  The host combines the blocks in block order; a CUB radix sort of the lengths gives the
// median (the mean of the two middle values for an even count, as Statistics.median).
#include <cub/cub.cuh>

#include <cmath>
#include <vector>

#include "common.cuh"

namespace sdfgpu {
namespace {

constexpr int kStatBlocks = 296;  // 2 per SM
constexpr int kStatThreads = 256;

struct EdgePart {
  double lmin, lmax, lsum;  // shortest, longest edge; sum of the edges
  double smin, smax;        // smallest / largest edge sum of one triangle
  int64_t imin, imax;       // their triangles (first index on ties)
};

__device__ __forceinline__ void take_min(double& v, int64_t& i, double v2, int64_t i2) {
  if (v2 < v || (v2 == v && i2 >= 0 && (i < 0 || i2 < i))) { v = v2; i = i2; }
}
__device__ __forceinline__ void take_max(double& v, int64_t& i, double v2, int64_t i2) {
  if (v2 > v || (v2 == v && i2 >= 0 && (i < 0 || i2 < i))) { v = v2; i = i2; }
}

__global__ void __launch_bounds__(kStatThreads) k_edge_stats(const TriRec64* __restrict__ rec, int64_t nel,
                                                             double* __restrict__ len, EdgePart* __restrict__ part) {
  EdgePart p = {INFINITY, -INFINITY, 0.0, INFINITY, -INFINITY, -1, -1};
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    const double l0 = rec[el].L[0], l1 = rec[el].L[1], l2 = rec[el].L[2];
    len[3 * el] = l0;
    len[3 * el + 1] = l1;
    len[3 * el + 2] = l2;
    p.lmin = fmin(p.lmin, fmin(l0, fmin(l1, l2)));
    p.lmax = fmax(p.lmax, fmax(l0, fmax(l1, l2)));
    const double s = (l0 + l1) + l2;  // sum(distances, dims = 1) of the column
    p.lsum += s;
    take_min(p.smin, p.imin, s, el);
    take_max(p.smax, p.imax, s, el);
  }
  // warp, then block, in a fixed order
  __shared__ EdgePart sh[kStatThreads / 32];
  for (int off = 16; off > 0; off >>= 1) {
    const double lmin = __shfl_down_sync(0xffffffffu, p.lmin, off), lmax = __shfl_down_sync(0xffffffffu, p.lmax, off);
    const double lsum = __shfl_down_sync(0xffffffffu, p.lsum, off);
    const double smin = __shfl_down_sync(0xffffffffu, p.smin, off), smax = __shfl_down_sync(0xffffffffu, p.smax, off);
    const long long imin = __shfl_down_sync(0xffffffffu, (long long)p.imin, off);
    const long long imax = __shfl_down_sync(0xffffffffu, (long long)p.imax, off);
    p.lmin = fmin(p.lmin, lmin);
    p.lmax = fmax(p.lmax, lmax);
    p.lsum += lsum;
    take_min(p.smin, p.imin, smin, imin);
    take_max(p.smax, p.imax, smax, imax);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[w] = p;
  __syncthreads();
  if (threadIdx.x == 0) {
    EdgePart b = sh[0];
    for (int k = 1; k < kStatThreads / 32; ++k) {
      b.lmin = fmin(b.lmin, sh[k].lmin);
      b.lmax = fmax(b.lmax, sh[k].lmax);
      b.lsum += sh[k].lsum;
      take_min(b.smin, b.imin, sh[k].smin, sh[k].imin);
      take_max(b.smax, b.imax, sh[k].smax, sh[k].imax);
    }
    part[blockIdx.x] = b;
  }
}

}  // namespace
}  // namespace sdfgpu

using namespace sdfgpu;

extern "C" {

int sdfgpu_mesh_edge_stats(sdfgpu_ctx* ctx, double out[6], int64_t idx_out[2]) {
  SDF_TRY(begin_call(ctx));
  if (!out) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "out must not be NULL");
  if (!ctx->has_mesh) return fail(ctx, SDFGPU_ERR_NO_MESH, "no mesh: call sdfgpu_set_mesh first");
  const int64_t nel = ctx->mesh.nel;
  if (nel < 1) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "the mesh has no triangles");
  if (3 * nel > 0x7fffffffLL) return fail(ctx, SDFGPU_ERR_CAPACITY, "more than 2^31 edges");
  cudaStream_t st = ctx->stream;
  const int n = (int)(3 * nel);
  double *len, *len2;
  EdgePart* part;
  SDF_TRY(scratch_t(ctx, "edge_len", (size_t)n, &len));
  SDF_TRY(scratch_t(ctx, "edge_len2", (size_t)n, &len2));
  SDF_TRY(scratch_t(ctx, "edge_part", (size_t)kStatBlocks, &part));
  const unsigned blocks = (unsigned)std::min<int64_t>(kStatBlocks, (nel + kStatThreads - 1) / kStatThreads);
  k_edge_stats<<<blocks, kStatThreads, 0, st>>>(buf<TriRec64>(ctx, "rec"), nel, len, part);
  SDF_KERNEL(ctx);
  size_t tmp_bytes = 0;
  SDF_CUDA(ctx, cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, len, len2, n, 0, 64, st));
  void* tmp;
  SDF_TRY(scratch(ctx, "cub_tmp_edges", tmp_bytes, &tmp));
  SDF_CUDA(ctx, cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, len, len2, n, 0, 64, st));
  std::vector<EdgePart> hp(blocks);
  double mid[2] = {0.0, 0.0};
  SDF_CUDA(ctx, cudaMemcpyAsync(hp.data(), part, sizeof(EdgePart) * blocks, cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(mid, len2 + (n - 1) / 2, sizeof(double) * (n % 2 ? 1 : 2), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  EdgePart b = hp[0];
  for (unsigned k = 1; k < blocks; ++k) {
    const EdgePart& q = hp[k];
    b.lmin = std::fmin(b.lmin, q.lmin);
    b.lmax = std::fmax(b.lmax, q.lmax);
    b.lsum += q.lsum;
    // blocks cover interleaved index ranges, so ties between blocks go to the smaller index
    if (q.smin < b.smin || (q.smin == b.smin && q.imin < b.imin)) { b.smin = q.smin; b.imin = q.imin; }
    if (q.smax > b.smax || (q.smax == b.smax && q.imax < b.imax)) { b.smax = q.smax; b.imax = q.imax; }
  }
  out[0] = b.lmin;
  out[1] = b.lmax;
  out[2] = b.lsum / (double)n;
  out[3] = n % 2 ? mid[0] : mid[0] / 2 + mid[1] / 2;  // Statistics.middle(a, b) = a/2 + b/2
  out[4] = b.smin / 3.0;  // mean of the smallest triangle's three edges
  out[5] = b.smax / 3.0;
  if (idx_out) {
    idx_out[0] = b.imin;
    idx_out[1] = b.imax;
  }
  return SDFGPU_OK;
}

}  // extern "C"
