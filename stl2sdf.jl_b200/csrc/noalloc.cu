// noalloc.cu -- sdfgpu_distances_noalloc: the true point-triangle distance of every grid node for
// callers that cannot allocate GPU memory.
//
// Who needs this: code that runs where a cudaMalloc is not allowed or not possible -- inside a
// host callback or a custom allocator hook, in a process whose device memory is owned by another
// framework's pool, or in a real-time loop that must not take the allocator's locks or trigger
// device-wide synchronisation.  The regular entry points keep their scratch (triangle records,
// LBVH, tile lists) in buffers they allocate on first use; this one keeps its only scratch, the
// per-triangle records, in the fixed device array below and never allocates.
//
// Limits and sharing:
//   * at most kNoAllocMaxTriangles triangles (larger meshes are rejected with an error);
//   * the work is one FP64 step per (node, triangle) pair, so a call may hold the GPU for a long
//     time: calls with more than kNoAllocMaxSteps pairs are rejected with an error;
//   * the array lives in every GPU that loads the library, until the process exits;
//   * every call reuses the same array and it keeps the last call's contents, so two calls that
//     overlap on the GPU (different streams, or several host threads) race and corrupt each
//     other -- callers must serialise them;
//   * every call looks up the array's address on the current device (cudaGetSymbolAddress, which
//     allocates nothing), so nothing cached goes stale when a context is torn down and rebuilt;
//   * the call synchronizes its stream before it returns (to read the error word), so it must not
//     be called while that stream is being captured.
//
// Work: one thread per node folds every triangle in index order with the reference's FP64 step
// (true minimum), so the result is bit-identical to sdfgpu_distances in the same mode.
#include <cmath>
#include <string>

#include "common.cuh"

namespace sdfgpu {

namespace {

constexpr int64_t kNoAllocMaxTriangles = 16384;
constexpr double kNoAllocMaxSteps = 68719476736.0;  // 2^36 (node, triangle) FP64 steps, well under a second
constexpr size_t kNoAllocBytes = 256 + sizeof(TriRec64) * (size_t)kNoAllocMaxTriangles;  // ~5.8 MB

// The only scratch of sdfgpu_distances_noalloc: an error word in the first 256 bytes, then the
// triangle records.  In host code this name is only a handle for cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

__global__ void k_na_prep(const double* __restrict__ X, int64_t nnp, const int64_t* __restrict__ IEN, int64_t nel,
                          unsigned char* scratch) {
  int* flag = reinterpret_cast<int*>(scratch);
  TriRec64* rec = reinterpret_cast<TriRec64*>(scratch + 256);
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    TriRec64 r;
    d3 v[3];
    for (int k = 0; k < 3; ++k) {
      int64_t vi = IEN[3 * el + k];
      if (vi < 1 || vi > nnp) {
        atomicExch(flag, 1);
        vi = 1;
      }
      vi -= 1;
      v[k] = {X[3 * vi], X[3 * vi + 1], X[3 * vi + 2]};
      r.v[3 * k] = v[k].x; r.v[3 * k + 1] = v[k].y; r.v[3 * k + 2] = v[k].z;
    }
    const d3 e[3] = {v_sub(v[1], v[0]), v_sub(v[2], v[1]), v_sub(v[0], v[2])};
    for (int j = 0; j < 3; ++j) {
      r.L[j] = v_norm(e[j]);
      const d3 u = v_div(e[j], r.L[j]);
      r.u[3 * j] = u.x; r.u[3 * j + 1] = u.y; r.u[3 * j + 2] = u.z;
    }
    const d3 nn = v_cross(e[0], v_neg(e[2]));
    const d3 n = v_div(nn, v_norm(nn));
    r.n[0] = n.x; r.n[1] = n.y; r.n[2] = n.z;
    for (int a = 0; a < 3; ++a) {
      r.bmin[a] = fmin(r.v[a], fmin(r.v[3 + a], r.v[6 + a]));
      r.bmax[a] = fmax(r.v[a], fmax(r.v[3 + a], r.v[6 + a]));
    }
    r.pad = 0;
    factor_bary(r);
    rec[el] = r;
  }
}

__global__ void __launch_bounds__(128) k_na_dist(const unsigned char* scratch, int64_t nel, GridP g, int clamp,
                                                 double* __restrict__ out) {
  const TriRec64* rec = reinterpret_cast<const TriRec64*>(scratch + 256);
  if (*reinterpret_cast<const volatile int*>(scratch) != 0) return;  // bad index: leave the output as it was
  for (int64_t lin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lin < g.ngp; lin += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = lin % g.n[0], j = (lin / g.n[0]) % g.n[1], k = lin / (g.n[0] * g.n[1]);
    const d3 p = node_coord(g.o, g.h, i, j, k);
    double m = 1.0e10;
    d3 proj = {0.0, 0.0, 0.0};
    for (int64_t t = 0; t < nel; ++t) tri_step64(rec[t], p, m, proj, false);
    if (clamp && fabs(m) > fabs(g.h)) m = g.h;
    out[lin] = m;
  }
}

}  // namespace

}  // namespace sdfgpu

using namespace sdfgpu;

extern "C" int sdfgpu_distances_noalloc(const double* d_X, int64_t nnp, const int64_t* d_IEN, int64_t nel,
                                        const double origin[3], double h, const int64_t N[3], int32_t mode,
                                        double* d_dist_out, void* stream) {
  if (!d_X || !d_IEN || !d_dist_out || !origin || !N)
    return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "sdfgpu_distances_noalloc: NULL argument");
  if (mode != SDFGPU_MODE_EXACT && mode != SDFGPU_MODE_UNBOUNDED)
    return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT,
                "sdfgpu_distances_noalloc supports SDFGPU_MODE_EXACT and SDFGPU_MODE_UNBOUNDED only");
  if (nel < 1 || nnp < 3) return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "mesh needs at least 1 triangle and 3 vertices");
  if (nel > kNoAllocMaxTriangles)
    return fail(nullptr, SDFGPU_ERR_CAPACITY,
                "sdfgpu_distances_noalloc holds at most " + std::to_string(kNoAllocMaxTriangles) +
                    " triangles in its fixed device scratch; got " + std::to_string(nel) + " (use sdfgpu_distances)");
  if (!(h > 0.0) || !std::isfinite(h)) return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "cell size must be finite and > 0");
  double ngp_d = 1.0;
  for (int a = 0; a < 3; ++a) {
    if (N[a] < 0 || !std::isfinite(origin[a])) return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "bad grid");
    ngp_d *= (double)(N[a] + 1);
  }
  if (ngp_d > 2147483647.0) return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "grid has more than 2^31-1 nodes");
  if (ngp_d * (double)nel > kNoAllocMaxSteps)
    return fail(nullptr, SDFGPU_ERR_CAPACITY,
                "sdfgpu_distances_noalloc: nodes x triangles exceeds 2^36 FP64 steps (use sdfgpu_distances)");
  // The device address of the array on the current device, looked up on every call (host code
  // may not use the symbol's name as an address).
  void* scratch = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
  if (e != cudaSuccess)
    return fail(nullptr, SDFGPU_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  cudaStream_t st = (cudaStream_t)stream;
  GridP g{};
  for (int a = 0; a < 3; ++a) {
    g.o[a] = origin[a];
    g.N[a] = N[a];
    g.n[a] = N[a] + 1;
  }
  g.h = h;
  g.ngp = g.n[0] * g.n[1] * g.n[2];
  if ((e = cudaMemsetAsync(scratch, 0, sizeof(int), st)) != cudaSuccess)  // the error word starts at zero
    return fail(nullptr, SDFGPU_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  k_na_prep<<<grid_for(nel, 128), 128, 0, st>>>(d_X, nnp, d_IEN, nel, (unsigned char*)scratch);
  k_na_dist<<<grid_for(g.ngp, 128, 148 * 16), 128, 0, st>>>((const unsigned char*)scratch, nel, g,
                                                              mode == SDFGPU_MODE_EXACT, d_dist_out);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return fail(nullptr, SDFGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  int flag = 0;
  if ((e = cudaMemcpyAsync(&flag, scratch, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return fail(nullptr, SDFGPU_ERR_CUDA, std::string("sdfgpu_distances_noalloc: ") + cudaGetErrorString(e));
  if (flag)
    return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "IEN holds an index outside 1..nnp (d_dist_out left unchanged)");
  return SDFGPU_OK;
}
