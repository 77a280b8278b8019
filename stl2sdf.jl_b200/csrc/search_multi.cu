// search_multi.cu -- the unbounded (and learned-radius) searches of many meshes in one persistent
// launch, for sdfgpu_sdf_batch_ex(persistent = 1): the multi-mesh kernel over (item, brick) work
// items and its host side.  The brick search itself is the one of k_unbounded (unb_brick.inc); it
// lives in a translation unit of its own so that its out-of-line helpers do not change how the
// single-mesh kernels compile.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "unbounded.cuh"

namespace sdfgpu {
namespace {

// Many meshes' unbounded (or radius-started) searches in one persistent launch.  Work item w of
// [0, off[count]) is brick w - off[m] of item m (off: the exclusive prefix of the items' brick counts,
// then their total); the warps take work items from one queue, and a warp copies an item's
// arguments into its shared slot when its item changes.  kUnbListed: the work items listed in
// `list` (list_n of them: the bricks the radius-started launch did not certify).
template <int kMode>
__global__ void __launch_bounds__(kUnbThreads, 4)
    k_unbounded_multi(const UnbArgs* __restrict__ items, const int64_t* __restrict__ off, int count,
                      unsigned long long* next, const int64_t* __restrict__ list, const unsigned long long* list_n,
                      int64_t* counters) {
  constexpr bool kRadius = kMode == kUnbRadius, kListed = kMode == kUnbListed;
  __shared__ int s_stack[kUnbWarps][kWarpStack];
  // kRadius: each lane's radius and the warp's certified / fallback counts live in shared memory,
  // so the traversal loop keeps the plain search's registers
  __shared__ float s_r[kRadius ? kUnbThreads : 1];
  __shared__ unsigned s_cf[kRadius ? kUnbWarps : 1][2];
  __shared__ int s_keep_t[kKeep * kUnbThreads];
  __shared__ float s_keep_d[kKeep * kUnbThreads];
  __shared__ __align__(16) unsigned char s_args_raw[kUnbWarps][sizeof(UnbArgs)];  // the warp's item (raw: no constructor)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const UnbArgs& args = *reinterpret_cast<const UnbArgs*>(s_args_raw[w]);
  uint32_t fp64 = 0, errs = 0, visits = 0;  // per-thread statistics (far below 2^32)
  if (kRadius && lane == 0) s_cf[w][0] = s_cf[w][1] = 0u;
  const int64_t total = kListed ? (int64_t)*list_n : off[count];
  int cur = -1, lx = 0, ly = 0, lz = 0, rep = 0;
  for (;;) {
    unsigned long long t = 0ULL;
    if (lane == 0) t = atomicAdd(next, 1ULL);
    const int64_t q = (int64_t)__shfl_sync(0xffffffffu, t, 0);
    if (q >= total) break;
    const int64_t gw = kListed ? list[q] : q;
    int lo = 0, hi = count - 1;  // the item: the last m with off[m] <= gw
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (off[mid] <= gw) lo = mid;
      else hi = mid - 1;
    }
    if (lo != cur) {
      __syncwarp();
      const int* src = reinterpret_cast<const int*>(items + lo);
      int* dst = reinterpret_cast<int*>(s_args_raw[w]);
      for (int k = lane; k < (int)(sizeof(UnbArgs) / sizeof(int)); k += 32) dst[k] = src[k];
      __syncwarp();
      cur = lo;
      brick_lane(args.b, lane, lx, ly, lz, rep);
    }
    const UnbArgs& A = args;
    const GridP& g = A.g;
    int* stack = s_stack[w];
    const int64_t brick = gw - off[lo];
#include "unb_brick.inc"
  }
  for (int o = 16; o > 0; o >>= 1) fp64 += __shfl_down_sync(0xffffffffu, fp64, o);
  if (lane == 0) {
    if (fp64) count_add(counters, C_FP64, fp64);
    if (kRadius && s_cf[w][0]) count_add(counters, C_CERTIFIED, s_cf[w][0]);
    if (kRadius && s_cf[w][1]) count_add(counters, C_UNB_FALLBACK, s_cf[w][1]);
    if (errs) count_add(counters, C_ERR_STACK, errs);
    if (visits) count_add(counters, C_VISITS, visits);
  }
}
static_assert(sizeof(UnbArgs) % sizeof(int) == 0, "UnbArgs is copied in 4-byte words");
static_assert(sizeof(UnbArgs) <= sizeof(DistPlan::unb), "DistPlan::unb holds an UnbArgs");

}  // namespace

size_t unb_args_size() { return sizeof(UnbArgs); }

// Points a prepared unbounded plan's list of uncertified bricks at the batch's list: work items are
// numbered across the batch, this item's from `base`.
void plan_set_redo(DistPlan& Pl, int64_t* redo, unsigned long long* redo_n, int64_t base) {
  UnbArgs A;
  std::memcpy(&A, Pl.unb, sizeof(A));
  A.redo = redo;
  A.redo_n = redo_n;
  A.redo_base = base;
  std::memcpy(Pl.unb, &A, sizeof(A));
}

// Resident CTAs of the multi-mesh search (one wave, at most one warp per work item).  Call before a
// stream capture.
int unb_multi_grid(sdfgpu_ctx* ctx, int64_t total, int64_t* grid) {
  int per_sm = 0, sms = 148;
  SDF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_unbounded_multi<kUnbPlain>, kUnbThreads, 0));
  SDF_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  *grid = grid_for(total, kUnbWarps, (int64_t)sms * std::max(per_sm, 1));
  return 0;
}

// The unbounded searches of `count` prepared items in one persistent launch on stream st (launches
// only, so it can be captured in a graph).  d_items: their UnbArgs (plan.unb), d_off: the count + 1
// prefix of their brick counts; heads: 3 counters (the launch's queue, the listed launch's queue,
// the number of listed work items), zeroed here.  radius: the items' searches start from their
// learned radius, and the work items they do not certify (listed in `redo`) run the plain search
// in a second launch.
int unb_multi(sdfgpu_ctx* ctx, const void* d_items, const int64_t* d_off, int count, bool radius, int64_t* redo,
              unsigned long long* heads, int64_t grid, cudaStream_t st) {
  if (count < 1) return 0;
  SDF_CUDA(ctx, cudaMemsetAsync(heads, 0, 3 * sizeof(unsigned long long), st));
  const UnbArgs* it = static_cast<const UnbArgs*>(d_items);
  if (radius) {
    k_unbounded_multi<kUnbRadius><<<(unsigned)grid, kUnbThreads, 0, st>>>(it, d_off, count, heads, nullptr, nullptr,
                                                                           ctx->d_counters);
    SDF_KERNEL(ctx);
    k_unbounded_multi<kUnbListed><<<(unsigned)grid, kUnbThreads, 0, st>>>(it, d_off, count, heads + 1, redo, heads + 2,
                                                                           ctx->d_counters);
  } else {
    k_unbounded_multi<kUnbPlain><<<(unsigned)grid, kUnbThreads, 0, st>>>(it, d_off, count, heads, nullptr, nullptr,
                                                                          ctx->d_counters);
  }
  SDF_KERNEL(ctx);
  return 0;
}

}  // namespace sdfgpu
