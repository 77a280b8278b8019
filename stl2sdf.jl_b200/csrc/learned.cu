// learned.cu -- the exact unbounded distances the learned radius trains on (SDFGPU_MODE_LEARNED):
// the true minimum point-triangle distance (dfOnTriangularMesh.jl:101-177 without the clamp at
// :202-206) at the nodes of a sparse coarse grid, one thread per node and four nodes per warp.  The learned-radius search
// over the full grid is the packet search of SDFGPU_MODE_UNBOUNDED (k_unbounded, distance.cu)
// with every lane's first search bounded by its radius r(p).
#include "common.cuh"
#include "unbounded.cuh"

namespace sdfgpu {

namespace {

struct LearnArgs {
  UnbArgs u;
};


// Exact unbounded distances of a sparse node set (the coarse grid the radius network trains on):
// one thread per node walks the LBVH by itself, nearest child first, with a small stack of (node,
// squared box distance) pairs, entering a child only when its box lies within band(m) of the node
// (m: the FP32 minimum so far) and dropping stacked nodes that have fallen out of the bound without
// loading them.  On a coarse grid neighbouring nodes are far apart, so a warp's walks share little
// and a brick search would take the union of very different regions; per-thread walks do not.
// The walks' loads diverge (one address per active lane), so a warp walks four nodes and the
// coarse grid's few thousand nodes spread over every SM: the 13,824 training nodes of a
// 1.4M-triangle mesh take 2.8 ms of training in all, against 3.9 ms with 32 nodes per warp in
// 128-thread CTAs (8 per warp: 3.0 ms, 2 per warp: 2.8 ms); on a 5.7M-triangle mesh 3.5 ms against
// 3.9 ms (8 per warp: 3.4 ms, 2 per warp: 3.8 ms).
// Results are those of the other unbounded searches (FP64 resolution of the FP32 band in
// ascending triangle index; FP64 re-search of a node whose band overflowed).
constexpr int kPThreads = 32;       // one warp per CTA: the walks spread over every SM
constexpr int kPNodesPerWarp = 4;   // nodes a warp walks at a time, one per lane 0-3 (the rest idle)
constexpr int kTStack = 64;  // per-thread traversal stack (LBVH depth <= 64 for unique 64-bit keys)

template <bool kExact>
__device__ bool point_search(const LearnArgs& LA, const d3& p, const float3& p32, float lim_r, LaneBest& L,
                             double& m64, d3& proj, uint32_t& fp64, uint32_t& visits) {
  const UnbArgs& A = LA.u;
  int st_id[kTStack];
  float st_d[kTStack];
  int sp = 0, cur = 0;
  uint32_t n = 0;  // at most max_visits = 2 nel + 64 < 2^30
  auto bound = [&]() -> float {
    if (kExact) {
      const float mf = (float)m64;
      return fminf(lim_r, mf + A.eD_abs + A.eD_rel * mf);
    }
    return L.m < INFINITY ? fminf(lim_r, band_of(A, L.m)) : lim_r;
  };
  while (true) {
    if (++n > A.max_visits) return false;
    const BNode nd = A.nodes[cur];
    float3 lo0, hi0, lo1, hi1;
    child_box(nd, 0, lo0, hi0);
    child_box(nd, 1, lo1, hi1);
    const int c0 = nd.d.x, c1 = nd.d.y;
    const float d0 = lo0.x > hi0.x ? INFINITY : child_d2(A, nd, cur, 0, p32, lo0, hi0);
    const float d1 = lo1.x > hi1.x ? INFINITY : child_d2(A, nd, cur, 1, p32, lo1, hi1);
#pragma unroll
    for (int k = 0; k < 2; ++k) {  // leaf children, nearer first
      const bool second = (k == 1) == (d0 <= d1);
      const int c = second ? c1 : c0;
      const float dc = second ? d1 : d0;
      if (!(c & kLeafBit)) continue;
      const float b = bound() + A.pad;
      if (!(dc <= b * b)) continue;
      const int leaf = c & 0x7fffffff;
      const LeafTri T = A.ltri[leaf];
      const int prim = __float_as_int(T.n.w);
      const float D = sqrtf(leaf_d2(p32, T));
      if (D > bound()) continue;
      if (kExact) {
        step64_call(A.rec, prim, p, m64, proj);
        ++fp64;
      } else {
        lane_offer<kPThreads>(A, L, D, prim);
      }
    }
    const float b = bound() + A.pad, b2 = b * b;  // inner children: enter the nearer, stack the farther
    const bool g0 = !(c0 & kLeafBit) && d0 <= b2, g1 = !(c1 & kLeafBit) && d1 <= b2;
    if (g0 && g1) {
      if (sp >= kTStack) return false;
      const bool near0 = d0 <= d1;
      st_id[sp] = near0 ? c1 : c0;
      st_d[sp] = near0 ? d1 : d0;
      ++sp;
      cur = near0 ? c0 : c1;
      continue;
    }
    if (g0 || g1) {
      cur = g0 ? c0 : c1;
      continue;
    }
    bool found = false;
    while (sp > 0) {
      --sp;
      const float bb = bound() + A.pad;
      if (st_d[sp] <= bb * bb) {
        cur = st_id[sp];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  visits += n;
  return true;
}

__global__ void __launch_bounds__(kPThreads) k_nearest_points(LearnArgs LA) {
  __shared__ int s_keep_t[kKeep * kPThreads];
  __shared__ float s_keep_d[kKeep * kPThreads];
  const UnbArgs& A = LA.u;
  const GridP& g = A.g;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  uint32_t fp64 = 0, errs = 0, visits = 0;  // per-thread statistics (far below 2^32)
  for (int64_t base = warp * kPNodesPerWarp; base < g.ngp; base += nwarps * kPNodesPerWarp) {
    const int64_t lin = base + lane;
    if (lane >= kPNodesPerWarp || lin >= g.ngp) continue;
    const int64_t i = lin % g.n[0], j = (lin / g.n[0]) % g.n[1], k = lin / (g.n[0] * g.n[1]);
    const d3 p = gnode(g, i, j, k);
    const float3 p32 = local32(g, p);
    LaneBest L;
    L.m = INFINITY;
    L.occ = 0u;
    L.t = s_keep_t + threadIdx.x;
    L.d = s_keep_d + threadIdx.x;
    double m64 = kBig;
    d3 proj = {0.0, 0.0, 0.0};
    bool ok = point_search<false>(LA, p, p32, INFINITY, L, m64, proj, fp64, visits);
    if (ok && (L.occ & kBandOverflow)) ok = point_search<true>(LA, p, p32, band_of(A, L.m), L, m64, proj, fp64, visits);
    else if (ok) lane_resolve<kPThreads>(A, L, p, m64, proj, fp64);
    if (!ok) ++errs;
    A.dist[lin] = m64;
  }
  for (int off = 16; off > 0; off >>= 1) {
    fp64 += __shfl_down_sync(0xffffffffu, fp64, off);
    errs += __shfl_down_sync(0xffffffffu, errs, off);
    visits += __shfl_down_sync(0xffffffffu, visits, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (fp64) count_add(A.counters, C_FP64, fp64);
    if (errs) count_add(A.counters, C_ERR_STACK, errs);
    if (visits) count_add(A.counters, C_VISITS, visits);
  }
}

}  // namespace

namespace {

LearnArgs point_args(sdfgpu_ctx* ctx, const GridP& g, double* d_dist) {
  const float E = (float)g.E;
  LearnArgs LA{};
  UnbArgs& A = LA.u;
  A.g = g;
  A.nodes = buf<BNode>(ctx, "nodes");
  A.obb = buf<OBox>(ctx, "obb");
  A.rec = buf<TriRec64>(ctx, "rec");
  A.pad = kUnbPadRel * E;
  A.eD_abs = 4.0e-6f * E;
  A.eD_rel = 4.0e-6f;
  A.max_visits = 2 * ctx->mesh.nel + 64;
  A.dist = d_dist;
  A.counters = ctx->d_counters;
  A.ltri = buf<LeafTri>(ctx, "ltri");
  return LA;
}

}  // namespace

// Exact unbounded distances of the nodes of a sparse grid, one thread per node (no closest points).
int run_nearest_points(sdfgpu_ctx* ctx, const GridP& g, double* d_dist) {
  const LearnArgs LA = point_args(ctx, g, d_dist);
  const int64_t warps = (g.ngp + kPNodesPerWarp - 1) / kPNodesPerWarp;
  k_nearest_points<<<(unsigned)std::min<int64_t>(warps, 148 * 32), kPThreads, 0, ctx->stream>>>(LA);
  SDF_KERNEL(ctx);
  return 0;
}

}  // namespace sdfgpu
