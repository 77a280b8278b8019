// learned.cu -- the nearest-triangle search of SDFGPU_MODE_LEARNED: the unbounded distance
// (dfOnTriangularMesh.jl:101-177 with the true minimum and no clamp at :202-206) with every node's
// search bounded in advance by the learned radius r(p) (radius.cu).
//
// Why a known bound changes the search.  The plain search (k_unbounded) is a depth-first packet
// traversal: one warp walks the LBVH one node at a time, because each lane's bound only appears as
// leaves are reached, and every step is a dependent load.  With r(p) known before the search, the
// set of LBVH nodes a brick of nodes can need is fixed up front -- every node whose box lies within
// R = max r(p) of the brick's box -- so the warp expands 32 of them per step (one per lane,
// independent loads), and stops descending at subtrees of at most kCluster leaves ("clusters":
// contiguous runs of the Morton-sorted leaves, whose FP32 vertices and boxes are stored in leaf
// order, see k_leaf_order in mesh.cu).  Each lane then tests the gathered clusters against its own
// bound and folds the triangles of the clusters it needs, all lanes in step.  As lanes find
// triangles their bounds shrink to band(m) and the brick bound R shrinks with them.  Before the
// expansion every brick takes one greedy nearest-first descent to a cluster near its centre and
// folds it on every lane, so the lanes' bounds are close to their distances from the start.  With no
// radius array every bound is infinite and the search rests on that seed alone (the coarse grid the
// network trains on is computed this way, and it measures what the network adds).
//
// Certification (the same rule as the plain search seeded with r): a lane whose FP32 minimum m
// satisfies m + err(m) <= r has its FP64 nearest triangle within r, and every triangle within r
// was offered to its band, so the FP64 resolution in ascending triangle index gives the exact
// result.  Lanes without such a minimum, and every lane of a brick whose traversal stack
// overflowed, continue with the plain packet search (warp_search) from what they found, which is
// the fallback the statistics count.  Results are bit-identical to SDFGPU_MODE_UNBOUNDED.
#include "common.cuh"
#include "unbounded.cuh"

namespace sdfgpu {

namespace {

constexpr int kLWarps = 4;                // warps per CTA
constexpr int kLThreads = kLWarps * 32;
constexpr int kLStack = 512;              // per-warp stack of inner LBVH nodes still to expand
constexpr int kLQueue = 96;               // per-warp queue of gathered clusters (<= 31 + 64 at a time)
constexpr int kCluster = 8;               // subtrees of at most this many leaves are folded, not expanded

struct LearnArgs {
  UnbArgs u;
  const float4* lv32;  // leaf-ordered FP32 vertices (3 per leaf)
  const float4* lbox;  // leaf-ordered FP32 boxes (2 per leaf; lo.w = triangle index)
  int64_t max_rounds;  // bound on the expansion rounds of one brick
};

// Squared distance between two boxes.
__device__ __forceinline__ float boxbox_d2(float3 alo, float3 ahi, float3 blo, float3 bhi) {
  const float dx = fmaxf(fmaxf(alo.x - bhi.x, blo.x - ahi.x), 0.f);
  const float dy = fmaxf(fmaxf(alo.y - bhi.y, blo.y - ahi.y), 0.f);
  const float dz = fmaxf(fmaxf(alo.z - bhi.z, blo.z - ahi.z), 0.f);
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

__device__ __forceinline__ float warp_max(float v) {
  for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
  for (int off = 16; off > 0; off >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// The lane's current FP32 search bound: its radius bound until it has a minimum, then the smaller
// of that and band(m).  Negative for lanes outside the grid (they need nothing).
__device__ __forceinline__ float lane_bound(const UnbArgs& A, const LaneBest& L, float lim_r, bool valid) {
  if (!valid) return -1.f;
  return L.m < INFINITY ? fminf(lim_r, band_of(A, L.m)) : lim_r;
}

__global__ void __launch_bounds__(kLThreads) k_learned(LearnArgs LA) {
  __shared__ int s_stack[kLWarps][kLStack];
  __shared__ float4 s_q[kLWarps][kLQueue][2];
  __shared__ int s_keep_t[kKeep * kLThreads];
  __shared__ float s_keep_d[kKeep * kLThreads];
  const UnbArgs& A = LA.u;
  const GridP& g = A.g;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* stack = s_stack[w];
  float4(*Q)[2] = s_q[w];
  const unsigned lt = (1u << lane) - 1u;  // lanes below this one
  const int lx = lane % A.b[0], ly = (lane / A.b[0]) % A.b[1], lz = lane / (A.b[0] * A.b[1]);
  const int rep = A.b[0] / 2 + A.b[0] * (A.b[1] / 2 + A.b[1] * (A.b[2] / 2));
  int64_t fp64 = 0, cert = 0, fallback = 0, errs = 0, visits = 0;
  for (int64_t brick = next_brick(A, lane); brick < A.nbricks; brick = next_brick(A, lane)) {
    const int64_t bx = brick % A.nb[0], by = (brick / A.nb[0]) % A.nb[1], bz = brick / (A.nb[0] * A.nb[1]);
    const int64_t i = bx * A.b[0] + lx, j = by * A.b[1] + ly, k = bz * A.b[2] + lz;
    const bool valid = i <= g.N[0] && j <= g.N[1] && k <= g.N[2];
    const d3 p = gnode(g, min(i, g.N[0]), min(j, g.N[1]), min(k, g.N[2]));
    const float3 p32 = local32(g, p);
    const int64_t lin = i + g.n[0] * (j + g.n[1] * k);
    LaneBest L;
    L.m = INFINITY;
    L.overflow = false;
    L.t = s_keep_t + threadIdx.x;
    L.d = s_keep_d + threadIdx.x;
#pragma unroll
    for (int q = 0; q < kKeep; ++q) {
      L.t[q * kLThreads] = -1;
      L.d[q * kLThreads] = INFINITY;
    }
    double m64 = kBig;
    d3 proj = {0.0, 0.0, 0.0};
    // no radius array: the same search with every bound infinite (it then starts from the seed)
    const float r = !valid ? 0.f : (A.radius ? A.radius[lin] : INFINITY);
    // every triangle with FP64 distance <= r has FP32 distance <= lim_r
    const float lim_r = r + A.eD_abs + A.eD_rel * r;
    const float3 blo = make_float3(warp_min(valid ? p32.x : INFINITY), warp_min(valid ? p32.y : INFINITY),
                                   warp_min(valid ? p32.z : INFINITY));
    const float3 bhi = make_float3(warp_max(valid ? p32.x : -INFINITY), warp_max(valid ? p32.y : -INFINITY),
                                   warp_max(valid ? p32.z : -INFINITY));
    // Seed: one greedy descent toward the brick's centre (the child whose box is nearer, all lanes
    // reading the same node) to the first cluster, folded on every lane, so each lane has a
    // minimum -- close to its own -- before the wide expansion begins.
    {
      const float3 bc = make_float3(0.5f * (blo.x + bhi.x), 0.5f * (blo.y + bhi.y), 0.5f * (blo.z + bhi.z));
      int nid = 0, sfirst = 0, scnt = 0;
      for (int depth = 0; depth < 128; ++depth) {
        const BNode nd = A.nodes[nid];
        float3 lo0, hi0, lo1, hi1;
        child_box(nd, 0, lo0, hi0);
        child_box(nd, 1, lo1, hi1);
        const int gamma = nd.d.x & 0x7fffffff;
        const int n0 = gamma - nd.d.z + 1, n1 = nd.d.w - gamma;
        const float k0 = (lo0.x > hi0.x || n0 < 1) ? INFINITY : box_d2(bc, lo0, hi0);
        const float k1 = (lo1.x > hi1.x || n1 < 1) ? INFINITY : box_d2(bc, lo1, hi1);
        const bool right = k1 < k0;
        const int cid = right ? nd.d.y : nd.d.x, cn = right ? n1 : n0;
        if ((cid & kLeafBit) || cn <= kCluster) {
          sfirst = right ? gamma + 1 : nd.d.z;
          scnt = cn;
          break;
        }
        nid = cid;
      }
      if (valid)
        for (int t = 0; t < scnt; ++t) {
          const int leaf = sfirst + t;
          const float D = sqrtf(pt_tri_d2(p32, f3(LA.lv32[3 * leaf]), f3(LA.lv32[3 * leaf + 1]),
                                          f3(LA.lv32[3 * leaf + 2])));
          if (D <= lane_bound(A, L, lim_r, true)) lane_offer<kLThreads>(A, L, D, __float_as_int(LA.lbox[2 * leaf].w));
        }
    }
    bool ok = true, overflowed = false;
    int sp = 1, q = 0;
    if (lane == 0) stack[0] = 0;
    __syncwarp();
    for (int64_t round = 0;; ++round) {
      if (round > LA.max_rounds) {
        ok = false;
        break;
      }
      if (sp > 0) {  // expand up to 32 inner nodes, one per lane
        const float Rb = warp_max(lane_bound(A, L, lim_r, valid)) + A.pad;
        const float R2 = Rb * Rb;
        const int n = min(sp, 32);
        const int nid = lane < n ? stack[sp - 1 - lane] : -1;
        __syncwarp();
        sp -= n;
        visits += n;
        bool push[2] = {false, false}, clu[2] = {false, false};
        int cid[2] = {0, 0}, first[2] = {0, 0}, cnt[2] = {0, 0};
        float key[2] = {0.f, 0.f};
        float3 clo[2], chi[2];
        if (nid >= 0) {
          const BNode nd = A.nodes[nid];
          child_box(nd, 0, clo[0], chi[0]);
          child_box(nd, 1, clo[1], chi[1]);
          const int gamma = nd.d.x & 0x7fffffff;
          cid[0] = nd.d.x;
          cid[1] = nd.d.y;
          first[0] = nd.d.z;
          cnt[0] = gamma - nd.d.z + 1;
          first[1] = gamma + 1;
          cnt[1] = nd.d.w - gamma;
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            if (clo[c].x > chi[c].x || cnt[c] < 1) continue;  // empty child
            key[c] = boxbox_d2(clo[c], chi[c], blo, bhi);
            if (key[c] > R2) continue;
            if ((cid[c] & kLeafBit) || cnt[c] <= kCluster) clu[c] = true;
            else push[c] = true;
          }
        }
        // each lane's nearer child goes to the upper block (popped first)
        const bool swap = push[0] && push[1] && key[1] < key[0];
        if (swap) {
          const int t = cid[0];
          cid[0] = cid[1];
          cid[1] = t;
        }
        const unsigned mp0 = __ballot_sync(0xffffffffu, push[0]), mp1 = __ballot_sync(0xffffffffu, push[1]);
        const unsigned mc0 = __ballot_sync(0xffffffffu, clu[0]), mc1 = __ballot_sync(0xffffffffu, clu[1]);
        const int np = __popc(mp0) + __popc(mp1), nc = __popc(mc0) + __popc(mc1);
        if (sp + np > kLStack) {  // the brick continues with the plain search
          ok = false;
          overflowed = true;
          break;
        }
        if (push[1]) stack[sp + __popc(mp1 & lt)] = cid[1];  // slot 1 below, slot 0 (the nearer) above
        if (push[0]) stack[sp + __popc(mp1) + __popc(mp0 & lt)] = cid[0];
        if (clu[0]) {
          const int at = q + __popc(mc0 & lt);
          Q[at][0] = make_float4(clo[0].x, clo[0].y, clo[0].z, __int_as_float(first[0]));
          Q[at][1] = make_float4(chi[0].x, chi[0].y, chi[0].z, __int_as_float(cnt[0]));
        }
        if (clu[1]) {
          const int at = q + __popc(mc0) + __popc(mc1 & lt);
          Q[at][0] = make_float4(clo[1].x, clo[1].y, clo[1].z, __int_as_float(first[1]));
          Q[at][1] = make_float4(chi[1].x, chi[1].y, chi[1].z, __int_as_float(cnt[1]));
        }
        sp += np;
        q += nc;
        __syncwarp();
      }
      // fold the newest (up to) 32 clusters until fewer than 32 wait, so the next expansion's (at
      // most 64) clusters fit the queue
      while (q >= 32 || (sp == 0 && q > 0)) {
        const int kq = min(q, 32), base = q - kq;
        float lim = lane_bound(A, L, lim_r, valid);
        float lb = lim + A.pad;
        unsigned mask = 0u;
        for (int c = 0; c < kq; ++c) {
          const float4 a = Q[base + c][0], b = Q[base + c][1];
          if (box_d2(p32, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z)) <= lb * lb) mask |= 1u << c;
        }
        if (!valid) mask = 0u;
        while (mask) {
          const int c = __ffs(mask) - 1;
          mask &= mask - 1u;
          const int f0 = __float_as_int(Q[base + c][0].w), nleaf = __float_as_int(Q[base + c][1].w);
          for (int t = 0; t < nleaf; ++t) {
            const int leaf = f0 + t;
            const float4 bl = LA.lbox[2 * leaf], bh = LA.lbox[2 * leaf + 1];
            lim = lane_bound(A, L, lim_r, true);
            lb = lim + A.pad;
            if (box_d2(p32, make_float3(bl.x, bl.y, bl.z), make_float3(bh.x, bh.y, bh.z)) > lb * lb) continue;
            const float D = sqrtf(pt_tri_d2(p32, f3(LA.lv32[3 * leaf]), f3(LA.lv32[3 * leaf + 1]),
                                            f3(LA.lv32[3 * leaf + 2])));
            if (D <= lim) lane_offer<kLThreads>(A, L, D, __float_as_int(bl.w));
          }
        }
        q = base;
        __syncwarp();
      }
      if (sp == 0 && q == 0) break;
    }
    __syncwarp();
    const bool certified = ok && valid && L.m < INFINITY && L.m + A.eD_abs + A.eD_rel * L.m <= r;
    if (certified) ++cert;
    if (valid && !certified) ++fallback;
    if (!ok && !overflowed && lane == 0) ++errs;  // the round bound was reached (a fault, not a fallback)
    bool good = true;
    if (__any_sync(0xffffffffu, valid && !certified))
      good = warp_search<false, kLThreads>(A, stack, lane, rep, p, p32, valid && !certified, INFINITY, L, m64, proj,
                                           fp64, visits);
    const bool over = valid && L.overflow;
    if (good && __any_sync(0xffffffffu, over))
      good = warp_search<true, kLThreads>(A, stack, lane, rep, p, p32, over, band_of(A, L.m), L, m64, proj, fp64,
                                          visits);
    if (valid && !over) lane_resolve<kLThreads>(A, L, p, m64, proj, fp64);
    if (!good && lane == 0) ++errs;
    if (valid) {
      A.dist[lin] = m64;
      if (A.xp) {
        A.xp[3 * lin] = proj.x;
        A.xp[3 * lin + 1] = proj.y;
        A.xp[3 * lin + 2] = proj.z;
      }
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    fp64 += __shfl_down_sync(0xffffffffu, fp64, off);
    cert += __shfl_down_sync(0xffffffffu, cert, off);
    fallback += __shfl_down_sync(0xffffffffu, fallback, off);
  }
  if (lane == 0) {
    if (fp64) count_add(A.counters, C_FP64, fp64);
    if (cert) count_add(A.counters, C_CERTIFIED, cert);
    if (fallback) count_add(A.counters, C_UNB_FALLBACK, fallback);
    if (errs) count_add(A.counters, C_ERR_STACK, errs);
    if (visits) count_add(A.counters, C_VISITS, visits);
  }
}

// Exact unbounded distances of a sparse node set (the coarse grid the radius network trains on):
// one thread per node walks the LBVH by itself, nearest child first, with a small stack of (node,
// squared box distance) pairs, entering a child only when its box lies within band(m) of the node
// (m: the FP32 minimum so far) and dropping stacked nodes that have fallen out of the bound without
// loading them.  On a coarse grid neighbouring nodes are far apart, so a warp's walks share little
// and a brick search would take the union of very different regions; per-thread walks do not.
// Results are those of the other unbounded searches (FP64 resolution of the FP32 band in
// ascending triangle index; FP64 re-search of a node whose band overflowed).
constexpr int kPThreads = 128;
constexpr int kTStack = 64;  // per-thread traversal stack (LBVH depth <= 64 for unique 64-bit keys)

template <bool kExact>
__device__ bool point_search(const LearnArgs& LA, const d3& p, const float3& p32, float lim_r, LaneBest& L,
                             double& m64, d3& proj, int64_t& fp64, int64_t& visits) {
  const UnbArgs& A = LA.u;
  int st_id[kTStack];
  float st_d[kTStack];
  int sp = 0, cur = 0;
  int64_t n = 0;
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
    const float d0 = lo0.x > hi0.x ? INFINITY : box_d2(p32, lo0, hi0);
    const float d1 = lo1.x > hi1.x ? INFINITY : box_d2(p32, lo1, hi1);
#pragma unroll
    for (int k = 0; k < 2; ++k) {  // leaf children, nearer first
      const bool second = (k == 1) == (d0 <= d1);
      const int c = second ? c1 : c0;
      const float dc = second ? d1 : d0;
      if (!(c & kLeafBit)) continue;
      const float b = bound() + A.pad;
      if (!(dc <= b * b)) continue;
      const int leaf = c & 0x7fffffff;
      const int prim = __float_as_int(LA.lbox[2 * leaf].w);
      const float D = sqrtf(pt_tri_d2(p32, f3(LA.lv32[3 * leaf]), f3(LA.lv32[3 * leaf + 1]), f3(LA.lv32[3 * leaf + 2])));
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
  int64_t fp64 = 0, errs = 0, visits = 0;
  for (int64_t lin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lin < g.ngp; lin += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = lin % g.n[0], j = (lin / g.n[0]) % g.n[1], k = lin / (g.n[0] * g.n[1]);
    const d3 p = gnode(g, i, j, k);
    const float3 p32 = local32(g, p);
    LaneBest L;
    L.m = INFINITY;
    L.overflow = false;
    L.t = s_keep_t + threadIdx.x;
    L.d = s_keep_d + threadIdx.x;
#pragma unroll
    for (int q = 0; q < kKeep; ++q) {
      L.t[q * kPThreads] = -1;
      L.d[q * kPThreads] = INFINITY;
    }
    double m64 = kBig;
    d3 proj = {0.0, 0.0, 0.0};
    bool ok = point_search<false>(LA, p, p32, INFINITY, L, m64, proj, fp64, visits);
    if (ok && L.overflow) ok = point_search<true>(LA, p, p32, band_of(A, L.m), L, m64, proj, fp64, visits);
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

LearnArgs learn_args(sdfgpu_ctx* ctx, const GridP& g, const float* radius, double* d_dist, double* d_xp) {
  const MeshDev& M = ctx->mesh;
  const float E = (float)g.E;
  LearnArgs LA;
  UnbArgs& A = LA.u;
  A.g = g;
  A.nodes = buf<BNode>(ctx, "nodes");
  A.leaf_prim = buf<int32_t>(ctx, "leaf_prim");
  A.v32 = buf<float4>(ctx, "v32");
  A.rec = buf<TriRec64>(ctx, "rec");
  A.pad = 2.0e-6f * E;
  A.eD_abs = 4.0e-6f * E;
  A.eD_rel = 4.0e-6f;
  A.max_visits = 2 * M.nel + 64;
  A.radius = radius;
  A.dist = d_dist;
  A.xp = d_xp;
  A.counters = ctx->d_counters;
  A.nbricks = 1;
  for (int a = 0; a < 3; ++a) {
    A.b[a] = ctx->brick[a];
    A.nb[a] = cdiv(g.n[a], A.b[a]);
    A.nbricks *= A.nb[a];
  }
  LA.lv32 = buf<float4>(ctx, "lv32");
  LA.lbox = buf<float4>(ctx, "lbox32");
  A.next = nullptr;
  LA.max_rounds = 4 * M.nel + 64;  // every round expands at least one node or folds one cluster
  return LA;
}

}  // namespace

// The learned-radius search over the grid g (radius: one FP32 bound per node, or NULL: unbounded).
int run_learned(sdfgpu_ctx* ctx, const GridP& g, const float* radius, double* d_dist, double* d_xp) {
  LearnArgs LA = learn_args(ctx, g, radius, d_dist, d_xp);
  // one resident wave of CTAs draining the brick queue
  SDF_TRY(scratch_t(ctx, "brick_next", 1, &LA.u.next));
  SDF_CUDA(ctx, cudaMemsetAsync(LA.u.next, 0, sizeof(unsigned long long), ctx->stream));
  int per_sm = 0, sms = 148;
  SDF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_learned, kLThreads, 0));
  SDF_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  k_learned<<<grid_for(LA.u.nbricks, kLWarps, (int64_t)sms * (per_sm > 0 ? per_sm : 1)), kLThreads, 0, ctx->stream>>>(LA);
  SDF_KERNEL(ctx);
  return 0;
}

// Exact unbounded distances of the nodes of a sparse grid, one thread per node (no closest points).
int run_nearest_points(sdfgpu_ctx* ctx, const GridP& g, double* d_dist) {
  const LearnArgs LA = learn_args(ctx, g, nullptr, d_dist, nullptr);
  k_nearest_points<<<grid_for(g.ngp, kPThreads, 148 * 16), kPThreads, 0, ctx->stream>>>(LA);
  SDF_KERNEL(ctx);
  return 0;
}

}  // namespace sdfgpu
