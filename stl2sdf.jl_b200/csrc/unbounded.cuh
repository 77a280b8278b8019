// unbounded.cuh -- the nearest-triangle search of SDFGPU_MODE_UNBOUNDED and SDFGPU_MODE_LEARNED:
// the kernel arguments, the per-lane FP32 band of candidate triangles with its FP64 resolution in
// ascending triangle index, and the warp's packet traversal of the LBVH (k_unbounded,
// distance.cu; the per-node walk of the training grid, learned.cu, shares the band).
//
// Every search returns, for each node, the FP64 minimum over all triangles of the point-triangle
// distance (tri_step64 without the vertex-skip rule), ties to the lowest triangle index -- the
// result of folding every triangle in index order (dfOnTriangularMesh.jl:101-177 with the true
// minimum).  The FP32 search only decides which triangles can hold that minimum: a child subtree
// is entered when the larger of its axis-aligned and its oriented box distance (OBox, mesh.cu)
// lies within the lane's bound plus the FP32 margin kUnbPadRel E.

#pragma once

#include "common.cuh"

namespace sdfgpu {
namespace {

constexpr double kBig = 1.0e10;  // abs(-1.0e10), the reference's initial running minimum

__device__ __forceinline__ float3 local32(const GridP& g, const d3& p) {
  return make_float3((float)(p.x - g.center[0]), (float)(p.y - g.center[1]), (float)(p.z - g.center[2]));
}

__device__ __forceinline__ void child_box(const BNode& nd, int side, float3& lo, float3& hi) {
  if (side == 0) {
    lo = make_float3(nd.a.x, nd.a.y, nd.a.z);
    hi = make_float3(nd.a.w, nd.b.x, nd.b.y);
  } else {
    lo = make_float3(nd.b.z, nd.b.w, nd.c.x);
    hi = make_float3(nd.c.y, nd.c.z, nd.c.w);
  }
}

constexpr int kUnbWarps = 8;     // warps per CTA of k_unbounded
constexpr int kWarpStack = 64;   // per-warp traversal stack (shared memory)
constexpr int kKeep = 8;         // per-lane triangles kept inside the FP32 band of the minimum

struct UnbArgs {
  GridP g;
  const BNode* nodes;
  const LeafTri* ltri;  // leaf-ordered FP32 triangle records
  const TriRec64* rec;
  float pad;
  float eD_abs, eD_rel;
  int64_t max_visits;
  const float* radius;  // learned radius per brick, at its centre (nullable)
  double* dist;
  double* xp;
  int64_t* counters;
  int32_t b[3];         // brick of one warp: nodes along x, y, z (product 32)
  int64_t nb[3];        // bricks per axis
  int64_t nbricks;
  unsigned long long* next;  // brick queue: warps take the next brick with one atomic (zeroed per launch)
  const OBox* obb;           // oriented boxes of the LBVH children (obb[2 node + side])
  const int64_t* bricks = nullptr;               // nullable: search only these bricks ...
  const unsigned long long* bricks_n = nullptr;  // ... this many (read on the device)
  int64_t* redo = nullptr;                       // the radius-bounded search lists here the bricks ...
  unsigned long long* redo_n = nullptr;          // ... it did not certify (a counter zeroed per launch)
  int64_t redo_base = 0;                         // added to the listed brick index (a batch's item offset)
};

// FP32 margin of every box test of the unbounded searches, as a multiple of the frame's scale E:
// 2e-6 E for the FP32 point-triangle distance and the axis-aligned box distance, plus 2e-5 E for
// the oriented-box bound (its FP32 evaluation and the FP32 rounding of its axes stay below
// 2.3e-6 E for points within E of the centre on every axis).
constexpr float kUnbPadRel = 2.2e-5f;

// Squared lower bound on the distance from p to the child `side` of LBVH node nid: the larger of
// its axis-aligned and its oriented box (leaves: the axis-aligned box only).
__device__ __forceinline__ float child_d2(const UnbArgs& A, const BNode& nd, int nid, int side, float3 p, float3 lo,
                                          float3 hi) {
  const float d = box_d2(p, lo, hi);
  const int c = side ? nd.d.y : nd.d.x;
  if (c & kLeafBit) return d;
  return fmaxf(d, obox_d2(p, A.obb[2 * nid + side]));
}
__device__ __forceinline__ float child_d2(const BNode& nd, const OBox& o, int side, float3 p, float3 lo, float3 hi) {
  const float d = box_d2(p, lo, hi);
  const int c = side ? nd.d.y : nd.d.x;
  if (c & kLeafBit) return d;
  return fmaxf(d, obox_d2(p, o));
}

// Instantiations of the grid searches (k_unbounded, distance.cu; k_unbounded_multi, search_multi.cu):
// kUnbPlain every brick unbounded; kUnbRadius each lane started from its learned radius;
// kUnbListed the plain search over listed bricks.
constexpr int kUnbPlain = 0, kUnbRadius = 1, kUnbListed = 2;
// Lane `lane`'s node (lx, ly, lz) in a warp brick of shape b, and the brick's central lane rep.
__device__ __forceinline__ void brick_lane(const int32_t b[3], int lane, int& lx, int& ly, int& lz, int& rep) {
  lx = lane % b[0];
  ly = (lane / b[0]) % b[1];
  lz = lane / (b[0] * b[1]);
  rep = b[0] / 2 + b[0] * (b[1] / 2 + b[1] * (b[2] / 2));
}

// The warp's next brick from the launch's queue (bricks differ widely in cost, so a static split
// leaves warps idle at the end); every lane gets the same index.
__device__ __forceinline__ int64_t next_brick(const UnbArgs& A, int lane) {
  unsigned long long b = 0ULL;
  if (lane == 0) b = atomicAdd(A.next, 1ULL);
  return (int64_t)__shfl_sync(0xffffffffu, b, 0);
}

// FP32 square root of a leaf's squared distance by the approximate instruction (sqrt.approx.f32:
// within a few units in the last place, below 1e-6 relative -- inside the band's eD_rel = 4e-6 with
// the leaf distance's own 4e-7 d + 6.4e-10 E), one MUFU operation instead of the correctly rounded
// sequence.
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The FP64 step out of line: it is rare on this path, and inlining it would size the registers of
// the whole traversal loop for it.
__device__ __noinline__ void step64_call(const TriRec64* rec, int prim, const d3& p, double& m64, d3& proj) {
  tri_step64(rec[prim], p, m64, proj, false);
}

// Per-lane state of the FP32 search: the smallest FP32 point-triangle distance m (INF before the
// first hit) and the triangles whose FP32 distance lies within band(m) = m + 2 err(m), one of
// which is the true (FP64) nearest: |FP32 - FP64| <= err for every distance, so the FP64 winner t*
// has D32(t*) <= d64(t*) + err <= d64(t_m) + err <= m + 2 err.  The kept triangles live in shared
// memory (slot q of thread x at q * S + x, S the CTA's thread count: consecutive threads,
// consecutive banks), which keeps the traversal's registers low; bits 0..7 of occ mark the slots in
// use (so a new search starts with occ = 0 and no slot needs clearing), bit 8 that the band held
// more than kKeep triangles at some point.
constexpr int kUnbThreads = kUnbWarps * 32;
constexpr unsigned kBandOverflow = 0x100u;
struct LaneBest {
  float m;
  unsigned occ;  // slots in use (bits 0..7), kBandOverflow
  int* t;        // shared: kept triangle ids
  float* d;      // shared: their FP32 distances
};

template <class P>
__device__ __forceinline__ float band_of(const P& A, float m) { return m + 2.f * (A.eD_abs + A.eD_rel * m); }

template <int S, class P>
__device__ __forceinline__ void lane_offer(const P& A, LaneBest& L, float D, int tri) {
  if (D < L.m) {
    L.m = D;
    const float bd = band_of(A, D);
    for (unsigned o = L.occ & 0xffu; o; o &= o - 1u) {  // drop the kept triangles now outside the band
      const int q = __ffs(o) - 1;
      if (L.d[q * S] > bd) L.occ &= ~(1u << q);
    }
  } else if (D > band_of(A, L.m)) {
    return;
  }
  // no duplicate check: a search reaches each leaf at most once (every LBVH node has one parent and
  // is pushed at most once), every search starts with an empty band, and the FP64 re-search of an
  // overflowed band takes its FP64 steps without offering
  const unsigned fr = ~L.occ & 0xffu;
  if (!fr) {
    L.occ |= kBandOverflow;
    return;
  }
  const int q = __ffs(fr) - 1;
  L.d[q * S] = D;
  L.t[q * S] = tri;
  L.occ |= 1u << q;
}

// One warp searches the LBVH for the nearest triangles of its 32 nodes together (a packet
// traversal).  The stack is the warp's, in shared memory; a child is visited when its box lies
// within the bound of at least one active lane -- band(m) of the lane's FP32 minimum, or r0 before
// its first hit -- nearer child first as seen from the brick's central lane `rep`.  Every load of
// a node or triangle is the same address for the whole warp.  kExact: every leaf triangle within a
// lane's bound runs the FP64 step at once (used with a tight r0 for lanes whose band overflowed);
// otherwise leaves only feed the lane's FP32 band.  Returns false when the visit or stack bound is
// exceeded.
template <bool kExact, int S, class P>
__device__ bool warp_search(const P& A, int* stack, int lane, int rep, const d3& p, const float3& p32,
                            bool active, float r0, LaneBest& L, double& m64, d3& proj, uint32_t& fp64,
                            uint32_t& visits_out) {
  int sp = 1;
  if (lane == 0) stack[0] = 0;
  __syncwarp();
  uint32_t visits = 0;  // at most max_visits = 2 nel + 64 < 2^30
  bool ok = true;
  while (sp > 0) {
    if (++visits > A.max_visits) { ok = false; break; }
    const int nid = stack[--sp];
    __syncwarp();
    // the node and both oriented boxes in one round of loads (leaf children carry kNoObb boxes)
    const BNode nd = A.nodes[nid];
    const OBox ob0 = A.obb[2 * nid], ob1 = A.obb[2 * nid + 1];
    float3 lo0, hi0, lo1, hi1;
    child_box(nd, 0, lo0, hi0);
    child_box(nd, 1, lo1, hi1);
    const bool e0 = lo0.x > hi0.x, e1 = lo1.x > hi1.x;  // empty child
    const float d0 = child_d2(nd, ob0, 0, p32, lo0, hi0), d1 = child_d2(nd, ob1, 1, p32, lo1, hi1);
    float lim;
    if (kExact) {
      const float mf = (float)m64;
      lim = fminf(r0, mf + A.eD_abs + A.eD_rel * mf);
    } else {
      lim = L.m < INFINITY ? band_of(A, L.m) : r0 + A.eD_abs + A.eD_rel * r0;
    }
    const float b = lim + A.pad;
    const float b2 = b * b;
    const bool w0 = active && !e0 && d0 <= b2, w1 = active && !e1 && d1 <= b2;
    const unsigned m0 = __ballot_sync(0xffffffffu, w0), m1 = __ballot_sync(0xffffffffu, w1);
    const float rd0 = __shfl_sync(0xffffffffu, e0 ? INFINITY : d0, rep);
    const float rd1 = __shfl_sync(0xffffffffu, e1 ? INFINITY : d1, rep);
    const bool swap = rd1 < rd0;
    const int cn = swap ? nd.d.y : nd.d.x, cf = swap ? nd.d.x : nd.d.y;
    const unsigned mn = swap ? m1 : m0, mfar = swap ? m0 : m1;
    const bool wn = swap ? w1 : w0, wf = swap ? w0 : w1;
#pragma unroll
    for (int q = 0; q < 2; ++q) {  // leaves now, near one first
      const int c = q == 0 ? cn : cf;
      const bool want = q == 0 ? wn : wf;
      if (!(c & kLeafBit) || (q == 0 ? mn : mfar) == 0u) continue;
      const LeafTri T = A.ltri[c & 0x7fffffff];
      const int prim = __float_as_int(T.n.w);
      const float D = sqrt_approx(leaf_d2(p32, T));
      if (kExact) {
        const float mf = (float)m64;
        if (want && D <= fminf(r0, mf + A.eD_abs + A.eD_rel * mf)) {
          step64_call(A.rec, prim, p, m64, proj);
          ++fp64;
        }
      } else {
        const float limq = L.m < INFINITY ? band_of(A, L.m) : r0 + A.eD_abs + A.eD_rel * r0;
        if (want && D <= limq) lane_offer<S>(A, L, D, prim);
      }
    }
    // inner children, the far one pushed first so the near one is popped next
    if (mfar != 0u && !(cf & kLeafBit)) {
      if (sp >= kWarpStack) { ok = false; break; }
      if (lane == 0) stack[sp] = cf;
      ++sp;
    }
    if (mn != 0u && !(cn & kLeafBit)) {
      if (sp >= kWarpStack) { ok = false; break; }
      if (lane == 0) stack[sp] = cn;
      ++sp;
    }
    __syncwarp();
  }
  __syncwarp();
  visits_out += visits;
  return ok;
}

// FP64 steps over the kept triangles inside the final band, in ascending triangle index (so exact
// ties keep the lowest index, as a fold in index order does).
template <int S>
__device__ __forceinline__ void lane_resolve(const UnbArgs& A, const LaneBest& L, const d3& p, double& m64, d3& proj,
                                             uint32_t& fp64) {
  const float bd = band_of(A, L.m);
  int last = -1;
#pragma unroll 1
  for (int it = 0; it < kKeep; ++it) {
    int best = 0x7fffffff;
    for (unsigned o = L.occ & 0xffu; o; o &= o - 1u) {
      const int q = __ffs(o) - 1;
      const int tq = L.t[q * S];
      if (L.d[q * S] <= bd && tq > last && tq < best) best = tq;
    }
    if (best == 0x7fffffff) break;
    step64_call(A.rec, best, p, m64, proj);
    ++fp64;
    last = best;
  }
}


}  // namespace
}  // namespace sdfgpu
