// distance.cu -- evalDistancesOnTriMesh (src/SignedDistances/dfOnTriangularMesh.jl:19-209).
//
// Reference semantics (SDFGPU_MODE_REF_RULE).  For node p the candidates are
//   C(p) = { t : |centroid_t - p|^2 <= (2.5 h)^2 }                      (:48, :79)
// or, when C(p) is empty, the triangles of the 3 nearest vertices (:82-94).  They are folded in
// ascending triangle index with the reference's per-candidate step (box reject against the
// running minimum, barycentric face test, edge feet, vertices only when no edge foot improved the
// minimum) and the result is clamped to h (:202-206).
//
// B200 layout of the work:
//   1. tile lists -- the grid is cut into tiles of T0 x T1 x T2 nodes.  One thread per triangle
//      emits a (tile, triangle) pair for every tile its 2.5h centroid ball reaches; a stable CUB
//      radix sort by tile keeps the triangles of each tile in ascending index, which is exactly
//      the fold order.  No per-node sort is ever needed.
//   2. fold -- one CTA per tile, one thread per node.  Every thread walks its tile's sorted list.
//      FP32 does the bulk: the centroid-ball test in mesh-local coordinates and a point-triangle
//      distance D.  A candidate with D > m + err (m = running FP64 minimum) provably cannot change
//      the fold (every value the reference step could assign is >= D), so only candidates inside
//      that band run the FP64 step of exact64.cuh, which replays the reference arithmetic.  Near
//      the surface that is ~ln(|C(p)|) evaluations per node instead of |C(p)|.
//   3. knn fallback -- only meshes whose triangles are large against h (max centroid-to-vertex
//      distance rho >= 1.5h) can have a triangle within h of a node whose C(p) is empty.  For
//      those meshes a triangle scatter flags the nodes within h of any triangle, and those nodes
//      (or, when closest points are requested, every node with empty C(p)) run the 3-nearest-vertex
//      fallback on the LBVH.  Every other node with empty C(p) has a result > h, so it is h.
//
// SDFGPU_MODE_EXACT uses the same tiles with lists of the triangles whose box lies within h of
// the tile; SDFGPU_MODE_UNBOUNDED is a per-node LBVH nearest-triangle search without the clamp.
#include <cub/cub.cuh>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "fold32.cuh"
#include "unbounded.cuh"

namespace sdfgpu {

namespace {


__device__ __forceinline__ void node_ijk(const GridP& g, int64_t lin, int64_t& i, int64_t& j, int64_t& k) {
  i = lin % g.n[0];
  const int64_t r = lin / g.n[0];
  j = r % g.n[1];
  k = r / g.n[1];
}


// Index range [lo, hi] of the nodes whose coordinate along axis a can lie in [x0, x1].
__device__ __forceinline__ bool axis_range(const GridP& g, int a, double x0, double x1, int64_t& lo, int64_t& hi) {
  const double shift = (double)gidx(g, a, 0);
  double f0 = (x0 - g.o[a]) / g.h - shift - 1e-6, f1 = (x1 - g.o[a]) / g.h - shift + 1e-6;
  f0 = fmax(f0, -1.0);
  f1 = fmin(f1, (double)g.N[a] + 1.0);
  if (!(f0 <= f1)) return false;
  lo = (int64_t)ceil(f0);
  hi = (int64_t)floor(f1);
  if (lo < 0) lo = 0;
  if (hi > g.N[a]) hi = g.N[a];
  return lo <= hi;
}

// Emits (tile, triangle) pairs.  REF_RULE: tiles whose nodes can lie within R of the centroid;
// EXACT: tiles whose nodes can lie within R of the triangle's box.
template <bool kFill>
__global__ void k_tile_pairs(const double4* __restrict__ cent, const TriRec64* __restrict__ rec, int64_t nel,
                             GridP g, int mode, double R, int32_t* __restrict__ tri_cnt,
                             const int32_t* __restrict__ tri_off, int32_t* __restrict__ tile_cnt,
                             uint32_t* __restrict__ keys, int32_t* __restrict__ vals, int32_t* __restrict__ nonempty) {
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    double lo[3], hi[3];
    if (mode == SDFGPU_MODE_REF_RULE) {
      const double4 c = cent[el];
      lo[0] = c.x - R; hi[0] = c.x + R;
      lo[1] = c.y - R; hi[1] = c.y + R;
      lo[2] = c.z - R; hi[2] = c.z + R;
    } else {
      for (int a = 0; a < 3; ++a) { lo[a] = rec[el].bmin[a] - R; hi[a] = rec[el].bmax[a] + R; }
    }
    int64_t t0[3], t1[3];
    bool empty = false;
    for (int a = 0; a < 3; ++a) {
      int64_t i0, i1;
      if (!axis_range(g, a, lo[a], hi[a], i0, i1)) { empty = true; break; }
      t0[a] = i0 / g.t[a];
      t1[a] = i1 / g.t[a];
    }
    int32_t count = 0;
    if (!empty) {
      int32_t base = kFill ? tri_off[el] : 0;
      for (int64_t tz = t0[2]; tz <= t1[2]; ++tz)
        for (int64_t ty = t0[1]; ty <= t1[1]; ++ty)
          for (int64_t tx = t0[0]; tx <= t1[0]; ++tx) {
            if (mode == SDFGPU_MODE_REF_RULE) {
              // ball (centre c, radius R) against the tile's node box
              const int64_t ia[3] = {tx * g.t[0], ty * g.t[1], tz * g.t[2]};
              const int64_t ib[3] = {min(ia[0] + g.t[0] - 1, g.N[0]), min(ia[1] + g.t[1] - 1, g.N[1]),
                                     min(ia[2] + g.t[2] - 1, g.N[2])};
              double s = 0.0;
              for (int a = 0; a < 3; ++a) {
                const double c = 0.5 * (lo[a] + hi[a]);
                const double b0 = g.o[a] + g.h * (double)gidx(g, a, ia[a]);
                const double b1 = g.o[a] + g.h * (double)gidx(g, a, ib[a]);
                const double d = c < b0 ? b0 - c : (c > b1 ? c - b1 : 0.0);
                s += d * d;
              }
              if (s > R * R * (1.0 + 1e-9)) continue;
            }
            const uint32_t tile = (uint32_t)((tz * g.nt[1] + ty) * g.nt[0] + tx);
            if (kFill) {
              keys[base + count] = tile;
              vals[base + count] = (int32_t)el;
            } else {
              if (atomicAdd(&tile_cnt[tile], 1) == 0) atomicAdd(nonempty, 1);  // the tile's first pair
            }
            ++count;
          }
    }
    if (!kFill) tri_cnt[el] = count;
  }
}

struct FoldArgs {
  GridP g;
  int mode;
  const int32_t* tile_off;
  const int32_t* tile_cnt;
  const int32_t* order;  // tiles by descending list length: work item w folds tile order[w]
  const int32_t* vals;
  const TriRec64* rec;
  const double4* cent;
  const float4* v32;
  const float4* c32;
  double r2;        // (2.5h)^2, the reference's inrange radius squared
  float r2_in;      // FP32 squared radius below which the centroid test is certain
  float r2_out;     // FP32 squared radius above which the centroid test certainly fails
  float eD_abs;     // FP32 point-triangle distance error bound: eD_abs + eD_rel * m
  float eD_rel;
  double* dist;
  double* xp;
  uint8_t* status;
  int64_t* counters;
};

// Per-warp shared staging of 32 list entries in the tile's local frame (origin = the tile's first
// node): the candidate for the FP32 step, its centroid and box, and per (entry, lane) the squared
// FP32 point-triangle distance that survived phase A, in units of h^2 and rounded down to FP16.
// Rounding is monotone, so rd16(fl(D2 / h^2)) <= fl(fl(lim^2) / h^2) whenever D2 <= fl(lim^2): phase
// B's recheck against the running minimum passes every entry its FP32 form would pass (at worst a
// few more, which the step then leaves unchanged), at half the shared memory, which buys occupancy.
struct __align__(16) WarpStage {
  Cand32 c[32];
  float4 cc[32];          // centroid - origin; .w = |centroid - origin|
  float4 lo[32], hi[32];  // box of the triangle in the local frame
  __half D2[32][32];      // [entry][lane]: rd16(squared FP32 point-triangle distance / h^2)
};

// One CTA per tile, one lane per node.  The tile's ascending triangle list is consumed 32 entries
// at a time.
//   Phase A (FP32, all lanes in step): centroid-ball test (FP64 only inside its error band), box
//   test and point-triangle distance D against the running minimum m: an entry farther than m
//   cannot change the fold, because every value the reference step assigns is at least the true
//   point-triangle distance.
//   Phase B: lanes drain their surviving entries lowest-first (ascending triangle index) through
//   the FP32 replay of the reference step (fold32.cuh).  Only a decision inside its error band
//   runs the FP64 reference step (exact64.cuh); the FP64 value of the final winner is recomputed
//   once, so the output has the reference arithmetic's bits.
__device__ __forceinline__ void fold_tile(const FoldArgs& A, int64_t item, unsigned char* smem_raw) {
  const int64_t tile = A.order[item];
  WarpStage& S = reinterpret_cast<WarpStage*>(smem_raw)[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31;
  const GridP& g = A.g;
  const int64_t tx = tile % g.nt[0], ty = (tile / g.nt[0]) % g.nt[1], tz = tile / (g.nt[0] * g.nt[1]);
  const int lx = threadIdx.x % g.t[0], ly = (threadIdx.x / g.t[0]) % g.t[1], lz = threadIdx.x / (g.t[0] * g.t[1]);
  const int64_t i = tx * g.t[0] + lx, j = ty * g.t[1] + ly, k = tz * g.t[2] + lz;
  // lz < t[2]: a CTA larger than the tile (a multi-mesh launch sized for its largest tile) has threads
  // past the tile, which only take part in the warp-wide steps
  const bool valid = lz < g.t[2] && i <= g.N[0] && j <= g.N[1] && k <= g.N[2];
  const int64_t lin = i + g.n[0] * (j + g.n[1] * k);
  const d3 p = gnode(g, i, j, k);
  const d3 t0 = gnode(g, tx * g.t[0], ty * g.t[1], tz * g.t[2]);
  const float3 pl = make_float3((float)(p.x - t0.x), (float)(p.y - t0.y), (float)(p.z - t0.z));
  const float plen = len3(pl);
  const float sr = (float)(2.5 * g.h);
  const float ih2 = fminf((float)(1.0 / (g.h * g.h)), 1.0e30f);  // finite, so 0 * ih2 is 0
  const int32_t start = A.tile_off[tile], end = start + A.tile_cnt[tile];
  const bool ref = A.mode == SDFGPU_MODE_REF_RULE;
  // running minimum: FP32 estimate m32 (error em), exact m64 when m64_ok, else the winner to
  // recompute it from
  double m64 = kBig;
  d3 proj = {0.0, 0.0, 0.0};
  bool m64_ok = true, any = false;
  float m32 = (float)kBig, em = 0.f;
  int win_tri = -1, win_feat = 0, win_gid = -1;
  int64_t fp64 = 0;
  for (int32_t base = start; base < end; base += 32) {
    const int nE = min(32, end - base);
    if ((int)lane < nE) {
      const int32_t tri = __ldg(&A.vals[base + lane]);
      const TriRec64& r = A.rec[tri];
      const d3 v0 = rec_v(r, 0), v1 = rec_v(r, 1), v2 = rec_v(r, 2);
      const float3 a = make_float3((float)(v0.x - t0.x), (float)(v0.y - t0.y), (float)(v0.z - t0.z));
      const float3 e1 = make_float3((float)(v1.x - v0.x), (float)(v1.y - v0.y), (float)(v1.z - v0.z));
      const float3 e2 = make_float3((float)(v2.x - v0.x), (float)(v2.y - v0.y), (float)(v2.z - v0.z));
      const bool ok = __ldg(&A.c32[tri]).w != 0.f;
      make_cand(a, e1, e2, ok, __float_as_int(__ldg(&A.v32[3 * tri]).w), __float_as_int(__ldg(&A.v32[3 * tri + 1]).w),
                __float_as_int(__ldg(&A.v32[3 * tri + 2]).w), tri, S.c[lane]);
      const double4 cd = A.cent[tri];
      const float3 cc = make_float3((float)(cd.x - t0.x), (float)(cd.y - t0.y), (float)(cd.z - t0.z));
      S.cc[lane] = make_float4(cc.x, cc.y, cc.z, len3(cc));
      const float3 b = a + e1, q = a + e2;
      S.lo[lane] = make_float4(fminf(a.x, fminf(b.x, q.x)), fminf(a.y, fminf(b.y, q.y)), fminf(a.z, fminf(b.z, q.z)), 0.f);
      S.hi[lane] = make_float4(fmaxf(a.x, fmaxf(b.x, q.x)), fmaxf(a.y, fmaxf(b.y, q.y)), fmaxf(a.z, fmaxf(b.z, q.z)), 0.f);
    }
    __syncwarp();
    uint32_t bits = 0;
    if (valid) {
      for (int q = 0; q < nE; ++q) {
        if (ref) {
          const float4 cc = S.cc[q];
          const float dx = cc.x - pl.x, dy = cc.y - pl.y, dz = cc.z - pl.z;
          const float s32 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          const float ec = kU * 16.f * (plen + cc.w);
          if (s32 > (sr + ec) * (sr + ec)) continue;
          if (s32 >= (sr - ec) * (sr - ec)) {  // inside the FP32 error band: the reference's test decides
            const double4 cd = A.cent[S.c[q].gid.w];
            const double ex = ds(cd.x, p.x), ey = ds(cd.y, p.y), ez = ds(cd.z, p.z);
            double s = dm(ex, ex);
            s = da(s, dm(ey, ey));
            s = da(s, dm(ez, ez));
            if (!(s <= A.r2)) continue;
          }
        }
        any = true;
        const Cand32& c = S.c[q];
        const float lim = m32 + em + cand_err(c, plen);
        const float lim2 = lim * lim;
        if (box_d2(pl, f3(S.lo[q]), f3(S.hi[q])) > lim2) continue;
        const float D2 = cand_d2(pl, c);
        if (D2 <= lim2) {
          bits |= 1u << q;
          S.D2[q][lane] = __float2half_rd(D2 * ih2);
        }
      }
    }
    while (__any_sync(0xffffffffu, bits != 0)) {
      // each lane skips, in ascending order, the entries the running minimum has since excluded, so
      // a warp iteration runs one step on every lane that still has a live entry
      int q = -1;
      while (bits) {
        const int qq = __ffs(bits) - 1;
        bits &= bits - 1;
        const float lim = m32 + em + cand_err(S.c[qq], plen);
        if (__half2float(S.D2[qq][lane]) <= lim * lim * ih2) {
          q = qq;
          break;
        }
      }
      if (q >= 0) {
        const Cand32& c = S.c[q];
        {
          float val, err;
          int feat;
          const int act = step32(pl, plen, c, m32, em, ref, win_gid, val, feat, err);
          if (act == S_ASSIGN) {
            m32 = val;
            em = err;
            win_tri = c.gid.w;
            win_feat = feat;
            win_gid = feat >= F_VERT0 ? (feat == F_VERT0 ? c.gid.x : (feat == F_VERT1 ? c.gid.y : c.gid.z)) : -1;
            m64_ok = false;
          } else if (act == S_AMBIG) {
            if (!m64_ok) {
              feature64(A.rec[win_tri], p, win_feat, m64, proj);
              m64_ok = true;
            }
            tri_step64(A.rec[c.gid.w], p, m64, proj, ref);
            m32 = (float)m64;
            em = kU * 2.f * m32;
            win_gid = -1;
            ++fp64;
          }
        }
      }
    }
    __syncwarp();
  }
  int cand = 0;
  if (valid) {
    const bool clamped = m32 - em > (float)g.h * (1.0f + 4.0f * kU);
    if (!m64_ok && (!clamped || A.xp)) {
      feature64(A.rec[win_tri], p, win_feat, m64, proj);
      m64_ok = true;
      ++fp64;
    }
    double d = m64_ok ? m64 : g.h;
    if (fabs(d) > fabs(g.h)) d = g.h;  // clamp (dfOnTriangularMesh.jl:202-206)
    A.dist[lin] = d;
    if (A.xp) {
      A.xp[3 * lin] = proj.x;
      A.xp[3 * lin + 1] = proj.y;
      A.xp[3 * lin + 2] = proj.z;
    }
    A.status[lin] = any ? 1 : 0;
    cand = any ? 1 : 0;
  }
  // warp-aggregated counters
  for (int off = 16; off > 0; off >>= 1) {
    fp64 += __shfl_down_sync(0xffffffffu, fp64, off);
    cand += __shfl_down_sync(0xffffffffu, cand, off);
  }
  if (lane == 0) {
    if (fp64) count_add(A.counters, C_FP64, fp64);
    if (cand) count_add(A.counters, C_CAND_NODES, cand);
  }
}


__global__ void __launch_bounds__(256) k_tile_fold(FoldArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fold_tile(A, blockIdx.x, smem_raw);
}

// The fold of many meshes in one persistent launch: work item w (0 <= w < total) is tile
// w - off[m] of mesh m, off[] the exclusive prefix of the meshes' tile counts; CTAs stride over the
// items.  Each mesh keeps its own tile shape; the CTA holds the largest tile of the batch.
__global__ void __launch_bounds__(256) k_tile_fold_multi(const FoldArgs* __restrict__ args,
                                                         const int64_t* __restrict__ off, int nmesh, int64_t total) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) unsigned char sA_raw[sizeof(FoldArgs)];
  __shared__ int s_mesh;
  FoldArgs& sA = *reinterpret_cast<FoldArgs*>(sA_raw);
  for (int64_t w = blockIdx.x; w < total; w += gridDim.x) {
    if (threadIdx.x == 0) {
      int lo = 0, hi = nmesh - 1;  // the last mesh whose first item is <= w
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= w) lo = mid; else hi = mid - 1;
      }
      s_mesh = lo;
      sA = args[lo];
    }
    __syncthreads();
    fold_tile(sA, w - off[s_mesh], smem_raw);
    __syncthreads();  // sA and s_mesh are rewritten for the next item
  }
}

// Sort keys of the tile order: list length saturated to 16 bits, and the tile index.
// The nodes of tiles without candidates: a node with an empty candidate set clamps to h
// (dfOnTriangularMesh.jl:202-206; the 3-nearest-vertex fallback, when the mesh needs it, runs after
// and finds these nodes by their status 0).  One coalesced pass over the nodes instead of a fold
// CTA per empty tile; it writes exactly what fold_tile writes for such a tile.
__global__ void k_fill_empty(GridP g, const int32_t* __restrict__ tile_cnt, double* __restrict__ dist,
                             double* __restrict__ xp, uint8_t* __restrict__ status) {
  for (int64_t lin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lin < g.ngp; lin += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j, k;
    node_ijk(g, lin, i, j, k);
    const int64_t tile = (k / g.t[2] * g.nt[1] + j / g.t[1]) * g.nt[0] + i / g.t[0];
    if (tile_cnt[tile] != 0) continue;
    dist[lin] = g.h;
    status[lin] = 0;
    if (xp) {
      xp[3 * lin] = 0.0;
      xp[3 * lin + 1] = 0.0;
      xp[3 * lin + 2] = 0.0;
    }
  }
}

__global__ void k_tile_keys(const int32_t* __restrict__ cnt, int64_t n, uint16_t* __restrict__ key,
                            int32_t* __restrict__ idx) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    key[q] = (uint16_t)min(cnt[q], 65535);
    idx[q] = (int32_t)q;
  }
}

// Flags the nodes within h (+ FP32 margin) of a triangle.
__global__ void k_band(const float4* __restrict__ v32, const TriRec64* __restrict__ rec, int64_t nel, GridP g,
                       double hb, float hb2, uint8_t* __restrict__ band) {
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo[3], hi[3];
    bool empty = false;
    for (int a = 0; a < 3; ++a)
      if (!axis_range(g, a, rec[el].bmin[a] - hb, rec[el].bmax[a] + hb, lo[a], hi[a])) { empty = true; break; }
    if (empty) continue;
    const float3 a = f3(v32[3 * el]), b = f3(v32[3 * el + 1]), c = f3(v32[3 * el + 2]);
    for (int64_t k = lo[2]; k <= hi[2]; ++k)
      for (int64_t j = lo[1]; j <= hi[1]; ++j)
        for (int64_t i = lo[0]; i <= hi[0]; ++i) {
          const d3 p = gnode(g, i, j, k);
          if (pt_tri_d2(local32(g, p), a, b, c) <= hb2) band[i + g.n[0] * (j + g.n[1] * k)] = 1;
        }
  }
}

constexpr int kStack = 64;
constexpr int kKnnCap = 256;

struct KnnArgs {
  GridP g;
  const uint8_t* status;
  const uint8_t* band;  // NULL: every node with an empty candidate set
  const BNode* nodes;
  const int32_t* leaf_prim;
  const int32_t* tri_idx;  // not used (IEN64 is read instead)
  const int64_t* IEN;
  const double* X;
  const int32_t* ine_off;
  const int32_t* ine;
  const TriRec64* rec;
  float pad;
  int64_t max_visits;
  double* dist;
  double* xp;
  int64_t* counters;
};

// knn(vtx_kdtree, p, 3) + union of INE + ordered fold (dfOnTriangularMesh.jl:82-177).
__global__ void k_knn_fallback(KnnArgs A) {
  const GridP& g = A.g;
  int64_t done = 0;
  for (int64_t lin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lin < g.ngp; lin += (int64_t)gridDim.x * blockDim.x) {
    if (A.status[lin]) continue;
    if (A.band && !A.band[lin]) continue;
    int64_t i, j, k;
    node_ijk(g, lin, i, j, k);
    const d3 p = gnode(g, i, j, k);
    const float3 p32 = local32(g, p);
    double bs[3] = {INFINITY, INFINITY, INFINITY};
    int64_t bv[3] = {-1, -1, -1};
    int stack[kStack];
    int sp = 0;
    stack[sp++] = 0;
    bool overflow = false;
    int64_t visits = 0;
    while (sp > 0) {
      if (++visits > A.max_visits) { overflow = true; break; }
      const BNode nd = A.nodes[stack[--sp]];
      const float r = isinf(bs[2]) ? INFINITY : (float)sqrt(bs[2]) + A.pad;
      const int ch[2] = {nd.d.x, nd.d.y};
      for (int side = 0; side < 2; ++side) {
        float3 lo, hi;
        child_box(nd, side, lo, hi);
        if (lo.x > hi.x) continue;
        if (!isinf(r) && box_d2(p32, lo, hi) > r * r) continue;
        if (ch[side] & kLeafBit) {
          const int prim = A.leaf_prim[ch[side] & 0x7fffffff];
          for (int q = 0; q < 3; ++q) {
            const int64_t vi = A.IEN[3 * (int64_t)prim + q] - 1;
            if (vi == bv[0] || vi == bv[1] || vi == bv[2]) continue;
            const double dx = ds(A.X[3 * vi], p.x), dy = ds(A.X[3 * vi + 1], p.y), dz = ds(A.X[3 * vi + 2], p.z);
            double s = dm(dx, dx);
            s = da(s, dm(dy, dy));
            s = da(s, dm(dz, dz));
            // insert (s, vi) into the sorted top 3 (ties to the lower vertex index)
            int pos = 3;
            while (pos > 0 && (s < bs[pos - 1] || (s == bs[pos - 1] && vi < bv[pos - 1]))) --pos;
            if (pos < 3) {
              for (int z = 2; z > pos; --z) { bs[z] = bs[z - 1]; bv[z] = bv[z - 1]; }
              bs[pos] = s;
              bv[pos] = vi;
            }
          }
        } else {
          if (sp >= kStack) { overflow = true; break; }
          stack[sp++] = ch[side];
        }
      }
      if (overflow) break;
    }
    if (overflow) { count_add(A.counters, C_ERR_STACK, 1); continue; }
    int32_t cand[kKnnCap];
    int nc = 0;
    for (int q = 0; q < 3 && !overflow; ++q) {
      if (bv[q] < 0) continue;
      for (int32_t e = A.ine_off[bv[q]]; e < A.ine_off[bv[q] + 1]; ++e) {
        if (nc >= kKnnCap) { overflow = true; break; }
        cand[nc++] = A.ine[e];
      }
    }
    if (overflow) { count_add(A.counters, C_ERR_CAPACITY, 1); continue; }
    for (int a = 1; a < nc; ++a) {  // insertion sort, then unique
      const int32_t v = cand[a];
      int b = a - 1;
      while (b >= 0 && cand[b] > v) { cand[b + 1] = cand[b]; --b; }
      cand[b + 1] = v;
    }
    double m = kBig;
    d3 proj = {0.0, 0.0, 0.0};
    for (int a = 0; a < nc; ++a) {
      if (a > 0 && cand[a] == cand[a - 1]) continue;
      tri_step64(A.rec[cand[a]], p, m, proj, true);
    }
    double d = m;
    if (fabs(d) > fabs(g.h)) d = g.h;
    A.dist[lin] = d;
    if (A.xp) {
      A.xp[3 * lin] = proj.x;
      A.xp[3 * lin + 1] = proj.y;
      A.xp[3 * lin + 2] = proj.z;
    }
    ++done;
  }
  for (int off = 16; off > 0; off >>= 1) done += __shfl_down_sync(0xffffffffu, done, off);
  if ((threadIdx.x & 31) == 0 && done) count_add(A.counters, C_KNN, done);
}

// True nearest triangle of every node (no clamp), one warp per brick of 32 nodes.  With a learned
// radius (predicted at the brick centre c, r = rc + |p - c| for node p) each lane's search starts
// bounded by r, and a lane that finds a triangle below r is exact (below).  Lanes whose band
// overflowed search once more with FP64 steps bounded by the band.
// kMode kUnbPlain: every brick, unbounded.  kUnbRadius (the learned mode, A.radius set): one pass
// that starts each lane's minimum at its radius r; a brick with a lane that the pass does not
// certify is appended to A.redo and left unwritten.  kUnbListed: the plain search over the bricks
// listed in A.bricks (the learned mode's second launch).



template <int kMode>
__global__ void __launch_bounds__(kUnbThreads, 4) k_unbounded(UnbArgs A) {
  constexpr bool kRadius = kMode == kUnbRadius, kListed = kMode == kUnbListed;
  __shared__ int s_stack[kUnbWarps][kWarpStack];
  // kRadius: each lane's radius and the warp's certified / fallback counts live in shared memory,
  // so the traversal loop keeps the plain search's registers
  __shared__ float s_r[kRadius ? kUnbThreads : 1];
  __shared__ unsigned s_cf[kRadius ? kUnbWarps : 1][2];
  __shared__ int s_keep_t[kKeep * kUnbThreads];
  __shared__ float s_keep_d[kKeep * kUnbThreads];
  const GridP& g = A.g;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* stack = s_stack[w];
  const int lx = lane % A.b[0], ly = (lane / A.b[0]) % A.b[1], lz = lane / (A.b[0] * A.b[1]);
  const int rep = A.b[0] / 2 + A.b[0] * (A.b[1] / 2 + A.b[1] * (A.b[2] / 2));
  // per-thread statistics (32-bit: a thread's totals stay far below 2^32)
  uint32_t fp64 = 0, errs = 0, visits = 0;
  if (kRadius && lane == 0) s_cf[w][0] = s_cf[w][1] = 0u;
  const int64_t total = kListed ? (int64_t)*A.bricks_n : A.nbricks;
  for (int64_t q = next_brick(A, lane); q < total; q = next_brick(A, lane)) {
    const int64_t brick = kListed ? A.bricks[q] : q;
#include "unb_brick.inc"
  }
  for (int off = 16; off > 0; off >>= 1) fp64 += __shfl_down_sync(0xffffffffu, fp64, off);
  if (lane == 0) {
    if (fp64) count_add(A.counters, C_FP64, fp64);
    if (kRadius && s_cf[w][0]) count_add(A.counters, C_CERTIFIED, s_cf[w][0]);
    if (kRadius && s_cf[w][1]) count_add(A.counters, C_UNB_FALLBACK, s_cf[w][1]);
    if (errs) count_add(A.counters, C_ERR_STACK, errs);
    if (visits) count_add(A.counters, C_VISITS, visits);
  }
}


int ceil_log2(uint64_t v) {
  int b = 0;
  while ((1ULL << b) < v) ++b;
  return b < 1 ? 1 : b;
}

}  // namespace

namespace {

// The unbounded search's arguments for grid g on the current mesh (FP32 error model as in
// run_distances), with the learned radius of every brick when use_learned and the network's bound
// is on; the context stream waits for the LBVH and its oriented boxes.
int unb_setup(sdfgpu_ctx* ctx, const GridP& g, int use_learned, double* d_dist, double* d_xp, UnbArgs& A) {
  // FP32 error model: coordinates in the mesh-local frame are within E, so each FP32 coordinate
  // carries at most 2^-24 E; the distance band (4e-6 E + 4e-6 d) keeps a >= 5x margin over the
  // worst accumulation, the box margin kUnbPadRel E a >= 8x one.
  const float E = (float)g.E;
  SDF_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_obb, 0));  // the search walks the LBVH and its oriented boxes
  A = UnbArgs{g, buf<BNode>(ctx, "nodes"), buf<LeafTri>(ctx, "ltri"), buf<TriRec64>(ctx, "rec"), kUnbPadRel * E,
             4.0e-6f * E, 4.0e-6f, 2 * ctx->mesh.nel + 64, nullptr, d_dist, d_xp, ctx->d_counters};
  A.obb = buf<OBox>(ctx, "obb");
  A.nbricks = 1;
  for (int a = 0; a < 3; ++a) {
    A.b[a] = ctx->brick[a];
    A.nb[a] = cdiv(g.n[a], A.b[a]);
    A.nbricks *= A.nb[a];
  }
  if (use_learned) {
    // the network's radius at each brick centre c, rc = (dhat (1 + alpha) + beta * coarse spacing
    // / s) s (a margin for the network's error and for the interpolation between its training
    // nodes); a node p of the brick searches within rc + |p - c| (k_unbounded).  alpha = +inf:
    // no radius, the same search without the network's bound.
    const RadiusNorm& R = ctx->radius;
    if (!std::isinf(R.alpha)) {
      float* radius;
      SDF_TRY(scratch_t(ctx, "radius", (size_t)A.nbricks, &radius));
      SDF_TRY(run_radius(ctx, &g, nullptr, A.nbricks, R.alpha, (float)(R.beta * R.coarse_h / R.s), radius, A.b));
      A.radius = radius;
    }
  }
  return 0;
}

}  // namespace

int run_distances(sdfgpu_ctx* ctx, const GridP& g, int mode, int use_learned, double* d_dist, double* d_xp) {
  cudaStream_t st = ctx->stream;
  if (mode == SDFGPU_MODE_UNBOUNDED) {
    UnbArgs A;
    SDF_TRY(unb_setup(ctx, g, use_learned, d_dist, d_xp, A));
    SDF_MARK(ctx, T_TILES);
    // one resident wave of CTAs draining the brick queue: queue heads of the two launches and the
    // count of bricks handed from the bounded to the plain search, zeroed together
    unsigned long long* heads;
    SDF_TRY(scratch_t(ctx, "brick_next", 3, &heads));
    SDF_CUDA(ctx, cudaMemsetAsync(heads, 0, 3 * sizeof(unsigned long long), st));
    int per_sm = 0, sms = 148;
    SDF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_unbounded<kUnbPlain>, kUnbWarps * 32, 0));
    SDF_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const unsigned grid = grid_for(A.nbricks, kUnbWarps, (int64_t)sms * std::max(per_sm, 1));
    A.next = heads;
    if (A.radius) {
      SDF_TRY(scratch_t(ctx, "brick_redo", (size_t)A.nbricks, &A.redo));
      A.redo_n = heads + 2;
      k_unbounded<kUnbRadius><<<grid, kUnbWarps * 32, 0, st>>>(A);
      SDF_KERNEL(ctx);
      A.radius = nullptr;  // the listed bricks (usually none), with the plain search
      A.bricks = A.redo;
      A.bricks_n = A.redo_n;
      A.next = heads + 1;
      k_unbounded<kUnbListed><<<grid, kUnbWarps * 32, 0, st>>>(A);
    } else {
      k_unbounded<kUnbPlain><<<grid, kUnbWarps * 32, 0, st>>>(A);
    }
    SDF_KERNEL(ctx);
    SDF_MARK(ctx, T_FOLD);
    return 0;
  }

  DistPlan P;
  SDF_TRY(dist_prepare(ctx, g, mode, d_dist, d_xp, P));
  SDF_MARK(ctx, T_TILES);
  SDF_TRY(dist_fold(ctx, P));
  SDF_MARK(ctx, T_FOLD);
  if (P.knn) SDF_TRY(dist_knn(ctx, P, st, true));
  return 0;
}

// Tile lists of the reference rule (or the h-bounded exact mode) and the fold's arguments; when the
// mesh needs the 3-nearest-vertex fallback, its incidence lists, band flags and arguments too.
// A batch item's unbounded (or learned) search, prepared for the multi-mesh launch: its arguments
// and, in the learned mode, the radius of every brick, in the item's own buffers.
int unb_prepare(sdfgpu_ctx* ctx, const GridP& g, int use_learned, double* d_dist, double* d_xp, DistPlan& Pl) {
  UnbArgs A;
  SDF_TRY(unb_setup(ctx, g, use_learned, d_dist, d_xp, A));
  std::memcpy(Pl.unb, &A, sizeof(A));
  Pl.g = g;
  Pl.unbounded = true;
  Pl.unb_radius = A.radius != nullptr;
  Pl.nbricks = A.nbricks;
  Pl.ntiles = 0;
  Pl.knn = false;
  return 0;
}

int dist_prepare(sdfgpu_ctx* ctx, const GridP& g, int mode, double* d_dist, double* d_xp, DistPlan& Pl,
                 int use_learned) {
  if (mode == SDFGPU_MODE_UNBOUNDED) return unb_prepare(ctx, g, use_learned, d_dist, d_xp, Pl);
  static_assert(sizeof(FoldArgs) <= sizeof(Pl.fold), "DistPlan::fold too small");
  static_assert(sizeof(KnnArgs) <= sizeof(Pl.knn_args), "DistPlan::knn_args too small");
  cudaStream_t st = ctx->stream;
  const MeshDev& M = ctx->mesh;
  const int64_t nel = M.nel;
  TriRec64* rec = buf<TriRec64>(ctx, "rec");
  double4* cent = buf<double4>(ctx, "cent64");
  float4* v32 = buf<float4>(ctx, "v32");
  float4* c32 = buf<float4>(ctx, "c32");
  const float E = (float)g.E;
  const float eD_abs = 4.0e-6f * E;
  const float eD_rel = 4.0e-6f;
  const float pad = 2.0e-6f * E;
  const double sr = 2.5 * g.h;
  const double R = mode == SDFGPU_MODE_REF_RULE ? sr * (1.0 + 1e-9) + 1e-6 * g.E : g.h * (1.0 + 1e-9) + 1e-6 * g.E;
  int32_t *tri_cnt, *tri_off, *tile_cnt, *tile_off, *vals, *vals2;
  uint32_t *keys, *keys2;
  uint8_t* status;
  SDF_TRY(scratch_t(ctx, "tri_cnt", (size_t)nel + 1, &tri_cnt));
  SDF_TRY(scratch_t(ctx, "tri_off", (size_t)nel + 1, &tri_off));
  SDF_TRY(scratch_t(ctx, "tile_cnt", (size_t)g.ntiles + 1, &tile_cnt));
  SDF_TRY(scratch_t(ctx, "tile_off", (size_t)g.ntiles + 1, &tile_off));
  SDF_TRY(scratch_t(ctx, "status", (size_t)g.ngp, &status));
  SDF_CUDA(ctx, cudaMemsetAsync(tile_cnt, 0, sizeof(int32_t) * (g.ntiles + 1), st));
  SDF_CUDA(ctx, cudaMemsetAsync(tri_cnt + nel, 0, sizeof(int32_t), st));
  int32_t* nonempty;
  SDF_TRY(scratch_t(ctx, "tile_nonempty", 1, &nonempty));
  SDF_CUDA(ctx, cudaMemsetAsync(nonempty, 0, sizeof(int32_t), st));
  k_tile_pairs<false><<<grid_for(nel, 128), 128, 0, st>>>(cent, rec, nel, g, mode, R, tri_cnt, nullptr, tile_cnt,
                                                          nullptr, nullptr, nonempty);
  SDF_KERNEL(ctx);
  SDF_TRY(cub_scan_i32(ctx, tri_cnt, tri_off, nel + 1));
  int32_t total = 0, n_nonempty = 0;
  SDF_CUDA(ctx, cudaMemcpyAsync(&total, tri_off + nel, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(&n_nonempty, nonempty, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  if (total < 0) return fail(ctx, SDFGPU_ERR_CAPACITY, "more than 2^31 (tile, triangle) pairs; use a coarser grid");
  ctx->h_counters[C_TILE_PAIRS] = total;
  const size_t P = (size_t)std::max<int32_t>(total, 1);
  SDF_TRY(scratch_t(ctx, "pair_keys", P, &keys));
  SDF_TRY(scratch_t(ctx, "pair_keys2", P, &keys2));
  SDF_TRY(scratch_t(ctx, "pair_vals", P, &vals));
  SDF_TRY(scratch_t(ctx, "pair_vals2", P, &vals2));
  if (total > 0) {
    k_tile_pairs<true><<<grid_for(nel, 128), 128, 0, st>>>(cent, rec, nel, g, mode, R, nullptr, tri_off, nullptr,
                                                           keys, vals, nullptr);
    SDF_KERNEL(ctx);
    const int bits = ceil_log2((uint64_t)g.ntiles + 1);
    size_t tmp_bytes = 0;
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, total, 0, bits, st));
    void* tmp;
    SDF_TRY(scratch(ctx, "cub_tmp", tmp_bytes, &tmp));
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, total, 0, bits, st));
  }
  SDF_TRY(cub_scan_i32(ctx, tile_cnt, tile_off, g.ntiles + 1));
  // Longest lists first: the CTAs of the heaviest tiles start in the first wave and the light ones
  // fill the last, which shortens the tail of the launch (any order gives the same results).
  int32_t *ord_in, *order;
  uint16_t *tkey, *tkey2;
  SDF_TRY(scratch_t(ctx, "tile_ord_in", (size_t)g.ntiles, &ord_in));
  SDF_TRY(scratch_t(ctx, "tile_order", (size_t)g.ntiles, &order));
  SDF_TRY(scratch_t(ctx, "tile_key", (size_t)g.ntiles, &tkey));
  SDF_TRY(scratch_t(ctx, "tile_key2", (size_t)g.ntiles, &tkey2));
  k_tile_keys<<<grid_for(g.ntiles, 256), 256, 0, st>>>(tile_cnt, g.ntiles, tkey, ord_in);
  SDF_KERNEL(ctx);
  {
    size_t tmp_bytes = 0;
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, tkey, tkey2, ord_in, order, g.ntiles,
                                                            0, 16, st));
    void* tmp;
    SDF_TRY(scratch(ctx, "cub_tmp_order", tmp_bytes, &tmp));
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_bytes, tkey, tkey2, ord_in, order, g.ntiles, 0,
                                                            16, st));
  }

  FoldArgs A;
  A.g = g;
  A.mode = mode;
  A.tile_off = tile_off;
  A.tile_cnt = tile_cnt;
  A.order = order;
  A.vals = vals2;
  A.rec = rec;
  A.cent = cent;
  A.v32 = v32;
  A.c32 = c32;
  A.r2 = sr * sr;
  const double e_c = 1e-6 * (g.E + sr);
  A.r2_in = (float)((sr - e_c) * (sr - e_c));
  A.r2_out = (float)((sr + e_c) * (sr + e_c));
  A.eD_abs = eD_abs;
  A.eD_rel = eD_rel;
  A.dist = d_dist;
  A.xp = d_xp;
  A.status = status;
  A.counters = ctx->d_counters;
  if (g.ntiles > 0x7fffffffLL) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "grid has too many tiles");
  std::memcpy(Pl.fold, &A, sizeof(A));
  Pl.g = g;
  Pl.ntiles = g.ntiles;
  Pl.nonempty = n_nonempty;
  Pl.threads = g.t[0] * g.t[1] * g.t[2];
  Pl.knn = false;
  if (mode == SDFGPU_MODE_REF_RULE) {
    // Can a node with an empty candidate set still have a triangle within h?  Only when some
    // triangle reaches farther than 1.5h from its centroid (|c - p| <= d + rho <= h + rho).
    const bool big_tris = M.rho_max * (1.0 + 1e-9) + 1e-6 * g.E >= 1.5 * g.h;
    if (big_tris || d_xp) {
      SDF_TRY(ensure_ine(ctx));
      uint8_t* band = nullptr;
      if (!d_xp) SDF_TRY(scratch_t(ctx, "band", (size_t)g.ngp, &band));
      KnnArgs K;
      K.g = g;
      K.status = status;
      K.band = band;
      K.nodes = buf<BNode>(ctx, "nodes");
      K.leaf_prim = buf<int32_t>(ctx, "leaf_prim");
      K.tri_idx = nullptr;
      K.IEN = buf<int64_t>(ctx, "IEN64");
      K.X = buf<double>(ctx, "X64");
      K.ine_off = buf<int32_t>(ctx, "ine_off");
      K.ine = buf<int32_t>(ctx, "ine");
      K.rec = rec;
      K.pad = pad;
      K.max_visits = 2 * nel + 64;
      K.dist = d_dist;
      K.xp = d_xp;
      K.counters = ctx->d_counters;
      std::memcpy(Pl.knn_args, &K, sizeof(K));
      Pl.knn = true;
      Pl.band = band;
      Pl.band_v32 = v32;
      Pl.band_rec = rec;
      Pl.nel = nel;
      Pl.hb = g.h * (1.0 + 1e-9) + (double)eD_abs + 2e-6 * g.E;
    }
  }
  return 0;
}

// The fold of one mesh on the context stream (one CTA per tile).
int dist_fold(sdfgpu_ctx* ctx, const DistPlan& Pl) {
  FoldArgs A;
  std::memcpy(&A, Pl.fold, sizeof(A));
  const size_t smem = sizeof(WarpStage) * (size_t)(Pl.threads / 32);
  if (smem > 48 * 1024)  // tiles of more than 5 warps stage more than the default 48 KB
    SDF_CUDA(ctx, cudaFuncSetAttribute(k_tile_fold, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // the tiles with candidates come first in the fold's order (longest list first); the rest are
  // written by one pass over the nodes
  const int64_t nfold = Pl.nonempty >= 0 ? Pl.nonempty : Pl.ntiles;
  if (nfold < Pl.ntiles) {
    k_fill_empty<<<grid_for(Pl.g.ngp, 256), 256, 0, ctx->stream>>>(Pl.g, A.tile_cnt, A.dist, A.xp, A.status);
    SDF_KERNEL(ctx);
  }
  if (nfold > 0) {
    k_tile_fold<<<(unsigned)nfold, Pl.threads, smem, ctx->stream>>>(A);
    SDF_KERNEL(ctx);
  }
  return 0;
}

// The 3-nearest-vertex fallback after the fold, on stream st: launches only (no allocation, no host
// wait), so it can be captured in a graph.  wait_bvh: order st after the LBVH build first.
int dist_knn(sdfgpu_ctx* ctx, const DistPlan& Pl, cudaStream_t st, bool wait_bvh) {
  const GridP& g = Pl.g;
  if (Pl.band) {
    SDF_CUDA(ctx, cudaMemsetAsync(Pl.band, 0, (size_t)g.ngp, st));
    k_band<<<grid_for(Pl.nel, 128), 128, 0, st>>>(Pl.band_v32, Pl.band_rec, Pl.nel, g, Pl.hb, (float)(Pl.hb * Pl.hb),
                                                   Pl.band);
    SDF_KERNEL(ctx);
  }
  if (wait_bvh) SDF_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev_bvh, 0));  // the fallback walks the LBVH
  KnnArgs K;
  std::memcpy(&K, Pl.knn_args, sizeof(K));
  k_knn_fallback<<<grid_for(g.ngp, 128, 148 * 16), 128, 0, st>>>(K);
  SDF_KERNEL(ctx);
  return 0;
}

// The folds of several meshes (plans prepared by dist_prepare on their own contexts, all with the
// same tile volume) in one persistent launch on stream st.  d_args / d_off: device copies of the
// plans' fold arguments and of the exclusive prefix of their tile counts, already uploaded.
// Resident CTAs of the multi-mesh fold (all SMs at full occupancy, at most one per work item); also
// raises the kernel's shared-memory limit when needed.  Call before a stream capture.
int dist_fold_multi_grid(sdfgpu_ctx* ctx, int threads, int64_t total, int64_t* grid) {
  const size_t smem = sizeof(WarpStage) * (size_t)(threads / 32);
  if (smem > 48 * 1024)
    SDF_CUDA(ctx, cudaFuncSetAttribute(k_tile_fold_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0, sms = 148;
  SDF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_fold_multi, threads, smem));
  SDF_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  *grid = std::max<int64_t>(1, std::min<int64_t>(total, (int64_t)sms * std::max(per_sm, 1)));
  return 0;
}

int dist_fold_multi(sdfgpu_ctx* ctx, const void* d_args, const int64_t* d_off, int count, int64_t total, int threads,
                    int64_t grid, cudaStream_t st) {
  if (count < 1 || total < 1) return 0;
  const size_t smem = sizeof(WarpStage) * (size_t)(threads / 32);
  k_tile_fold_multi<<<(unsigned)grid, threads, smem, st>>>((const FoldArgs*)d_args, d_off, count, total);
  SDF_KERNEL(ctx);
  return 0;
}

size_t fold_args_size() { return sizeof(FoldArgs); }


// Points a plan's kernels at another counter array (a batch sums its folds' counters in one place).
void plan_set_counters(DistPlan& Pl, int64_t* counters) {
  FoldArgs A;
  std::memcpy(&A, Pl.fold, sizeof(A));
  A.counters = counters;
  std::memcpy(Pl.fold, &A, sizeof(A));
  if (Pl.knn) {
    KnnArgs K;
    std::memcpy(&K, Pl.knn_args, sizeof(K));
    K.counters = counters;
    std::memcpy(Pl.knn_args, &K, sizeof(K));
  }
}

}  // namespace sdfgpu
