// sign.cu -- raycast_sign_detection (src/SignedDistances/RaycastingSignDetection.jl:337-404).
//
// Per node the reference casts the prioritized directions (:162-227) and votes by the parity of
// the distinct Möller–Trumbore hits (:114-154): 6 axis rays, then batches of 4 until the vote
// is confident (:234-288), then the generalized winding number when confidence < 0.6 (:376-380).
//
// B200 layout of the work:
//   * The 6 axis rays are the only rays every node casts, and they are grid-structured.  For a
//     ray along +x from node (i, j, k) every Möller–Trumbore decision except t > eps depends only
//     on the row (j, k): h = cross(e_x, e2) has an exactly zero x component, so u and v never see
//     the node's x.  And the -x ray of the same node sees a = -a, f = -f, the same u and v, and
//     t = -t exactly.  So one list of (row, triangle) hits per axis serves both directions of
//     every node of the row.  The lists are built by a triangle scatter over the rows its
//     projected box covers (FP64 decisions, exactly the reference's); each node then evaluates
//     only t for the hits of its three rows with the reference's formula, sorts, de-duplicates
//     within eps and takes parities.  A warp walks 32 consecutive nodes of one row, so the row's
//     hits are broadcast loads.
//   * Nodes whose 6 votes disagree continue with the reference's batches on the LBVH: FP32 slab
//     tests with an explicit margin prune, FP64 Möller–Trumbore decides.
//   * Nodes left with confidence < threshold sum the winding number over all triangles, one CTA
//     per node with a fixed-order block reduction.
#include <cub/cub.cuh>

#include <cstring>

#include "common.cuh"

namespace sdfgpu {

__constant__ double c_dirs[36 * 3];

namespace {

constexpr double kEps = 1e-8;  // check_ray_inside_bvh default (:118), passed to MT (:132)
constexpr int kRowCap = 64;    // hits per row a node sorts in registers/local memory
constexpr int kRayCap = 256;   // hits per generic ray
constexpr int kStack = 64;

// A row hit: the Möller–Trumbore constants of one triangle for one grid row, from which each node
// of the row gets t with the reference's operation order (see the per-axis formulas below).
struct __align__(16) RowHit {
  double v1a;  // v1 coordinate along the row axis
  double K1, K2, P;
  double ea, eb, fa, fb;
  double f;
  double key;  // approximate hit coordinate along the axis (row ordering only)
};

template <int AX>
__device__ __forceinline__ double row_t(const RowHit& r, double xa) {
  const double s = ds(xa, r.v1a);
  if (AX == 0) {
    const double qy = ds(r.K1, dm(s, r.ea));
    const double qz = ds(dm(s, r.eb), r.K2);
    return dm(r.f, da(da(r.P, dm(r.fa, qy)), dm(r.fb, qz)));
  } else if (AX == 1) {
    const double qx = ds(dm(s, r.ea), r.K1);
    const double qz = ds(r.K2, dm(s, r.eb));
    return dm(r.f, da(da(dm(r.fa, qx), r.P), dm(r.fb, qz)));
  } else {
    const double qx = ds(r.K1, dm(s, r.ea));
    const double qy = ds(dm(s, r.eb), r.K2);
    return dm(r.f, da(da(dm(r.fa, qx), dm(r.fb, qy)), r.P));
  }
}

// Möller–Trumbore decisions of the +AX ray through (ob, oc) against the triangle; on a pass fills
// the row-hit constants.  The along-axis origin is v1's own coordinate (any value gives the same
// decisions, see the file comment).
template <int AX>
__device__ __forceinline__ bool row_test(const TriRec64& r, double ob, double oc, RowHit* out) {
  const d3 v1 = rec_v(r, 0), v2 = rec_v(r, 1), v3 = rec_v(r, 2);
  d3 o, d;
  if (AX == 0) { o = {v1.x, ob, oc}; d = {1.0, 0.0, 0.0}; }
  else if (AX == 1) { o = {ob, v1.y, oc}; d = {0.0, 1.0, 0.0}; }
  else { o = {ob, oc, v1.z}; d = {0.0, 0.0, 1.0}; }
  const d3 e1 = v_sub(v2, v1), e2 = v_sub(v3, v1);
  const d3 h = v_cross(d, e2);
  const double a = v_dot(e1, h);
  if (fabs(a) < kEps) return false;
  const double f = dd(1.0, a);
  const d3 s = v_sub(o, v1);
  const double u = dm(f, v_dot(s, h));
  if (u < 0.0 || u > 1.0) return false;
  const d3 q = v_cross(s, e1);
  const double v = dm(f, v_dot(d, q));
  if (v < 0.0 || da(u, v) > 1.0) return false;
  if (out) {
    RowHit R;
    R.f = f;
    if (AX == 0) {
      R.v1a = v1.x; R.K1 = dm(s.z, e1.x); R.K2 = dm(s.y, e1.x); R.P = dm(e2.x, q.x);
      R.ea = e1.z; R.eb = e1.y; R.fa = e2.y; R.fb = e2.z;
    } else if (AX == 1) {
      R.v1a = v1.y; R.K1 = dm(s.z, e1.y); R.K2 = dm(s.x, e1.y); R.P = dm(e2.y, q.y);
      R.ea = e1.z; R.eb = e1.x; R.fa = e2.x; R.fb = e2.z;
    } else {
      R.v1a = v1.z; R.K1 = dm(s.y, e1.z); R.K2 = dm(s.x, e1.z); R.P = dm(e2.z, q.z);
      R.ea = e1.y; R.eb = e1.x; R.fa = e2.x; R.fb = e2.y;
    }
    R.key = R.v1a + row_t<AX>(R, R.v1a);
    *out = R;
  }
  return true;
}

// The decisions of row_test in FP32 with explicit error bands (the bulk of the sign stage's
// arithmetic).  Returns 0 when the FP64 test certainly misses, 1 when it certainly hits, 2 when a
// decision lies inside its band (the caller replays row_test in FP64).
//
// With (P, Q) the transverse axes in cyclic order after AX, the +AX ray gives h = d x e2 with
// h_P = -e2_Q, h_Q = e2_P, h_AX = 0, so a = e1_Q e2_P - e1_P e2_Q, s.h = s_Q e2_P - s_P e2_Q and
// d.q = s_P e1_Q - s_Q e1_P (s_AX = 0).  The six inputs are the FP64 differences the reference
// forms, rounded once to FP32 (relative error u = 2^-24 each).  A difference of two products of
// rounded inputs is then within 4u (|p1| + |p2|) of the FP64 value (whose own error, ~2^-51 of the
// same sum, is far below); 6u is used.  With err_a, err_p those bounds, |A| >= 3 err_a (else the
// test is undecided) and den = |A| - err_a, the quotient U = fl(P_u / A) satisfies
//   |u - U| <= E_u = (1.5 err_p + 2 (|U| + 1) err_a) / den + 2u (|U| + 1)
// (|u| <= 2 (|U| + 1) follows from err_a <= den / 2), the same for v, and
// |(u + v) - fl(U + V)| <= E_u + E_v + 2u |U + V|.
constexpr float kU32 = 5.9604645e-8f;  // 2^-24

template <int AX>
__device__ __forceinline__ int row_test32(const TriRec64& r, double ob, double oc) {
  constexpr int P = AX == 0 ? 1 : (AX == 1 ? 2 : 0), Q = AX == 0 ? 2 : (AX == 1 ? 0 : 1);
  // row origin along P and Q (row_test's o: AX = 0 -> (y, z) = (ob, oc); AX = 1 -> (z, x) = (oc, ob);
  // AX = 2 -> (x, y) = (ob, oc))
  const double oP = AX == 1 ? oc : ob, oQ = AX == 1 ? ob : oc;
  const float e1P = (float)ds(r.v[3 + P], r.v[P]), e1Q = (float)ds(r.v[3 + Q], r.v[Q]);
  const float e2P = (float)ds(r.v[6 + P], r.v[P]), e2Q = (float)ds(r.v[6 + Q], r.v[Q]);
  const float sP = (float)ds(oP, r.v[P]), sQ = (float)ds(oQ, r.v[Q]);
  const float a1 = __fmul_rn(e1Q, e2P), a2 = __fmul_rn(e1P, e2Q);
  const float A = __fsub_rn(a1, a2);
  const float ea = 6.f * kU32 * (fabsf(a1) + fabsf(a2));
  const float aA = fabsf(A);
  if (aA + ea < (float)kEps) return 0;                          // |a| < eps certainly
  if (!(aA - ea >= (float)kEps) || !(aA >= 3.f * ea)) return 2;  // |a| near eps, or a ill-conditioned
  const float den = aA - ea;
  const float u1 = __fmul_rn(sQ, e2P), u2 = __fmul_rn(sP, e2Q);
  const float U = __fdiv_rn(__fsub_rn(u1, u2), A);
  const float Eu = (1.5f * 6.f * kU32 * (fabsf(u1) + fabsf(u2)) + 2.f * (fabsf(U) + 1.f) * ea) / den +
                   2.f * kU32 * (fabsf(U) + 1.f);
  if (U < -Eu || U > 1.f + Eu) return 0;
  const float v1 = __fmul_rn(sP, e1Q), v2 = __fmul_rn(sQ, e1P);
  const float V = __fdiv_rn(__fsub_rn(v1, v2), A);
  const float Ev = (1.5f * 6.f * kU32 * (fabsf(v1) + fabsf(v2)) + 2.f * (fabsf(V) + 1.f) * ea) / den +
                   2.f * kU32 * (fabsf(V) + 1.f);
  if (V < -Ev) return 0;
  const float UV = __fadd_rn(U, V);
  const float Euv = Eu + Ev + 2.f * kU32 * fabsf(UV);
  if (UV > 1.f + Euv) return 0;
  if (U >= Eu && U <= 1.f - Eu && V >= Ev && UV <= 1.f - Euv) return 1;
  return 2;
}

__device__ __forceinline__ bool axis_range2(const GridP& g, int a, double x0, double x1, int64_t& lo, int64_t& hi) {
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

template <int AX>
__device__ __forceinline__ void tri_rows(const GridP& g, const TriRec64& r, bool fill, int64_t row_base,
                                         int32_t* row_cnt, const int32_t* row_off, int32_t* row_cur, RowHit* hits,
                                         unsigned long long* rkey, int32_t* ridx, int64_t& nhit, int64_t& nband) {
  const int b = AX == 0 ? 1 : 0, c = AX == 2 ? 1 : 2;
  int64_t b0, b1, c0, c1;
  if (!axis_range2(g, b, r.bmin[b], r.bmax[b], b0, b1)) return;
  if (!axis_range2(g, c, r.bmin[c], r.bmax[c], c0, c1)) return;
  for (int64_t jc = c0; jc <= c1; ++jc) {
    const double oc = da(g.o[c], dm(g.h, (double)gidx(g, c, jc)));
    for (int64_t jb = b0; jb <= b1; ++jb) {
      const double ob = da(g.o[b], dm(g.h, (double)gidx(g, b, jb)));
      const int64_t row = row_base + jc * g.n[b] + jb;
      const int dec = row_test32<AX>(r, ob, oc);
      if (dec == 0) continue;
      if (!fill) {
        if (dec == 2) ++nband;  // inside the FP32 band: the FP64 test decides
        if (dec == 1 || row_test<AX>(r, ob, oc, nullptr)) { atomicAdd(&row_cnt[row], 1); ++nhit; }
      } else {
        RowHit R;
        if (row_test<AX>(r, ob, oc, &R)) {  // the hit's FP64 constants (and the band's decision)
          const int32_t pos = row_off[row] + atomicAdd(&row_cur[row], 1);
          hits[pos] = R;
          // sort key: row in the high word, the hit coordinate (ordered float bits) in the low word
          uint32_t u = __float_as_uint((float)R.key);
          u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
          rkey[pos] = ((unsigned long long)row << 32) | u;
          ridx[pos] = pos;
        }
      }
    }
  }
}

__global__ void k_rows(const TriRec64* __restrict__ rec, int64_t nel, GridP g, int64_t base_y, int64_t base_z,
                       bool fill, int32_t* row_cnt, const int32_t* row_off, int32_t* row_cur, RowHit* hits,
                       unsigned long long* rkey, int32_t* ridx, int64_t* counters) {
  int64_t nhit = 0, nband = 0;
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    const TriRec64 r = rec[el];
    tri_rows<0>(g, r, fill, 0, row_cnt, row_off, row_cur, hits, rkey, ridx, nhit, nband);
    tri_rows<1>(g, r, fill, base_y, row_cnt, row_off, row_cur, hits, rkey, ridx, nhit, nband);
    tri_rows<2>(g, r, fill, base_z, row_cnt, row_off, row_cur, hits, rkey, ridx, nhit, nband);
  }
  if (!fill) {
    for (int off = 16; off > 0; off >>= 1) {
      nhit += __shfl_down_sync(0xffffffffu, nhit, off);
      nband += __shfl_down_sync(0xffffffffu, nband, off);
    }
    if ((threadIdx.x & 31) == 0 && nhit) count_add(counters, C_ROW_HITS, nhit);
    if ((threadIdx.x & 31) == 0 && nband) count_add(counters, C_SIGN_BAND, nband);
  }
}

// Gathers the row hits into (row, hit coordinate) order after the radix sort of their keys.
__global__ void k_gather_rows(int64_t n, const int32_t* __restrict__ order, const RowHit* __restrict__ src,
                              RowHit* __restrict__ dst) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    dst[q] = src[order[q]];
}

// Number of distinct hits (gaps > eps) among sorted t values passing the direction's t > eps.
__device__ __forceinline__ int clusters_pos(const double* ts, int n) {
  int c = 0;
  double prev = 0.0;
  for (int a = 0; a < n; ++a) {
    if (!(ts[a] > kEps)) continue;
    if (c == 0 || fabs(ds(ts[a], prev)) > kEps) ++c;
    prev = ts[a];
  }
  return c;
}
__device__ __forceinline__ int clusters_neg(const double* ts, int n) {
  // the -axis ray sees t' = -t; ascending t' is descending t
  int c = 0;
  double prev = 0.0;
  for (int a = n - 1; a >= 0; --a) {
    const double tn = -ts[a];
    if (!(tn > kEps)) continue;
    if (c == 0 || fabs(ds(tn, prev)) > kEps) ++c;
    prev = tn;
  }
  return c;
}

// Parities of the +AX / -AX rays of every node.  Thread order runs along the AX rows.
// par bit0: +AX inside, bit1: -AX inside, bit7: row overflow (node takes the generic path).
template <int AX>
__global__ void __launch_bounds__(256) k_axis_parity(GridP g, int64_t row_base, const int32_t* __restrict__ row_off,
                                                     const int32_t* __restrict__ row_cnt,
                                                     const RowHit* __restrict__ hits, uint8_t* __restrict__ par) {
  const int b = AX == 0 ? 1 : 0, c = AX == 2 ? 1 : 2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < g.ngp; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ia = t % g.n[AX];
    const int64_t rest = t / g.n[AX];
    const int64_t jb = rest % g.n[b], jc = rest / g.n[b];
    int64_t idx[3];
    idx[AX] = ia; idx[b] = jb; idx[c] = jc;
    const int64_t lin = idx[0] + g.n[0] * (idx[1] + g.n[1] * idx[2]);
    const int64_t row = row_base + jc * g.n[b] + jb;
    const int32_t off = row_off[row], n = row_cnt[row];
    if (n > kRowCap) { par[lin] = 0x80; continue; }
    const double xa = da(g.o[AX], dm(g.h, (double)gidx(g, AX, ia)));
    double ts[kRowCap];
    for (int q = 0; q < n; ++q) {
      const double tv = row_t<AX>(hits[off + q], xa);
      int p = q - 1;
      while (p >= 0 && ts[p] > tv) { ts[p + 1] = ts[p]; --p; }
      ts[p + 1] = tv;
    }
    const int cp = clusters_pos(ts, n), cn = clusters_neg(ts, n);
    par[lin] = (uint8_t)((cp & 1) | ((cn & 1) << 1));
  }
}

// adaptive_point_in_mesh_raycast (:234-288).  cast(i) returns the parity of ray i (1-based) or
// -1 when that ray is not available to the caller.
template <class Cast>
__device__ __forceinline__ int vote_logic(int min_rays, int max_rays, Cast cast, double& sign, double& conf,
                                          int& total_out) {
  int inside = 0, total = 0;
  for (int i = 1; i <= min_rays; ++i) {
    const int r = cast(i);
    if (r < 0) return 1;
    inside += r;
    ++total;
  }
  double ratio = dd((double)inside, (double)total);
  double cf = fmax(ratio, ds(1.0, ratio));
  int used = min_rays;
  while (cf < 0.85 && used < max_rays) {
    const int batch = min(4, max_rays - used);
    for (int i = used + 1; i <= used + batch; ++i) {
      if (i <= 36) {
        const int r = cast(i);
        if (r < 0) return 1;
        inside += r;
        ++total;
      }
    }
    used += batch;
    ratio = dd((double)inside, (double)total);
    cf = fmax(ratio, ds(1.0, ratio));
    if (cf > 0.95) break;
  }
  sign = ratio > 0.5 ? 1.0 : -1.0;
  conf = cf;
  total_out = total;
  return 0;
}

__device__ __forceinline__ int axis_bit(uint8_t px, uint8_t py, uint8_t pz, int i) {
  // rays 1..6: +X +Y +Z -X -Y -Z
  switch (i) {
    case 1: return px & 1;
    case 2: return py & 1;
    case 3: return pz & 1;
    case 4: return (px >> 1) & 1;
    case 5: return (py >> 1) & 1;
    default: return (pz >> 1) & 1;
  }
}

struct VoteArgs {
  GridP g;
  const uint8_t* par[3];
  int min_rays, max_rays;
  double conf_thresh;
  int use_winding;
  double* sign;
  double* conf;
  int32_t* und_list;
  uint64_t* und_have;
  uint64_t* und_par;
  int32_t* wind_list;
  int64_t* counters;
};

__global__ void k_vote(VoteArgs A) {
  const GridP& g = A.g;
  for (int64_t lin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lin < g.ngp; lin += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t px = A.par[0][lin], py = A.par[1][lin], pz = A.par[2][lin];
    const bool ovf = ((px | py | pz) & 0x80) != 0;
    double s, cf;
    int total;
    const int rc = vote_logic(A.min_rays, A.max_rays,
                              [&](int i) { return (i <= 6 && !ovf) ? axis_bit(px, py, pz, i) : -1; }, s, cf, total);
    if (rc) {
      const int64_t slot = atomicAdd((unsigned long long*)&A.counters[C_LIST_UNDECIDED], 1ULL);
      A.und_list[slot] = (int32_t)lin;
      uint64_t have = 0, par = 0;
      if (!ovf) {
        have = 0x3FULL;
        for (int r = 1; r <= 6; ++r) par |= (uint64_t)axis_bit(px, py, pz, r) << (r - 1);
      }
      A.und_have[slot] = have;
      A.und_par[slot] = par;
      continue;
    }
    if (A.use_winding && cf < A.conf_thresh) {
      const int64_t slot = atomicAdd((unsigned long long*)&A.counters[C_LIST_WINDING], 1ULL);
      A.wind_list[slot] = (int32_t)lin;
      cf = 0.8;
    }
    A.sign[lin] = s;
    if (A.conf) A.conf[lin] = cf;
  }
}

struct RayArgs {
  GridP g;
  const BNode* nodes;
  const int32_t* leaf_prim;
  const TriRec64* rec;
  float pad;
  int64_t max_visits;
  const uint8_t* par[3];
  const int32_t* list;
  int min_rays, max_rays;
  double conf_thresh;
  int use_winding;
  double* sign;
  double* conf;
  int32_t* wind_list;
  int64_t* counters;
  uint64_t* have;     // per undecided node: rays whose parity is known
  uint64_t* parbits;  // per undecided node: their parities
  uint8_t* done;
  int32_t* req_node;  // requests of the current round
  int8_t* req_ray;
  int64_t* rq_cnt;    // requests per round
  int speculative;    // request all remaining rays at once (latency-bound when few nodes remain)
  int last_ray;       // last ray index the vote can cast: min(36, max(min_rays, max_rays))
};

__device__ __forceinline__ void child_box2(const BNode& nd, int side, float3& lo, float3& hi) {
  if (side == 0) {
    lo = make_float3(nd.a.x, nd.a.y, nd.a.z);
    hi = make_float3(nd.a.w, nd.b.x, nd.b.y);
  } else {
    lo = make_float3(nd.b.z, nd.b.w, nd.c.x);
    hi = make_float3(nd.c.y, nd.c.z, nd.c.w);
  }
}

// ray_triangle_intersection (:64-106) for a ray of any direction decided in FP32 with explicit
// error bands: 0 = the FP64 test certainly misses, 1 = it certainly hits, 2 = a decision lies in
// its band.  Inputs are the FP64 differences the reference forms (e1, e2, s = o - v1) and the
// direction, each rounded once to FP32.  Each component of h = d x e2 and q = s x e1 is within
// 4u of its FP64 value times its absolute-value sum (u = 2^-24), and each three-term dot product
// over them within 12u times the dot product of the absolute-value sums; the quotients u, v, t
// then carry the bound of row_test32's comment.  The caller replays mt64 for every hit, certain or
// not: the hit's t in FP64 is what the reference sorts and de-duplicates within eps.
__device__ __forceinline__ int mt32(const d3& o, const d3& d, const d3& v1, const d3& v2, const d3& v3) {
  const float3 e1 = make_float3((float)ds(v2.x, v1.x), (float)ds(v2.y, v1.y), (float)ds(v2.z, v1.z));
  const float3 e2 = make_float3((float)ds(v3.x, v1.x), (float)ds(v3.y, v1.y), (float)ds(v3.z, v1.z));
  const float3 sv = make_float3((float)ds(o.x, v1.x), (float)ds(o.y, v1.y), (float)ds(o.z, v1.z));
  const float3 dv = make_float3((float)d.x, (float)d.y, (float)d.z);
  // h = d x e2 and the absolute-value sums of its terms
  const float3 h = make_float3(__fsub_rn(__fmul_rn(dv.y, e2.z), __fmul_rn(dv.z, e2.y)),
                               __fsub_rn(__fmul_rn(dv.z, e2.x), __fmul_rn(dv.x, e2.z)),
                               __fsub_rn(__fmul_rn(dv.x, e2.y), __fmul_rn(dv.y, e2.x)));
  const float3 th = make_float3(fabsf(dv.y * e2.z) + fabsf(dv.z * e2.y), fabsf(dv.z * e2.x) + fabsf(dv.x * e2.z),
                                fabsf(dv.x * e2.y) + fabsf(dv.y * e2.x));
  auto dot = [](float3 a, float3 b) { return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z)); };
  auto adot = [](float3 a, float3 t) { return fabsf(a.x) * t.x + fabsf(a.y) * t.y + fabsf(a.z) * t.z; };
  const float A = dot(e1, h);
  const float ea = 12.f * kU32 * adot(e1, th);
  const float aA = fabsf(A);
  if (aA + ea < (float)kEps) return 0;
  if (!(aA - ea >= (float)kEps) || !(aA >= 3.f * ea)) return 2;
  const float den = aA - ea;
  auto band = [&](float X, float e) { return (1.5f * e + 2.f * (fabsf(X) + 1.f) * ea) / den + 2.f * kU32 * (fabsf(X) + 1.f); };
  const float U = __fdiv_rn(dot(sv, h), A);
  const float Eu = band(U, 12.f * kU32 * adot(sv, th));
  if (U < -Eu || U > 1.f + Eu) return 0;
  const float3 q = make_float3(__fsub_rn(__fmul_rn(sv.y, e1.z), __fmul_rn(sv.z, e1.y)),
                               __fsub_rn(__fmul_rn(sv.z, e1.x), __fmul_rn(sv.x, e1.z)),
                               __fsub_rn(__fmul_rn(sv.x, e1.y), __fmul_rn(sv.y, e1.x)));
  const float3 tq = make_float3(fabsf(sv.y * e1.z) + fabsf(sv.z * e1.y), fabsf(sv.z * e1.x) + fabsf(sv.x * e1.z),
                                fabsf(sv.x * e1.y) + fabsf(sv.y * e1.x));
  const float V = __fdiv_rn(dot(dv, q), A);
  const float Ev = band(V, 12.f * kU32 * adot(dv, tq));
  if (V < -Ev) return 0;
  const float UV = __fadd_rn(U, V);
  const float Euv = Eu + Ev + 2.f * kU32 * fabsf(UV);
  if (UV > 1.f + Euv) return 0;
  const float T = __fdiv_rn(dot(e2, q), A);
  const float Et = band(T, 12.f * kU32 * adot(e2, tq));
  if (T + Et <= (float)kEps) return 0;
  if (U >= Eu && U <= 1.f - Eu && V >= Ev && UV <= 1.f - Euv && T - Et > (float)kEps) return 1;
  return 2;
}

// check_ray_inside_bvh (:114-154) on the LBVH.  Returns parity, or -1 on buffer/stack overflow.
// *band counts the ray-triangle tests whose FP32 decision fell in its band.
__device__ int ray_parity(const RayArgs& A, const d3& p, const float3& p32, int dir, int64_t* band) {
  const d3 d = {c_dirs[3 * dir], c_dirs[3 * dir + 1], c_dirs[3 * dir + 2]};
  const float3 d32 = make_float3((float)d.x, (float)d.y, (float)d.z);
  const float3 inv = make_float3(1.0f / d32.x, 1.0f / d32.y, 1.0f / d32.z);
  double ts[kRayCap];
  int n = 0;
  int stack[kStack];
  int sp = 0;
  stack[sp++] = 0;
  int64_t visits = 0;
  while (sp > 0) {
    if (++visits > A.max_visits) return -1;
    const BNode nd = A.nodes[stack[--sp]];
    const int ch[2] = {nd.d.x, nd.d.y};
    for (int side = 0; side < 2; ++side) {
      float3 lo, hi;
      child_box2(nd, side, lo, hi);
      if (lo.x > hi.x) continue;
      if (!ray_box(p32, d32, inv, lo, hi, A.pad, A.pad)) continue;
      if (ch[side] & kLeafBit) {
        const TriRec64& r = A.rec[A.leaf_prim[ch[side] & 0x7fffffff]];
        const int dec = mt32(p, d, rec_v(r, 0), rec_v(r, 1), rec_v(r, 2));
        if (dec == 0) continue;
        if (dec == 2) ++*band;
        double t;
        if (mt64(p, d, rec_v(r, 0), rec_v(r, 1), rec_v(r, 2), kEps, t)) {
          if (n >= kRayCap) return -1;
          int q = n - 1;
          while (q >= 0 && ts[q] > t) { ts[q + 1] = ts[q]; --q; }
          ts[q + 1] = t;
          ++n;
        }
      } else {
        if (sp >= kStack) return -1;
        stack[sp++] = ch[side];
      }
    }
  }
  if (n == 0) return 0;
  int unique = 1;
  for (int a = 1; a < n; ++a)
    if (fabs(ds(ts[a], ts[a - 1])) > kEps) ++unique;
  return unique & 1;
}

// The reference's vote (:234-288) replayed over the rays whose parity is already known (bit i-1
// of `have` / `par` for ray i).  Returns 0 with sign/conf when the vote is decided; otherwise 1
// with [need_lo, need_hi] = the rays of the first incomplete step (the initial min_rays, or the
// current batch of 4), which the caller requests all at once.
__device__ __forceinline__ int vote_known(uint64_t have, uint64_t par, int min_rays, int max_rays, double& sign,
                                          double& conf, int& need_lo, int& need_hi) {
  int inside = 0, total = 0;
  for (int i = 1; i <= min_rays; ++i) {
    if (!((have >> (i - 1)) & 1)) { need_lo = i; need_hi = min_rays; return 1; }
    inside += (int)((par >> (i - 1)) & 1);
    ++total;
  }
  double ratio = dd((double)inside, (double)total);
  double cf = fmax(ratio, ds(1.0, ratio));
  int used = min_rays;
  while (cf < 0.85 && used < max_rays) {
    const int batch = min(4, max_rays - used);
    for (int i = used + 1; i <= used + batch; ++i) {
      if (i <= 36) {
        if (!((have >> (i - 1)) & 1)) { need_lo = i; need_hi = min(used + batch, 36); return 1; }
        inside += (int)((par >> (i - 1)) & 1);
        ++total;
      }
    }
    used += batch;
    ratio = dd((double)inside, (double)total);
    cf = fmax(ratio, ds(1.0, ratio));
    if (cf > 0.95) break;
  }
  sign = ratio > 0.5 ? 1.0 : -1.0;
  conf = cf;
  return 0;
}

// One round of the adaptive vote over the undecided nodes: decide, or request the next rays.
__global__ void k_round(RayArgs A, int64_t nund, int round, int last) {
  const GridP& g = A.g;
  int64_t* rq_cnt = A.rq_cnt + round;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nund; q += (int64_t)gridDim.x * blockDim.x) {
    if (A.done[q]) continue;
    double s, cf;
    int lo, hi;
    const uint64_t have = A.have[q], par = A.parbits[q];
    if (vote_known(have, par, A.min_rays, A.max_rays, s, cf, lo, hi)) {
      if (last) {  // unreachable: the rounds cover every batch up to the 36th direction
        count_add(A.counters, C_ERR_CAPACITY, 1);
        continue;
      }
      if (A.speculative) hi = A.last_ray;  // few nodes: cast every ray the vote could still need
      for (int i = lo; i <= hi; ++i) {
        if ((have >> (i - 1)) & 1) continue;
        const int64_t slot = atomicAdd((unsigned long long*)rq_cnt, 1ULL);
        A.req_node[slot] = (int32_t)q;
        A.req_ray[slot] = (int8_t)i;
      }
      continue;
    }
    const int64_t lin = A.list[q];
    if (A.use_winding && cf < A.conf_thresh) {
      const int64_t slot = atomicAdd((unsigned long long*)&A.counters[C_LIST_WINDING], 1ULL);
      A.wind_list[slot] = (int32_t)lin;
      cf = 0.8;
    }
    A.sign[lin] = s;
    if (A.conf) A.conf[lin] = cf;
    A.done[q] = 1;
    (void)g;
  }
}

// Casts the requested rays of a round, one thread per (node, ray).
__global__ void __launch_bounds__(128) k_rays(RayArgs A, int round) {
  const GridP& g = A.g;
  const int64_t count = A.rq_cnt[round];
  int64_t rays = 0, band = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = A.req_node[t];
    const int r = A.req_ray[t];
    const int64_t lin = A.list[q];
    const int64_t i = lin % g.n[0], j = (lin / g.n[0]) % g.n[1], k = lin / (g.n[0] * g.n[1]);
    const d3 p = gnode(g, i, j, k);
    const float3 p32 = make_float3((float)(p.x - g.center[0]), (float)(p.y - g.center[1]), (float)(p.z - g.center[2]));
    int v = ray_parity(A, p, p32, r - 1, &band);
    if (v < 0) { count_add(A.counters, C_ERR_CAPACITY, 1); v = 0; }
    const uint64_t bit = 1ULL << (r - 1);
    if (v) atomicOr((unsigned long long*)&A.parbits[q], (unsigned long long)bit);
    atomicOr((unsigned long long*)&A.have[q], (unsigned long long)bit);
    ++rays;
  }
  for (int off = 16; off > 0; off >>= 1) {
    rays += __shfl_down_sync(0xffffffffu, rays, off);
    band += __shfl_down_sync(0xffffffffu, band, off);
  }
  if ((threadIdx.x & 31) == 0 && rays) count_add(A.counters, C_EXTRA_RAYS, rays);
  if ((threadIdx.x & 31) == 0 && band) count_add(A.counters, C_SIGN_BAND, band);
}

// generalized_winding_number (:295-328).  The triangles are cut into fixed chunks; one CTA sums
// one chunk for one node (fixed-order block reduction) and k_winding_final adds the chunk sums
// in chunk order, so the result does not depend on scheduling and one node still fills the GPU.
constexpr int kWindChunk = 8192;

__global__ void __launch_bounds__(256) k_winding(GridP g, const TriRec64* __restrict__ rec, int64_t nel,
                                                 const int32_t* __restrict__ list, int64_t count, int nchunks,
                                                 double* __restrict__ partial) {
  __shared__ double red[256];
  const int chunk = blockIdx.x;
  for (int64_t q = blockIdx.y; q < count; q += gridDim.y) {
    const int64_t lin = list[q];
    const int64_t i = lin % g.n[0], j = (lin / g.n[0]) % g.n[1], k = lin / (g.n[0] * g.n[1]);
    const d3 p = gnode(g, i, j, k);
    double w = 0.0;
    const int64_t e1 = min((int64_t)(chunk + 1) * kWindChunk, nel);
    for (int64_t el = (int64_t)chunk * kWindChunk + threadIdx.x; el < e1; el += blockDim.x) {
      const TriRec64& r = rec[el];
      const d3 a = v_normalize(v_sub(rec_v(r, 0), p));
      const d3 b = v_normalize(v_sub(rec_v(r, 1), p));
      const d3 c = v_normalize(v_sub(rec_v(r, 2), p));
      const double num = v_dot(a, v_cross(b, c));
      const double den = da(da(da(1.0, v_dot(a, b)), v_dot(b, c)), v_dot(c, a));
      if (fabs(den) > 1e-10) {
        double sa = dm(2.0, atan2(fabs(num), den));
        if (num < 0) sa = -sa;
        w = da(w, sa);
      }
    }
    red[threadIdx.x] = w;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
      if ((int)threadIdx.x < s2) red[threadIdx.x] = da(red[threadIdx.x], red[threadIdx.x + s2]);
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[q * nchunks + chunk] = red[0];
    __syncthreads();
  }
}

__global__ void k_winding_final(const int32_t* __restrict__ list, int64_t count, int nchunks,
                                const double* __restrict__ partial, double* sign, int64_t* counters) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x) {
    double w = 0.0;
    for (int c = 0; c < nchunks; ++c) w = da(w, partial[q * nchunks + c]);
    const double wn = dd(w, 12.566370614359172);  // 4π
    sign[list[q]] = fabs(wn) > 0.5 ? 1.0 : -1.0;
    count_add(counters, C_WINDING, 1);
    if (fabs(fabs(wn) - 0.5) < 1e-9) count_add(counters, C_WIND_AMBIG, 1);
  }
}

__global__ void k_combine(int64_t n, const double* __restrict__ dist, const double* __restrict__ sign,
                          double* __restrict__ sdf) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    sdf[q] = dm(dist[q], sign[q]);
}

}  // namespace

int upload_directions(sdfgpu_ctx* ctx, const double* dirs) {
  SDF_CUDA(ctx, cudaMemcpyToSymbolAsync(c_dirs, dirs, sizeof(double) * 108, 0, cudaMemcpyHostToDevice, ctx->stream));
  return 0;
}

int sign_begin(sdfgpu_ctx* ctx, const GridP& g, SignPlan& P) {
  cudaStream_t st = ctx->sign_stream;
  const int64_t nel = ctx->mesh.nel;
  const TriRec64* rec = buf<TriRec64>(ctx, "rec");
  P.Rx = g.n[1] * g.n[2];
  P.Ry = g.n[0] * g.n[2];
  P.Rz = g.n[0] * g.n[1];
  P.nrows = P.Rx + P.Ry + P.Rz;
  if (P.nrows >= 0x7fffffffLL) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "grid has too many rows");
  SDF_TRY(scratch_t(ctx, "row_cnt", (size_t)P.nrows + 1, &P.row_cnt));
  SDF_TRY(scratch_t(ctx, "row_off", (size_t)P.nrows + 1, &P.row_off));
  SDF_TRY(scratch_t(ctx, "row_cur", (size_t)P.nrows + 1, &P.row_cur));
  SDF_CUDA(ctx, cudaMemsetAsync(P.row_cnt, 0, sizeof(int32_t) * (P.nrows + 1), st));
  SDF_CUDA(ctx, cudaMemsetAsync(P.row_cur, 0, sizeof(int32_t) * (P.nrows + 1), st));
  k_rows<<<grid_for(nel, 128), 128, 0, st>>>(rec, nel, g, P.Rx, P.Rx + P.Ry, false, P.row_cnt, nullptr, nullptr,
                                             nullptr, nullptr, nullptr, ctx->d_counters);
  SDF_KERNEL(ctx);
  SDF_TRY(cub_scan_i32(ctx, P.row_cnt, P.row_off, P.nrows + 1, st, "cub_tmp_scan_sign"));
  ctx->h_scalars[S_ROW_TOTAL] = -1;
  SDF_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars + S_ROW_TOTAL, P.row_off + P.nrows, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaEventRecord(ctx->ev_rows, st));
  return 0;
}

int sign_finish(sdfgpu_ctx* ctx, const GridP& g, SignPlan& P, int min_rays, int max_rays, double conf_thresh,
                int use_winding, double* d_sign, double* d_conf) {
  cudaStream_t st = ctx->sign_stream;
  const MeshDev& M = ctx->mesh;
  const int64_t nel = M.nel;
  const TriRec64* rec = buf<TriRec64>(ctx, "rec");
  const int64_t Rx = P.Rx, Ry = P.Ry, nrows = P.nrows;
  int32_t *row_cnt = P.row_cnt, *row_off = P.row_off, *row_cur = P.row_cur;
  SDF_CUDA(ctx, cudaEventSynchronize(ctx->ev_rows));
  int32_t total;
  std::memcpy(&total, ctx->h_scalars + S_ROW_TOTAL, sizeof(int32_t));  // the low 4 bytes hold the int32
  if (total < 0) return fail(ctx, SDFGPU_ERR_CAPACITY, "more than 2^31 row hits");
  RowHit *hits_raw, *hits;
  unsigned long long *rkey, *rkey2;
  int32_t *ridx, *ridx2;
  const size_t H = (size_t)std::max(total, 1);
  SDF_TRY(scratch_t(ctx, "row_hits_raw", H, &hits_raw));
  SDF_TRY(scratch_t(ctx, "row_hits", H, &hits));
  SDF_TRY(scratch_t(ctx, "row_key", H, &rkey));
  SDF_TRY(scratch_t(ctx, "row_key2", H, &rkey2));
  SDF_TRY(scratch_t(ctx, "row_idx", H, &ridx));
  SDF_TRY(scratch_t(ctx, "row_idx2", H, &ridx2));
  if (total > 0) {
    k_rows<<<grid_for(nel, 128), 128, 0, st>>>(rec, nel, g, Rx, Rx + Ry, true, nullptr, row_off, row_cur, hits_raw,
                                               rkey, ridx, ctx->d_counters);
    SDF_KERNEL(ctx);
    int bits = 32;
    while (bits < 64 && (1LL << (bits - 32)) < nrows) ++bits;
    size_t tmp_bytes = 0;
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, rkey, rkey2, ridx, ridx2, total, 0, bits, st));
    void* tmp;
    SDF_TRY(scratch(ctx, "cub_tmp_sign", tmp_bytes, &tmp));
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, rkey, rkey2, ridx, ridx2, total, 0, bits, st));
    k_gather_rows<<<grid_for(total, 256), 256, 0, st>>>(total, ridx2, hits_raw, hits);
    SDF_KERNEL(ctx);
  }
  uint8_t *px, *py, *pz;
  SDF_TRY(scratch_t(ctx, "par_x", (size_t)g.ngp, &px));
  SDF_TRY(scratch_t(ctx, "par_y", (size_t)g.ngp, &py));
  SDF_TRY(scratch_t(ctx, "par_z", (size_t)g.ngp, &pz));
  const unsigned gp = grid_for(g.ngp, 256, 148 * 16);
  SDF_MARK_ON(ctx, T_ROWS, st);
  k_axis_parity<0><<<gp, 256, 0, st>>>(g, 0, row_off, row_cnt, hits, px);
  SDF_KERNEL(ctx);
  k_axis_parity<1><<<gp, 256, 0, st>>>(g, Rx, row_off, row_cnt, hits, py);
  SDF_KERNEL(ctx);
  k_axis_parity<2><<<gp, 256, 0, st>>>(g, Rx + Ry, row_off, row_cnt, hits, pz);
  SDF_KERNEL(ctx);
  SDF_MARK_ON(ctx, T_PARITY, st);

  int32_t *und, *wind;
  uint64_t *und_have, *und_par;
  SDF_TRY(scratch_t(ctx, "und_list", (size_t)g.ngp, &und));
  SDF_TRY(scratch_t(ctx, "und_have", (size_t)g.ngp, &und_have));
  SDF_TRY(scratch_t(ctx, "und_par", (size_t)g.ngp, &und_par));
  SDF_TRY(scratch_t(ctx, "wind_list", (size_t)g.ngp, &wind));
  VoteArgs V;
  V.g = g;
  V.par[0] = px; V.par[1] = py; V.par[2] = pz;
  V.min_rays = min_rays;
  V.max_rays = max_rays;
  V.conf_thresh = conf_thresh;
  V.use_winding = use_winding;
  V.sign = d_sign;
  V.conf = d_conf;
  V.und_list = und;
  V.und_have = und_have;
  V.und_par = und_par;
  V.wind_list = wind;
  V.counters = ctx->d_counters;
  k_vote<<<grid_for(g.ngp, 256, 148 * 16), 256, 0, st>>>(V);
  SDF_KERNEL(ctx);
  SDF_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars + S_UNDECIDED, ctx->d_counters + C_LIST_UNDECIDED, sizeof(int64_t),
                                cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  const int64_t nund = ctx->h_scalars[S_UNDECIDED];
  if (nund > 0) {
    // Rounds of the adaptive vote: decide what is decidable, cast the next requested rays.
    constexpr int kRounds = 12;  // initial rays + at most 8 batches reach the 36 directions
    uint8_t* done;
    int32_t* req_node;
    int8_t* req_ray;
    int64_t* rq_cnt;
    SDF_TRY(scratch_t(ctx, "und_done", (size_t)nund, &done));
    SDF_TRY(scratch_t(ctx, "req_node", (size_t)nund * 36, &req_node));
    SDF_TRY(scratch_t(ctx, "req_ray", (size_t)nund * 36, &req_ray));
    SDF_TRY(scratch_t(ctx, "rq_cnt", (size_t)kRounds + 1, &rq_cnt));
    SDF_CUDA(ctx, cudaMemsetAsync(done, 0, (size_t)nund, st));
    SDF_CUDA(ctx, cudaMemsetAsync(rq_cnt, 0, sizeof(int64_t) * (kRounds + 1), st));
    SDF_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev_bvh, 0));  // the adaptive rays walk the LBVH
    RayArgs R;
    R.g = g;
    R.nodes = buf<BNode>(ctx, "nodes");
    R.leaf_prim = buf<int32_t>(ctx, "leaf_prim");
    R.rec = rec;
    R.pad = (float)(2e-6 * g.E);
    R.max_visits = 2 * nel + 64;
    R.par[0] = px; R.par[1] = py; R.par[2] = pz;
    R.list = und;
    R.min_rays = min_rays;
    R.max_rays = max_rays;
    R.conf_thresh = conf_thresh;
    R.use_winding = use_winding;
    R.sign = d_sign;
    R.conf = d_conf;
    R.wind_list = wind;
    R.counters = ctx->d_counters;
    R.have = und_have;
    R.parbits = und_par;
    R.done = done;
    R.req_node = req_node;
    R.req_ray = req_ray;
    R.rq_cnt = rq_cnt;
    R.speculative = nund <= 8192;
    R.last_ray = std::min(36, std::max(min_rays, max_rays));
    const int rounds = R.speculative ? 1 : kRounds;
    for (int r = 0; r < rounds; ++r) {
      k_round<<<grid_for(nund, 128), 128, 0, st>>>(R, nund, r, 0);
      SDF_KERNEL(ctx);
      k_rays<<<grid_for(nund * 8, 128, 148 * 32), 128, 0, st>>>(R, r);
      SDF_KERNEL(ctx);
    }
    k_round<<<grid_for(nund, 128), 128, 0, st>>>(R, nund, kRounds, 1);
    SDF_KERNEL(ctx);
  }
  if (use_winding) {
    SDF_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars + S_WINDING, ctx->d_counters + C_LIST_WINDING, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, st));
    SDF_CUDA(ctx, cudaStreamSynchronize(st));
    const int64_t nw = ctx->h_scalars[S_WINDING];
    if (nw > 0) {
      const int nchunks = (int)cdiv(nel, kWindChunk);
      double* partial;
      SDF_TRY(scratch_t(ctx, "wind_partial", (size_t)nw * nchunks, &partial));
      dim3 grid((unsigned)nchunks, (unsigned)std::min<int64_t>(nw, 65535));
      k_winding<<<grid, 256, 0, st>>>(g, rec, nel, wind, nw, nchunks, partial);
      SDF_KERNEL(ctx);
      k_winding_final<<<grid_for(nw, 128), 128, 0, st>>>(wind, nw, nchunks, partial, d_sign, ctx->d_counters);
      SDF_KERNEL(ctx);
    }
  }
  return 0;
}

// sdf = dist .* sign (stl_to_sdf.jl:119) on the context stream.
int run_combine(sdfgpu_ctx* ctx, const GridP& g, const double* d_dist, const double* d_sign, double* d_sdf) {
  return launch_combine(ctx, g.ngp, d_dist, d_sign, d_sdf, ctx->stream);
}

int launch_combine(sdfgpu_ctx* ctx, int64_t ngp, const double* d_dist, const double* d_sign, double* d_sdf,
                   cudaStream_t st) {
  k_combine<<<grid_for(ngp, 256, 148 * 16), 256, 0, st>>>(ngp, d_dist, d_sign, d_sdf);
  SDF_KERNEL(ctx);
  return 0;
}

}  // namespace sdfgpu
