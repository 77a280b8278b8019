// fold32.cuh -- the reference's per-candidate distance step (dfOnTriangularMesh.jl:101-176)
// decided in FP32 with explicit error bounds.
//
// Coordinates are relative to a nearby origin (the tile's first node): the node offset `pl`, the
// triangle's first vertex `a` and its edges `e1 = v2 - v1`, `e2 = v3 - v1` are FP64 differences
// rounded once to FP32, so every absolute error below is a small multiple of 2^-24 times the
// local scale Sc = |pl| + |a| + |e1| + |e2| (a few grid cells), not of the mesh's coordinates.
//
// Every quantity the step compares -- the in-plane distances behind the barycentric signs, the
// foot parameters P of the edge projections, the face / edge-foot / vertex distances -- is a
// Lipschitz function of those inputs with constant at most ~(1 + kappa), kappa = |e1||e2|/|e1 x
// e2| (1/sin of the angle at v1), so each carries an error below
//     ER = 2^-24 * Sc * (64 + 32 kappa)
// (a deliberately loose bound: a few dozen rounding steps of that size).  A decision is taken in
// FP32 only when its operands are separated by more than the sum of their bounds; otherwise the
// step reports AMBIG and the caller replays it in FP64 with the reference's arithmetic.  Exact
// vertex ties are recognised: the distance to a vertex is the same FP64 expression whichever
// triangle it comes from, so a candidate whose nearest vertex is the current winner's vertex
// cannot change the minimum.
//
// Per-triangle constants (unit edges, lengths, normal and reciprocals) are computed once per warp
// when an entry is staged, and the per-lane work compares squared distances, so the hot loops
// issue no square roots or divisions (those run on the SM's narrow special-function pipe).
#pragma once

#include "geom32.cuh"

namespace sdfgpu {

enum StepAction : int { S_NOOP = 0, S_ASSIGN = 1, S_AMBIG = 2 };

constexpr float kU = 5.9604645e-8f;  // 2^-24

// Staged candidate in the local frame.  Edges: ed0 = e1 (v1->v2), ed1 = e2 - e1 (v2->v3),
// ed2 = -e2 (v3->v1), lengths L0..L2, unit vectors u0..u2.
struct __align__(16) Cand32 {
  float4 a;    // v1 - origin; .w = kappa (inf when the triangle is not fit for FP32 decisions)
  float4 e1;   // .w = L0
  float4 e2;   // .w = L2
  float4 n;    // e1 x e2; .w = 1/|n|
  float4 u0;   // .w = L1
  float4 u1;   // .w = 1/(L0 |n|)
  float4 u2;   // .w = 1/(L1 |n|)
  int4 gid;    // global vertex ids (0-based); .w = triangle id
  float4 aux;  // .x = 1/(L2 |n|), .y = |a| + L0 + L2 (entry part of the local scale)
};

__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3f(a, a)); }
__device__ __forceinline__ float3 neg3(float3 a) { return make_float3(-a.x, -a.y, -a.z); }

__device__ __forceinline__ void make_cand(const float3 a, const float3 e1, const float3 e2, bool ok, int g0, int g1,
                                          int g2, int tri, Cand32& c) {
  const float3 ed1 = e2 - e1;
  const float L0 = len3(e1), L1 = len3(ed1), L2 = len3(e2);
  const float3 n = cross3f(e1, e2);
  const float nn = len3(n);
  const bool fine = ok && nn > 0.f && L0 > 0.f && L1 > 0.f && L2 > 0.f;
  const float inn = fine ? 1.0f / nn : 0.f;
  c.a = make_float4(a.x, a.y, a.z, fine ? L0 * L2 * inn : INFINITY);
  c.e1 = make_float4(e1.x, e1.y, e1.z, L0);
  c.e2 = make_float4(e2.x, e2.y, e2.z, L2);
  c.n = make_float4(n.x, n.y, n.z, inn);
  const float r0 = fine ? 1.0f / L0 : 0.f, r1 = fine ? 1.0f / L1 : 0.f, r2 = fine ? 1.0f / L2 : 0.f;
  c.u0 = make_float4(e1.x * r0, e1.y * r0, e1.z * r0, L1);
  c.u1 = make_float4(ed1.x * r1, ed1.y * r1, ed1.z * r1, r0 * inn);
  c.u2 = make_float4(-e2.x * r2, -e2.y * r2, -e2.z * r2, r1 * inn);
  c.gid = make_int4(g0, g1, g2, tri);
  c.aux = make_float4(r2 * inn, len3(a) + L0 + L2, 0.f, 0.f);
}

__device__ __forceinline__ float cand_err(const Cand32& c, float plen) {
  return kU * (plen + c.aux.y) * (64.f + 32.f * fminf(c.a.w, 1.0e6f));
}

// Squared point-triangle distance in the local frame (segments + plane when inside), no division
// or square root.
__device__ __forceinline__ float cand_d2(const float3 pl, const Cand32& c) {
  const float3 a = f3(c.a), e1 = f3(c.e1), e2 = f3(c.e2);
  const float3 w0 = pl - a, w1 = w0 - e1, w2 = w0 - e2;
  const float3 u0 = f3(c.u0), u1 = f3(c.u1), u2 = f3(c.u2);
  const float L0 = c.e1.w, L1 = c.u0.w, L2 = c.e2.w;
  const float P0 = fminf(fmaxf(dot3f(w0, u0), 0.f), L0);
  const float P1 = fminf(fmaxf(dot3f(w1, u1), 0.f), L1);
  const float P2 = fminf(fmaxf(dot3f(w2, u2), 0.f), L2);
  const float3 q0 = w0 - u0 * P0, q1 = w1 - u1 * P1, q2 = w2 - u2 * P2;
  float d2 = fminf(dot3f(q0, q0), fminf(dot3f(q1, q1), dot3f(q2, q2)));
  const float3 n = f3(c.n);
  if (dot3f(cross3f(e1, w0), n) >= 0.f && dot3f(cross3f(e2 - e1, w1), n) >= 0.f &&
      dot3f(cross3f(neg3(e2), w2), n) >= 0.f) {
    const float pd = dot3f(w0, n) * c.n.w;
    d2 = fminf(d2, pd * pd);
  }
  return d2;
}

// m, em: FP32 estimate of the running minimum and its error bound.  win_gid: global vertex id of
// the current winner when the winner is a vertex, else -1.  quirk: the reference's vertex-skip
// rule (REF_RULE) or the true minimum (EXACT).
__device__ __forceinline__ int step32(const float3 pl, float plen, const Cand32& c, float m, float em, bool quirk,
                                      int win_gid, float& val, int& feat, float& err) {
  const float kappa = c.a.w;
  if (!(kappa < 1.0e4f)) return S_AMBIG;
  const float ER = cand_err(c, plen);
  err = ER;
  const float lo = m - (ER + em), hi = m + (ER + em);
  const float lo2 = lo > 0.f ? lo * lo : -1.f, hi2 = hi * hi;
  const float3 a = f3(c.a), e1 = f3(c.e1), e2 = f3(c.e2), n = f3(c.n);
  const float3 wv[3] = {pl - a, pl - a - e1, pl - a - e2};
  const float3 ed[3] = {e1, e2 - e1, neg3(e2)};
  const float il[3] = {c.u1.w, c.u2.w, c.aux.x};
  // barycentric signs via the in-plane signed distance of p's projection from each edge line
  bool any_out = false, all_in = true;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float sd = dot3f(cross3f(ed[i], wv[i]), n) * il[i];
    if (sd < -ER) any_out = true;
    else if (!(sd > ER)) all_in = false;
  }
  if (!any_out && !all_in) return S_AMBIG;
  if (!any_out) {  // face branch
    const float f = fabsf(dot3f(wv[0], n)) * c.n.w;
    if (f < lo) { val = f; feat = F_FACE; return S_ASSIGN; }
    return f > hi ? S_NOOP : S_AMBIG;
  }
  // edge branch: feet on the three edges
  const float3 uu[3] = {f3(c.u0), f3(c.u1), f3(c.u2)};
  const float L[3] = {c.e1.w, c.u0.w, c.e2.w};
  float Ea = 3.0e38f, Eb = 3.0e38f;  // smallest and second smallest squared foot distances
  int jmin = -1;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const float P = dot3f(wv[j], uu[j]);
    if (P < -ER || P > L[j] + ER) continue;          // clearly invalid
    if (!(P > ER && P < L[j] - ER)) return S_AMBIG;  // validity undecided
    const float3 q = wv[j] - uu[j] * P;
    const float d2 = dot3f(q, q);
    if (d2 < Ea) { Eb = Ea; Ea = d2; jmin = j; }
    else if (d2 < Eb) Eb = d2;
  }
  const float dv[3] = {dot3f(wv[0], wv[0]), dot3f(wv[1], wv[1]), dot3f(wv[2], wv[2])};
  int kmin = 0;
  if (dv[1] < dv[kmin]) kmin = 1;
  if (dv[2] < dv[kmin]) kmin = 2;
  float Vb = 3.0e38f;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (k != kmin) Vb = fminf(Vb, dv[k]);
  const float Va = dv[kmin];
  const int vgid = kmin == 0 ? c.gid.x : (kmin == 1 ? c.gid.y : c.gid.z);
  if (jmin >= 0) {
    if (quirk) {
      if (Ea < lo2) {  // an edge foot improves the minimum: vertices are skipped
        const float E = sqrtf(Ea);
        if (sqrtf(Eb) - E <= 2.f * ER) return S_AMBIG;
        val = E; feat = F_EDGE0 + jmin;
        return S_ASSIGN;
      }
      if (!(Ea > hi2)) return S_AMBIG;
    } else {
      const float E = sqrtf(Ea), V = sqrtf(Va);
      if (E < V - 2.f * ER) {  // true minimum: the foot is nearer than every vertex
        if (E < lo) {
          if (sqrtf(Eb) - E <= 2.f * ER) return S_AMBIG;
          val = E; feat = F_EDGE0 + jmin;
          return S_ASSIGN;
        }
        return E > hi ? S_NOOP : S_AMBIG;
      }
      if (!(E > V + 2.f * ER)) return S_AMBIG;
    }
  }
  // vertex check
  if (Va < lo2) {
    const float V = sqrtf(Va);
    if (sqrtf(Vb) - V <= 2.f * ER) return S_AMBIG;
    val = V; feat = F_VERT0 + kmin;
    return S_ASSIGN;
  }
  if (Va > hi2) return S_NOOP;
  // |V - m| within the bounds: an exact tie when the winner is this very vertex and the others
  // are clearly farther (same FP64 expression, so "V < m" is false)
  if (vgid == win_gid && Vb > hi2) return S_NOOP;
  return S_AMBIG;
}

}  // namespace sdfgpu
