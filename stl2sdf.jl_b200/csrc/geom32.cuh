// geom32.cuh -- FP32 geometry for the bulk of the work: point-triangle distance and ray-box
// tests in mesh-local coordinates (vertices minus the mesh's bounding-box centre).  Every FP32
// result is used only as a filter with an explicit error margin; decisions that land inside the
// margin are re-made with the FP64 routines of exact64.cuh.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace sdfgpu {

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3f(float3 a, float3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ float3 cross3f(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// Squared distance from p to segment [a, a+e].
__device__ __forceinline__ float seg_d2(float3 p, float3 a, float3 e) {
  const float3 w = p - a;
  const float ee = dot3f(e, e);
  float t = ee > 0.f ? dot3f(w, e) / ee : 0.f;
  t = fminf(fmaxf(t, 0.f), 1.f);
  const float3 q = w - e * t;
  return dot3f(q, q);
}

// Squared distance from p to triangle (a, b, c): minimum of the three edge distances and, when
// p projects inside, the plane distance.  Degenerate triangles reduce to their edges.
__device__ __forceinline__ float pt_tri_d2(float3 p, float3 a, float3 b, float3 c) {
  const float3 ab = b - a, bc = c - b, ca = a - c;
  float d2 = fminf(seg_d2(p, a, ab), fminf(seg_d2(p, b, bc), seg_d2(p, c, ca)));
  const float3 n = cross3f(ab, c - a);
  const float nn = dot3f(n, n);
  if (nn > 0.f) {
    const float s1 = dot3f(cross3f(ab, p - a), n);
    const float s2 = dot3f(cross3f(bc, p - b), n);
    const float s3 = dot3f(cross3f(ca, p - c), n);
    if (s1 >= 0.f && s2 >= 0.f && s3 >= 0.f) {
      const float pd = dot3f(p - a, n);
      d2 = fminf(d2, pd * pd / nn);
    }
  }
  return d2;
}

// Oriented box of an LBVH child subtree (mesh-local FP32).  For every vertex x of the subtree's
// triangles, and so for every point of them, |x . a_k - c_k| <= e_k along the three stored axes
// a_k (the inequality holds in exact arithmetic on the stored FP32 values).  a0..a2 hold
// (a_k.x, a_k.y, a_k.z, c_k), e holds (e_0, e_1, e_2, 0).  A child without a fitted box carries
// extents kNoObb, for which the bound below is 0.
struct __align__(16) OBox {
  float4 a0, a1, a2, e;
};
constexpr float kNoObb = 3.0e38f;

// Squared lower bound on the distance from p to the points of an oriented box: the axes are
// orthonormal to FP32 rounding, so the sum over axes of (|p . a_k - c_k| - e_k)_+^2 is the squared
// distance to the box up to a relative 1e-6 (callers add an absolute margin for it and for the
// rounding of this evaluation).
__device__ __forceinline__ float obox_d2(float3 p, const OBox& o) {
  const float t0 = fabsf(fmaf(p.x, o.a0.x, fmaf(p.y, o.a0.y, fmaf(p.z, o.a0.z, -o.a0.w)))) - o.e.x;
  const float t1 = fabsf(fmaf(p.x, o.a1.x, fmaf(p.y, o.a1.y, fmaf(p.z, o.a1.z, -o.a1.w)))) - o.e.y;
  const float t2 = fabsf(fmaf(p.x, o.a2.x, fmaf(p.y, o.a2.y, fmaf(p.z, o.a2.z, -o.a2.w)))) - o.e.z;
  const float u0 = fmaxf(t0, 0.f), u1 = fmaxf(t1, 0.f), u2 = fmaxf(t2, 0.f);
  return fmaf(u0, u0, fmaf(u1, u1, u2 * u2));
}

// Leaf-ordered FP32 record of one triangle for the unbounded searches (mesh-local; every field
// rounded once from its FP64 value): vertex a, edges e0 = b - a and e1 = c - a, the inverse squared
// lengths of e0, e1 and c - b, the unit normal n and, for each edge, the unit in-plane normal m_k
// pointing into the triangle with its offset o_k (a point of the plane lies inside when
// (p - a).m_k >= o_k for k = 0, 1, 2).  A triangle without area has m_k = 0 and o_k = 1 and
// reduces to its three edges.
struct __align__(16) LeafTri {
  float4 a;   // a.xyz, 1 / |e0|^2
  float4 e0;  // e0.xyz, 1 / |e1|^2
  float4 e1;  // e1.xyz, 1 / |c - b|^2
  float4 n;   // n.xyz, triangle index (int bits)
  float4 m0;  // edge a -> b: m0.xyz, o0 = 0
  float4 m1;  // edge b -> c: m1.xyz, o1 = e0.m1
  float4 m2;  // edge c -> a: m2.xyz, o2 = e1.m2
};

__device__ __forceinline__ float clamp01(float t) { return fminf(fmaxf(t, 0.f), 1.f); }

// Squared distance from p to the triangle of T, without division or branch: the smallest squared
// distance to the three edges, and the squared plane distance when p projects inside.  Every
// rounding is relative to |w| <= d + |e| (w = p - a, d the distance, e the longest edge) or to
// |e|, and the inside test compares physical distances to the edge lines (no barycentric
// division), so for inputs within E of the origin the result is within about 7e-7 E + 4e-7 d of
// the exact distance to the FP64 triangle, whatever its shape -- at least 5x inside the FP32 band
// of the unbounded searches (4e-6 E + 4e-6 d).
__device__ __forceinline__ float leaf_d2(float3 p, const LeafTri& T) {
  const float wx = p.x - T.a.x, wy = p.y - T.a.y, wz = p.z - T.a.z;
  const float t0 = clamp01(fmaf(wx, T.e0.x, fmaf(wy, T.e0.y, wz * T.e0.z)) * T.a.w);
  const float t1 = clamp01(fmaf(wx, T.e1.x, fmaf(wy, T.e1.y, wz * T.e1.z)) * T.e0.w);
  const float q0x = fmaf(-t0, T.e0.x, wx), q0y = fmaf(-t0, T.e0.y, wy), q0z = fmaf(-t0, T.e0.z, wz);
  const float q1x = fmaf(-t1, T.e1.x, wx), q1y = fmaf(-t1, T.e1.y, wy), q1z = fmaf(-t1, T.e1.z, wz);
  const float e2x = T.e1.x - T.e0.x, e2y = T.e1.y - T.e0.y, e2z = T.e1.z - T.e0.z;  // c - b
  const float wbx = wx - T.e0.x, wby = wy - T.e0.y, wbz = wz - T.e0.z;              // p - b
  const float t2 = clamp01(fmaf(wbx, e2x, fmaf(wby, e2y, wbz * e2z)) * T.e1.w);
  const float q2x = fmaf(-t2, e2x, wbx), q2y = fmaf(-t2, e2y, wby), q2z = fmaf(-t2, e2z, wbz);
  float d2 = fminf(fmaf(q0x, q0x, fmaf(q0y, q0y, q0z * q0z)),
                   fminf(fmaf(q1x, q1x, fmaf(q1y, q1y, q1z * q1z)), fmaf(q2x, q2x, fmaf(q2y, q2y, q2z * q2z))));
  const bool in0 = fmaf(wx, T.m0.x, fmaf(wy, T.m0.y, wz * T.m0.z)) >= T.m0.w;
  const bool in1 = fmaf(wx, T.m1.x, fmaf(wy, T.m1.y, wz * T.m1.z)) >= T.m1.w;
  const bool in2 = fmaf(wx, T.m2.x, fmaf(wy, T.m2.y, wz * T.m2.z)) >= T.m2.w;
  const float dp = fmaf(wx, T.n.x, fmaf(wy, T.n.y, wz * T.n.z));
  if (in0 && in1 && in2) d2 = fminf(d2, dp * dp);
  return d2;
}

// Squared distance from p to the box [lo, hi].
__device__ __forceinline__ float box_d2(float3 p, float3 lo, float3 hi) {
  const float dx = fmaxf(fmaxf(lo.x - p.x, p.x - hi.x), 0.f);
  const float dy = fmaxf(fmaxf(lo.y - p.y, p.y - hi.y), 0.f);
  const float dz = fmaxf(fmaxf(lo.z - p.z, p.z - hi.z), 0.f);
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// Slab test of the half-line o + t d (t >= -tpad) against [lo - pad, hi + pad].  inv holds
// 1/d per axis (inf where d is 0; such axes test containment of o instead).
__device__ __forceinline__ bool ray_box(float3 o, float3 d, float3 inv, float3 lo, float3 hi, float pad,
                                        float tpad) {
  float t0 = -tpad, t1 = 3.0e38f;
  if (d.x != 0.f) {
    float a = (lo.x - pad - o.x) * inv.x, b = (hi.x + pad - o.x) * inv.x;
    t0 = fmaxf(t0, fminf(a, b)); t1 = fminf(t1, fmaxf(a, b));
  } else if (o.x < lo.x - pad || o.x > hi.x + pad) return false;
  if (d.y != 0.f) {
    float a = (lo.y - pad - o.y) * inv.y, b = (hi.y + pad - o.y) * inv.y;
    t0 = fmaxf(t0, fminf(a, b)); t1 = fminf(t1, fmaxf(a, b));
  } else if (o.y < lo.y - pad || o.y > hi.y + pad) return false;
  if (d.z != 0.f) {
    float a = (lo.z - pad - o.z) * inv.z, b = (hi.z + pad - o.z) * inv.z;
    t0 = fmaxf(t0, fminf(a, b)); t1 = fminf(t1, fmaxf(a, b));
  } else if (o.z < lo.z - pad || o.z > hi.z + pad) return false;
  return t0 <= t1 + tpad;
}

}  // namespace sdfgpu
