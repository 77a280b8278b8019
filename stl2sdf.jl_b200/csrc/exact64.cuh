// exact64.cuh -- FP64 device arithmetic that replays the reference's Julia Float64 expressions
// operation by operation.  Every product, sum and quotient is a separately rounded IEEE
// operation (__dmul_rn / __dadd_rn / __dsub_rn / __ddiv_rn / __dsqrt_rn never contract into an
// FMA), so a node evaluated here gets the same bits as the same expression evaluated on the host
// without FMA contraction.
//
// Reference expressions restated (paths relative to the stl2sdf.jl project):
//   dot(x, y) for length-3 Vector{Float64} (BLAS ddot): ((x1*y1) + x2*y2) + x3*y3
//   cross(a, b): LinearAlgebra.cross
//   norm(x): generic_norm2 (length < 32): sqrt((x1^2 + x2^2) + x3^2), with its zero / scaling cases
//   barycentricCoordinates  src/SignedDistances/dfOnTriangularMesh.jl:226-251, solved as Julia's
//     `\` solves a 3x3 Matrix{Float64}: triangular structure first, else LU with partial pivoting
//   per-candidate distance step  src/SignedDistances/dfOnTriangularMesh.jl:101-177
//   ray_triangle_intersection    src/SignedDistances/RaycastingSignDetection.jl:64-106
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace sdfgpu {

#define SDF_HD __host__ __device__ __forceinline__

struct d3 {
  double x, y, z;
};

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ d3 v_sub(const d3& a, const d3& b) { return {ds(a.x, b.x), ds(a.y, b.y), ds(a.z, b.z)}; }
__device__ __forceinline__ d3 v_add(const d3& a, const d3& b) { return {da(a.x, b.x), da(a.y, b.y), da(a.z, b.z)}; }
__device__ __forceinline__ d3 v_scale(const d3& a, double s) { return {dm(a.x, s), dm(a.y, s), dm(a.z, s)}; }
__device__ __forceinline__ d3 v_div(const d3& a, double s) { return {dd(a.x, s), dd(a.y, s), dd(a.z, s)}; }
__device__ __forceinline__ d3 v_neg(const d3& a) { return {-a.x, -a.y, -a.z}; }

__device__ __forceinline__ double v_dot(const d3& a, const d3& b) {
  double s = dm(a.x, b.x);
  s = da(s, dm(a.y, b.y));
  s = da(s, dm(a.z, b.z));
  return s;
}

__device__ __forceinline__ d3 v_cross(const d3& a, const d3& b) {
  return {ds(dm(a.y, b.z), dm(a.z, b.y)), ds(dm(a.z, b.x), dm(a.x, b.z)), ds(dm(a.x, b.y), dm(a.y, b.x))};
}

__device__ __forceinline__ double v_norm(const d3& a) {
  const double ax = fabs(a.x), ay = fabs(a.y), az = fabs(a.z);
  double m;
  if (isnan(ax) || isnan(ay) || isnan(az)) {
    m = __longlong_as_double(0x7ff8000000000000LL);
  } else {
    m = fmax(ax, fmax(ay, az));
  }
  if (m == 0.0 || isinf(m)) return m;
  const double mm = dm(m, m);
  if (isfinite(dm(dm(3.0, m), m)) && mm != 0.0) {
    double s = dm(a.x, a.x);
    s = da(s, dm(a.y, a.y));
    s = da(s, dm(a.z, a.z));
    return __dsqrt_rn(s);
  }
  const double qx = dd(ax, m), qy = dd(ay, m), qz = dd(az, m);
  double s = dm(qx, qx);
  s = da(s, dm(qy, qy));
  s = da(s, dm(qz, qz));
  return dm(m, __dsqrt_rn(s));
}

// LinearAlgebra.normalize: multiply by inv(norm); norms below 1/floatmax take the scaled branch.
__device__ __forceinline__ d3 v_normalize(const d3& a) {
  const double nrm = v_norm(a);
  const double delta = 1.0 / 1.7976931348623157e308;  // inv(prevfloat(typemax(Float64)))
  if (nrm >= delta) {
    const double inv = dd(1.0, nrm);
    return v_scale(a, inv);
  }
  const double ed = 2.220446049250313e-16 / delta;  // eps(1.0) / delta
  const d3 b = v_scale(a, ed);
  return v_scale(b, dd(1.0, dm(nrm, ed)));
}

// Per-triangle FP64 record (dfOnTriangularMesh.jl:307-368 plus the factored barycentric system).
// kind: 0 LU (A holds L below / U on and above the diagonal, piv the row swaps),
//       1 lower triangular, 2 upper triangular, 3 diagonal (A holds the unfactored matrix).
struct __align__(16) TriRec64 {
  double v[9];    // v1, v2, v3
  double u[9];    // e_j / L_j
  double L[3];    // |e_j|
  double n[3];    // unit normal cross(e1, -e3) / norm
  double bmin[3], bmax[3];
  double A[9];    // barycentric system (row major)
  int32_t kind;
  int32_t imax;   // row replaced by [1 1 1]
  int32_t piv;    // piv0 | piv1 << 4 | piv2 << 8
  int32_t pad;
};

__device__ __forceinline__ d3 rec_v(const TriRec64& r, int k) { return {r.v[3 * k], r.v[3 * k + 1], r.v[3 * k + 2]}; }

// Builds the barycentric matrix of one triangle and factors it exactly as the oracle's solve3.
__device__ inline void factor_bary(TriRec64& r) {
  const d3 x1 = rec_v(r, 0), x2 = rec_v(r, 1), x3 = rec_v(r, 2);
  const d3 n = {r.n[0], r.n[1], r.n[2]};
  double A[3][3] = {
      {ds(dm(x1.y, n.z), dm(x1.z, n.y)), ds(dm(x2.y, n.z), dm(x2.z, n.y)), ds(dm(x3.y, n.z), dm(x3.z, n.y))},
      {ds(dm(x1.z, n.x), dm(x1.x, n.z)), ds(dm(x2.z, n.x), dm(x2.x, n.z)), ds(dm(x3.z, n.x), dm(x3.x, n.z))},
      {ds(dm(x1.x, n.y), dm(x1.y, n.x)), ds(dm(x2.x, n.y), dm(x2.y, n.x)), ds(dm(x3.x, n.y), dm(x3.y, n.x))}};
  const double an[3] = {fabs(n.x), fabs(n.y), fabs(n.z)};
  int imax;
  if (isnan(an[0])) imax = 0;
  else if (isnan(an[1])) imax = 1;
  else if (isnan(an[2])) imax = 2;
  else {
    imax = 0;
    if (an[1] > an[imax]) imax = 1;
    if (an[2] > an[imax]) imax = 2;
  }
  A[imax][0] = A[imax][1] = A[imax][2] = 1.0;
  r.imax = imax;
  const bool tril = A[0][1] == 0.0 && A[0][2] == 0.0 && A[1][2] == 0.0;
  const bool triu = A[1][0] == 0.0 && A[2][0] == 0.0 && A[2][1] == 0.0;
  int piv[3] = {0, 1, 2};
  if (tril && triu) {
    r.kind = 3;
  } else if (tril) {
    r.kind = 1;
  } else if (triu) {
    r.kind = 2;
  } else {
    r.kind = 0;
    for (int j = 0; j < 3; ++j) {
      int p = j;
      double pm = fabs(A[j][j]);
      for (int i = j + 1; i < 3; ++i) {
        const double v = fabs(A[i][j]);
        if (v > pm) { pm = v; p = i; }
      }
      piv[j] = p;
      if (p != j)
        for (int k = 0; k < 3; ++k) { const double t = A[j][k]; A[j][k] = A[p][k]; A[p][k] = t; }
      if (A[j][j] != 0.0) {
        const double rcp = dd(1.0, A[j][j]);
        for (int i = j + 1; i < 3; ++i) A[i][j] = dm(A[i][j], rcp);
      }
      for (int i = j + 1; i < 3; ++i)
        for (int k = j + 1; k < 3; ++k) A[i][k] = ds(A[i][k], dm(A[i][j], A[j][k]));
    }
  }
  r.piv = piv[0] | (piv[1] << 4) | (piv[2] << 8);
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) r.A[3 * i + k] = A[i][k];
}

// barycentricCoordinates(x1, x2, x3, n, p) with the prepared system of the triangle.
__device__ __forceinline__ void bary_solve(const TriRec64& r, const d3& x, double lam[3]) {
  const double n0 = r.n[0], n1 = r.n[1], n2 = r.n[2];
  double b[3] = {ds(dm(x.y, n2), dm(x.z, n1)), ds(dm(x.z, n0), dm(x.x, n2)), ds(dm(x.x, n1), dm(x.y, n0))};
  b[r.imax] = 1.0;
  const double* A = r.A;
  switch (r.kind) {
    case 3:
      lam[0] = dd(b[0], A[0]); lam[1] = dd(b[1], A[4]); lam[2] = dd(b[2], A[8]);
      return;
    case 1: {
      double y1 = b[1], y2 = b[2];
      lam[0] = dd(b[0], A[0]);
      y1 = ds(y1, dm(lam[0], A[3]));
      y2 = ds(y2, dm(lam[0], A[6]));
      lam[1] = dd(y1, A[4]);
      y2 = ds(y2, dm(lam[1], A[7]));
      lam[2] = dd(y2, A[8]);
      return;
    }
    case 2: {
      double y0 = b[0], y1 = b[1];
      lam[2] = dd(b[2], A[8]);
      y0 = ds(y0, dm(lam[2], A[2]));
      y1 = ds(y1, dm(lam[2], A[5]));
      lam[1] = dd(y1, A[4]);
      y0 = ds(y0, dm(lam[1], A[1]));
      lam[0] = dd(y0, A[0]);
      return;
    }
    default: {
      double y[3] = {b[0], b[1], b[2]};
      const int p0 = r.piv & 15, p1 = (r.piv >> 4) & 15, p2 = (r.piv >> 8) & 15;
      if (p0 != 0) { const double t = y[0]; y[0] = y[p0]; y[p0] = t; }
      if (p1 != 1) { const double t = y[1]; y[1] = y[p1]; y[p1] = t; }
      if (p2 != 2) { const double t = y[2]; y[2] = y[p2]; y[p2] = t; }
      y[1] = ds(y[1], dm(y[0], A[3]));
      y[2] = ds(y[2], dm(y[0], A[6]));
      y[2] = ds(y[2], dm(y[1], A[7]));
      y[2] = dd(y[2], A[8]);
      y[0] = ds(y[0], dm(y[2], A[2]));
      y[1] = ds(y[1], dm(y[2], A[5]));
      y[1] = dd(y[1], A[4]);
      y[0] = ds(y[0], dm(y[1], A[1]));
      y[0] = dd(y[0], A[0]);
      lam[0] = y[0]; lam[1] = y[1]; lam[2] = y[2];
      return;
    }
  }
}

// One candidate of the reference's per-node loop (dfOnTriangularMesh.jl:104-176).  quirk = true
// keeps the reference rule (vertices only when no edge foot improved the running minimum);
// quirk = false evaluates the true point-triangle minimum with the same arithmetic.
__device__ inline void tri_step64(const TriRec64& r, const d3& p, double& m, d3& proj, bool quirk) {
  if (p.x < ds(r.bmin[0], m) || p.x > da(r.bmax[0], m)) return;
  if (p.y < ds(r.bmin[1], m) || p.y > da(r.bmax[1], m)) return;
  if (p.z < ds(r.bmin[2], m) || p.z > da(r.bmax[2], m)) return;
  double lam[3];
  bary_solve(r, p, lam);
  const d3 v0 = rec_v(r, 0), v1 = rec_v(r, 1), v2 = rec_v(r, 2);
  if (lam[0] >= 0.0 && lam[1] >= 0.0 && lam[2] >= 0.0) {
    const d3 xp = v_add(v_add(v_scale(v0, lam[0]), v_scale(v1, lam[1])), v_scale(v2, lam[2]));
    const double d = v_norm(v_sub(p, xp));
    if (d < m) { m = d; proj = xp; }
    return;
  }
  bool improved = false;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const d3 vj = rec_v(r, j);
    const d3 u = {r.u[3 * j], r.u[3 * j + 1], r.u[3 * j + 2]};
    const double P = v_dot(v_sub(p, vj), u);
    if (P >= 0.0 && P <= r.L[j]) {
      const d3 xp = v_add(vj, v_scale(u, P));
      const double d = v_norm(v_sub(p, xp));
      if (d < m) { m = d; proj = xp; improved = true; }
    }
  }
  if (!improved || !quirk) {
    const double d0 = v_norm(v_sub(p, v0)), d1 = v_norm(v_sub(p, v1)), d2 = v_norm(v_sub(p, v2));
    if (isnan(d0) || isnan(d1) || isnan(d2)) return;
    int idx = 0;
    double best = d0;
    if (d1 < best) { best = d1; idx = 1; }
    if (d2 < best) { best = d2; idx = 2; }
    if (best < m) { m = best; proj = idx == 0 ? v0 : (idx == 1 ? v1 : v2); }
  }
}

// Features a reference step can assign to the running minimum.
enum Feature : int { F_FACE = 0, F_EDGE0 = 1, F_EDGE1 = 2, F_EDGE2 = 3, F_VERT0 = 4, F_VERT1 = 5, F_VERT2 = 6 };

// The value (and closest point) tri_step64 assigns when `feat` wins: the same expressions, so the
// result has the same bits.
__device__ __forceinline__ void feature64(const TriRec64& r, const d3& p, int feat, double& d, d3& xp) {
  if (feat == F_FACE) {
    double lam[3];
    bary_solve(r, p, lam);
    xp = v_add(v_add(v_scale(rec_v(r, 0), lam[0]), v_scale(rec_v(r, 1), lam[1])), v_scale(rec_v(r, 2), lam[2]));
  } else if (feat <= F_EDGE2) {
    const int j = feat - F_EDGE0;
    const d3 vj = rec_v(r, j);
    const d3 u = {r.u[3 * j], r.u[3 * j + 1], r.u[3 * j + 2]};
    const double P = v_dot(v_sub(p, vj), u);
    xp = v_add(vj, v_scale(u, P));
  } else {
    xp = rec_v(r, feat - F_VERT0);
  }
  d = v_norm(v_sub(p, xp));
}

// Möller–Trumbore with the reference's decisions (RaycastingSignDetection.jl:64-106).
__device__ __forceinline__ bool mt64(const d3& o, const d3& d, const d3& v1, const d3& v2, const d3& v3,
                                     double eps, double& tout) {
  const d3 e1 = v_sub(v2, v1), e2 = v_sub(v3, v1);
  const d3 h = v_cross(d, e2);
  const double a = v_dot(e1, h);
  if (fabs(a) < eps) return false;
  const double f = dd(1.0, a);
  const d3 s = v_sub(o, v1);
  const double u = dm(f, v_dot(s, h));
  if (u < 0.0 || u > 1.0) return false;
  const d3 q = v_cross(s, e1);
  const double v = dm(f, v_dot(d, q));
  if (v < 0.0 || da(u, v) > 1.0) return false;
  const double t = dm(f, v_dot(e2, q));
  if (t > eps) { tout = t; return true; }
  return false;
}

// Node coordinate AABB_min .+ cell_size .* [i, j, k] (Grid.jl:90).
__device__ __forceinline__ d3 node_coord(const double o[3], double h, int64_t i, int64_t j, int64_t k) {
  return {da(o[0], dm(h, (double)i)), da(o[1], dm(h, (double)j)), da(o[2], dm(h, (double)k))};
}

}  // namespace sdfgpu
