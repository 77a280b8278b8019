// sdf_oracle.cpp -- CPU FP64 oracle for the SignedDistances hot path of stl2sdf.jl.
//
// TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path and the timed CPU
// baseline ("port") of bench.py.  Nothing in the product links, loads or calls it.
//
// It restates, in plain IEEE double arithmetic with no FMA contraction (built with
// -ffp-contract=off), the algorithm of the reference (paths relative to the reference project):
//   src/MeshGrid/Grid.jl:9-32                Grid constructor (cell size, padding, N, ngp)
//   src/MeshGrid/Grid.jl:82-96               generateGridPoints (node = AABB_min + h*[i,j,k])
//   src/MeshGrid/Grid_setup.jl:104-124       noninteractive_sdf_grid_setup (N_new = floor(ext/B))
//   src/SignedDistances/dfOnTriangularMesh.jl:19-209   evalDistancesOnTriMesh (candidate rule,
//                                            vertex-skip quirk, thread merge, clamp to cell_size)
//   src/SignedDistances/dfOnTriangularMesh.jl:226-251  barycentricCoordinates (3x3 solve)
//   src/SignedDistances/dfOnTriangularMesh.jl:329-368  prepare_triangle_data
//   src/SignedDistances/dfOnTriangularMesh.jl:385-392  point_in_box_range
//   src/SignedDistances/RaycastingSignDetection.jl:64-106   ray_triangle_intersection (MT)
//   src/SignedDistances/RaycastingSignDetection.jl:114-154  check_ray_inside_bvh (sort, dedupe)
//   src/SignedDistances/RaycastingSignDetection.jl:162-227  generate_ray_directions_prioritized
//   src/SignedDistances/RaycastingSignDetection.jl:234-288  adaptive_point_in_mesh_raycast
//   src/SignedDistances/RaycastingSignDetection.jl:295-328  generalized_winding_number
//   src/SignedDistances/RaycastingSignDetection.jl:337-404  raycast_sign_detection
//
// PARITY UNPINNED.  The reference is Julia 1.10; no Julia toolchain exists in this environment and
// the reference ships no golden vectors, so this restatement is not pinned against reference
// outputs.  It is pinned against analytic known answers (tests/test_oracle.py).  Third-party
// arithmetic that is not restated bit for bit:
//   * NearestNeighbors.jl 0.4.22 `inrange` return order: candidates are folded in ascending
//     triangle index (the order only matters for the vertex-skip quirk); `knn` ties broken by
//     lower vertex index; the Set{Int} union of the knn fallback is folded in ascending order.
//   * OpenBLAS ddot (Julia `dot` on Vector{Float64}) and getrf/getrs (Julia `\`): plain
//     left-to-right products without FMA; right-looking LU with partial pivoting.
//   * ImplicitBVH.jl 0.6.0 `traverse_rays`: assumed conservative (it only prunes), so the ray
//     candidates are every triangle whose box the ray meets; an own AABB BVH is used here.
//   * Julia's own sin/cos/atan: the C library's are used (differences of at most an ulp).
//
// Sign convention of the reference: +1 = inside, -1 = outside.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
  double x, y, z;
};

inline V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(const V3& a, const V3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 scale(const V3& a, double s) { return {a.x * s, a.y * s, a.z * s}; }  // vector * scalar
inline V3 divs(const V3& a, double s) { return {a.x / s, a.y / s, a.z / s}; }   // vector / scalar
inline V3 neg(const V3& a) { return {-a.x, -a.y, -a.z}; }

// Julia `dot` on Vector{Float64} -> BLAS ddot; for n = 3 the sum runs left to right.
inline double dot3(const V3& a, const V3& b) {
  double s = a.x * b.x;
  s = s + a.y * b.y;
  s = s + a.z * b.z;
  return s;
}

// LinearAlgebra.cross for length-3 vectors.
inline V3 cross(const V3& a, const V3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// LinearAlgebra.norm for a length-3 Vector{Float64}: generic_norm2 (length < NRM2_CUTOFF).
inline double norm3(const V3& a) {
  double ax = std::fabs(a.x), ay = std::fabs(a.y), az = std::fabs(a.z);
  double m;
  if (std::isnan(ax) || std::isnan(ay) || std::isnan(az)) {
    m = std::numeric_limits<double>::quiet_NaN();
  } else {
    m = std::max(ax, std::max(ay, az));
  }
  if (m == 0.0 || std::isinf(m)) return m;
  if (std::isfinite(3.0 * m * m) && (m * m) != 0.0) {
    double s = a.x * a.x;
    s = s + a.y * a.y;
    s = s + a.z * a.z;
    return std::sqrt(s);
  }
  double s = (ax / m) * (ax / m);
  s = s + (ay / m) * (ay / m);
  s = s + (az / m) * (az / m);
  return m * std::sqrt(s);
}

// LinearAlgebra.normalize (multiplies by inv(norm); tiny norms take the scaled branch).
inline V3 normalize3(const V3& a) {
  const double nrm = norm3(a);
  const double delta = 1.0 / std::numeric_limits<double>::max();
  if (nrm >= delta) {
    const double inv = 1.0 / nrm;
    return scale(a, inv);
  }
  const double ed = std::numeric_limits<double>::epsilon() / delta;
  V3 b = scale(a, ed);
  return scale(b, 1.0 / (nrm * ed));
}

// ---------------------------------------------------------------------------------------------
// Grid (Grid.jl:9-32, Grid_setup.jl:117-120, Grid.jl:90)
// ---------------------------------------------------------------------------------------------
struct Grid {
  double origin[3];  // padded AABB_min
  double amax[3];    // AABB_max after the exact-fit adjustment
  int64_t N[3];
  double h;
  int64_t ngp;
};

inline V3 node_coord(const Grid& g, int64_t lin) {
  const int64_t nx = g.N[0] + 1, ny = g.N[1] + 1;
  const int64_t i = lin % nx;
  const int64_t j = (lin / nx) % ny;
  const int64_t k = lin / (nx * ny);
  // AABB_min .+ cell_size .* [i, j, k]: one multiply, one add, no FMA.
  return {g.origin[0] + g.h * (double)i, g.origin[1] + g.h * (double)j,
          g.origin[2] + g.h * (double)k};
}

// ---------------------------------------------------------------------------------------------
// Triangle data (dfOnTriangularMesh.jl:307-368)
// ---------------------------------------------------------------------------------------------
struct Tri {
  V3 v[3];
  V3 e[3];   // e1 = v2 - v1, e2 = v3 - v2, e3 = v1 - v3
  double L[3];
  V3 n;      // cross(e1, -e3) / norm
  V3 c;      // (v1 + v2 + v3) / 3
  V3 bmin, bmax;
};

std::vector<Tri> prepare_triangles(const double* X, int64_t nnp, const int64_t* IEN, int64_t nel) {
  (void)nnp;
  std::vector<Tri> T((size_t)nel);
  for (int64_t el = 0; el < nel; ++el) {
    Tri& t = T[(size_t)el];
    for (int k = 0; k < 3; ++k) {
      const int64_t vi = IEN[3 * el + k] - 1;
      t.v[k] = {X[3 * vi + 0], X[3 * vi + 1], X[3 * vi + 2]};
    }
    t.e[0] = sub(t.v[1], t.v[0]);
    t.e[1] = sub(t.v[2], t.v[1]);
    t.e[2] = sub(t.v[0], t.v[2]);
    for (int j = 0; j < 3; ++j) t.L[j] = norm3(t.e[j]);
    V3 nn = cross(t.e[0], neg(t.e[2]));
    t.n = divs(nn, norm3(nn));
    t.c = divs(add(add(t.v[0], t.v[1]), t.v[2]), 3.0);
    t.bmin = {std::min(t.v[0].x, std::min(t.v[1].x, t.v[2].x)),
              std::min(t.v[0].y, std::min(t.v[1].y, t.v[2].y)),
              std::min(t.v[0].z, std::min(t.v[1].z, t.v[2].z))};
    t.bmax = {std::max(t.v[0].x, std::max(t.v[1].x, t.v[2].x)),
              std::max(t.v[0].y, std::max(t.v[1].y, t.v[2].y)),
              std::max(t.v[0].z, std::max(t.v[1].z, t.v[2].z))};
  }
  return T;
}

// ---------------------------------------------------------------------------------------------
// barycentricCoordinates (dfOnTriangularMesh.jl:226-251) with Julia's `\` for a 3x3 matrix:
// triangular structure is detected first (istril / istriu), otherwise LU with partial pivoting.
// ---------------------------------------------------------------------------------------------
void solve3(double A[3][3], double b[3], double x[3]) {
  const bool tril = A[0][1] == 0.0 && A[0][2] == 0.0 && A[1][2] == 0.0;
  const bool triu = A[1][0] == 0.0 && A[2][0] == 0.0 && A[2][1] == 0.0;
  if (tril && triu) {
    for (int i = 0; i < 3; ++i) x[i] = b[i] / A[i][i];
    return;
  }
  if (tril) {  // forward substitution, column oriented
    double y0 = b[0], y1 = b[1], y2 = b[2];
    x[0] = y0 / A[0][0];
    y1 = y1 - x[0] * A[1][0];
    y2 = y2 - x[0] * A[2][0];
    x[1] = y1 / A[1][1];
    y2 = y2 - x[1] * A[2][1];
    x[2] = y2 / A[2][2];
    return;
  }
  if (triu) {  // backward substitution, column oriented
    double y0 = b[0], y1 = b[1], y2 = b[2];
    x[2] = y2 / A[2][2];
    y0 = y0 - x[2] * A[0][2];
    y1 = y1 - x[2] * A[1][2];
    x[1] = y1 / A[1][1];
    y0 = y0 - x[1] * A[0][1];
    x[0] = y0 / A[0][0];
    return;
  }
  // LU with partial pivoting (first maximal |pivot|), scaling by the reciprocal pivot.
  int piv[3];
  for (int j = 0; j < 3; ++j) {
    int p = j;
    double pm = std::fabs(A[j][j]);
    for (int i = j + 1; i < 3; ++i) {
      const double v = std::fabs(A[i][j]);
      if (v > pm) { pm = v; p = i; }
    }
    piv[j] = p;
    if (p != j)
      for (int k = 0; k < 3; ++k) std::swap(A[j][k], A[p][k]);
    if (A[j][j] != 0.0) {
      const double r = 1.0 / A[j][j];
      for (int i = j + 1; i < 3; ++i) A[i][j] = A[i][j] * r;
    }
    for (int i = j + 1; i < 3; ++i)
      for (int k = j + 1; k < 3; ++k) A[i][k] = A[i][k] - A[i][j] * A[j][k];
  }
  double y[3] = {b[0], b[1], b[2]};
  for (int j = 0; j < 3; ++j)
    if (piv[j] != j) std::swap(y[j], y[piv[j]]);
  for (int j = 0; j < 3; ++j)
    for (int i = j + 1; i < 3; ++i) y[i] = y[i] - y[j] * A[i][j];
  for (int j = 2; j >= 0; --j) {
    y[j] = y[j] / A[j][j];
    for (int i = 0; i < j; ++i) y[i] = y[i] - y[j] * A[i][j];
  }
  x[0] = y[0]; x[1] = y[1]; x[2] = y[2];
}

void barycentric(const V3& x1, const V3& x2, const V3& x3, const V3& n, const V3& x, double lam[3]) {
  double A[3][3] = {
      {x1.y * n.z - x1.z * n.y, x2.y * n.z - x2.z * n.y, x3.y * n.z - x3.z * n.y},
      {x1.z * n.x - x1.x * n.z, x2.z * n.x - x2.x * n.z, x3.z * n.x - x3.x * n.z},
      {x1.x * n.y - x1.y * n.x, x2.x * n.y - x2.y * n.x, x3.x * n.y - x3.y * n.x}};
  double b[3] = {x.y * n.z - x.z * n.y, x.z * n.x - x.x * n.z, x.x * n.y - x.y * n.x};
  // findmax(abs.(n)): first maximum; a NaN counts as the maximum (first NaN wins).
  const double an[3] = {std::fabs(n.x), std::fabs(n.y), std::fabs(n.z)};
  int imax = 0;
  if (std::isnan(an[0])) imax = 0;
  else if (std::isnan(an[1])) imax = 1;
  else if (std::isnan(an[2])) imax = 2;
  else {
    imax = 0;
    if (an[1] > an[imax]) imax = 1;
    if (an[2] > an[imax]) imax = 2;
  }
  A[imax][0] = A[imax][1] = A[imax][2] = 1.0;
  b[imax] = 1.0;
  solve3(A, b, lam);
}

// ---------------------------------------------------------------------------------------------
// Per-candidate step of the distance loop (dfOnTriangularMesh.jl:101-177).
// quirk = true reproduces the reference (vertices only if no edge foot improved the running min);
// quirk = false evaluates the true point-triangle minimum with the same arithmetic.
// ---------------------------------------------------------------------------------------------
inline void tri_step(const Tri& t, const V3& p, double& m, V3& proj, bool quirk) {
  // point_in_box_range (dfOnTriangularMesh.jl:385-392)
  if (p.x < t.bmin.x - m || p.x > t.bmax.x + m) return;
  if (p.y < t.bmin.y - m || p.y > t.bmax.y + m) return;
  if (p.z < t.bmin.z - m || p.z > t.bmax.z + m) return;
  double lam[3];
  barycentric(t.v[0], t.v[1], t.v[2], t.n, p, lam);
  if (lam[0] >= 0.0 && lam[1] >= 0.0 && lam[2] >= 0.0) {  // minimum(λ) >= 0 (NaN -> false)
    V3 xp = add(add(scale(t.v[0], lam[0]), scale(t.v[1], lam[1])), scale(t.v[2], lam[2]));
    const double d = norm3(sub(p, xp));
    if (d < m) { m = d; proj = xp; }
    return;
  }
  bool improved = false;
  for (int j = 0; j < 3; ++j) {
    const V3 u = divs(t.e[j], t.L[j]);
    const double P = dot3(sub(p, t.v[j]), u);
    if (P >= 0.0 && P <= t.L[j]) {
      const V3 xp = add(t.v[j], scale(u, P));
      const double d = norm3(sub(p, xp));
      if (d < m) { m = d; proj = xp; improved = true; }
    }
  }
  if (!improved || !quirk) {
    const double vd[3] = {norm3(sub(p, t.v[0])), norm3(sub(p, t.v[1])), norm3(sub(p, t.v[2]))};
    if (std::isnan(vd[0]) || std::isnan(vd[1]) || std::isnan(vd[2])) return;  // findmin -> NaN
    int idx = 0;
    if (vd[1] < vd[idx]) idx = 1;
    if (vd[2] < vd[idx]) idx = 2;
    if (vd[idx] < m) { m = vd[idx]; proj = t.v[idx]; }
  }
}

// ---------------------------------------------------------------------------------------------
// Own AABB BVH (broad phase for every query of the oracle).  Boxes are exact coordinate min/max
// expanded by a tiny absolute margin, so ray and ball tests are conservative.
// ---------------------------------------------------------------------------------------------
struct BNode {
  double lo[3], hi[3];
  int64_t left, right;   // children (internal) or -1
  int64_t first, count;  // primitive range in `order` for leaves
};

struct BVH {
  std::vector<BNode> nodes;
  std::vector<int64_t> order;
  double margin = 0.0;
};

void build_bvh(const std::vector<Tri>& T, BVH& bvh) {
  const int64_t n = (int64_t)T.size();
  bvh.order.resize((size_t)n);
  for (int64_t i = 0; i < n; ++i) bvh.order[(size_t)i] = i;
  double ext = 0.0;
  for (const Tri& t : T) {
    ext = std::max(ext, std::max(std::fabs(t.bmin.x), std::fabs(t.bmax.x)));
    ext = std::max(ext, std::max(std::fabs(t.bmin.y), std::fabs(t.bmax.y)));
    ext = std::max(ext, std::max(std::fabs(t.bmin.z), std::fabs(t.bmax.z)));
  }
  bvh.margin = 1e-9 * (ext + 1.0);
  bvh.nodes.clear();
  bvh.nodes.reserve((size_t)(2 * n + 1));
  struct Job { int64_t node, first, count; };
  std::vector<Job> stack;
  bvh.nodes.push_back(BNode{});
  stack.push_back({0, 0, n});
  while (!stack.empty()) {
    Job jb = stack.back();
    stack.pop_back();
    BNode nd{};
    double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
    for (int a = 0; a < 3; ++a) { nd.lo[a] = 1e300; nd.hi[a] = -1e300; }
    for (int64_t i = jb.first; i < jb.first + jb.count; ++i) {
      const Tri& t = T[(size_t)bvh.order[(size_t)i]];
      const double lo[3] = {t.bmin.x, t.bmin.y, t.bmin.z}, hi[3] = {t.bmax.x, t.bmax.y, t.bmax.z};
      const double c[3] = {t.c.x, t.c.y, t.c.z};
      for (int a = 0; a < 3; ++a) {
        nd.lo[a] = std::min(nd.lo[a], lo[a]);
        nd.hi[a] = std::max(nd.hi[a], hi[a]);
        clo[a] = std::min(clo[a], c[a]);
        chi[a] = std::max(chi[a], c[a]);
      }
    }
    for (int a = 0; a < 3; ++a) { nd.lo[a] -= bvh.margin; nd.hi[a] += bvh.margin; }
    nd.left = nd.right = -1;
    nd.first = jb.first;
    nd.count = jb.count;
    if (jb.count > 4) {
      int axis = 0;
      double best = chi[0] - clo[0];
      for (int a = 1; a < 3; ++a)
        if (chi[a] - clo[a] > best) { best = chi[a] - clo[a]; axis = a; }
      const int64_t mid = jb.first + jb.count / 2;
      auto key = [&](int64_t id) {
        const Tri& t = T[(size_t)id];
        return axis == 0 ? t.c.x : (axis == 1 ? t.c.y : t.c.z);
      };
      std::nth_element(bvh.order.begin() + jb.first, bvh.order.begin() + mid,
                       bvh.order.begin() + jb.first + jb.count,
                       [&](int64_t a, int64_t b) {
                         const double ka = key(a), kb = key(b);
                         return ka < kb || (ka == kb && a < b);
                       });
      const int64_t l = (int64_t)bvh.nodes.size();
      bvh.nodes.push_back(BNode{});
      bvh.nodes.push_back(BNode{});
      nd.left = l;
      nd.right = l + 1;
      nd.count = 0;
      stack.push_back({l, jb.first, mid - jb.first});
      stack.push_back({l + 1, mid, jb.first + jb.count - mid});
    }
    bvh.nodes[(size_t)jb.node] = nd;
  }
}

inline double box_dist2(const BNode& b, const V3& p) {
  const double pc[3] = {p.x, p.y, p.z};
  double s = 0.0;
  for (int a = 0; a < 3; ++a) {
    double d = 0.0;
    if (pc[a] < b.lo[a]) d = b.lo[a] - pc[a];
    else if (pc[a] > b.hi[a]) d = pc[a] - b.hi[a];
    s += d * d;
  }
  return s;
}

// Every triangle whose box lies within distance r of p (conservative), appended to out.
void query_ball(const BVH& bvh, const V3& p, double r, std::vector<int64_t>& out) {
  if (bvh.nodes.empty() || bvh.order.empty()) return;
  const double r2 = r * r * (1.0 + 1e-12);
  int64_t st[128];
  int sp = 0;
  st[sp++] = 0;
  while (sp) {
    const BNode& b = bvh.nodes[(size_t)st[--sp]];
    if (box_dist2(b, p) > r2) continue;
    if (b.left < 0) {
      for (int64_t i = b.first; i < b.first + b.count; ++i) out.push_back(bvh.order[(size_t)i]);
    } else {
      st[sp++] = b.left;
      st[sp++] = b.right;
    }
  }
}

inline bool ray_box(const BNode& b, const V3& o, const V3& d) {
  const double oc[3] = {o.x, o.y, o.z}, dc[3] = {d.x, d.y, d.z};
  double t0 = 0.0, t1 = std::numeric_limits<double>::infinity();
  for (int a = 0; a < 3; ++a) {
    if (dc[a] == 0.0) {
      if (oc[a] < b.lo[a] || oc[a] > b.hi[a]) return false;
      continue;
    }
    double ta = (b.lo[a] - oc[a]) / dc[a], tb = (b.hi[a] - oc[a]) / dc[a];
    if (ta > tb) std::swap(ta, tb);
    const double slack = 1e-12 * (std::fabs(ta) + std::fabs(tb) + 1.0);
    t0 = std::max(t0, ta - slack);
    t1 = std::min(t1, tb + slack);
    if (t0 > t1) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------------------------
// Möller–Trumbore (RaycastingSignDetection.jl:64-106).  Returns true and t when the ray hits.
// ---------------------------------------------------------------------------------------------
inline bool ray_triangle(const V3& o, const V3& d, const V3& v1, const V3& v2, const V3& v3,
                         double eps, double& tout) {
  const V3 e1 = sub(v2, v1), e2 = sub(v3, v1);
  const V3 h = cross(d, e2);
  const double a = dot3(e1, h);
  if (std::fabs(a) < eps) return false;
  const double f = 1.0 / a;
  const V3 s = sub(o, v1);
  const double u = f * dot3(s, h);
  if (u < 0.0 || u > 1.0) return false;
  const V3 q = cross(s, e1);
  const double v = f * dot3(d, q);
  if (v < 0.0 || u + v > 1.0) return false;
  const double t = f * dot3(e2, q);
  if (t > eps) { tout = t; return true; }
  return false;
}

// check_ray_inside_bvh (RaycastingSignDetection.jl:114-154): odd count of distinct hits.
bool ray_inside(const BVH& bvh, const std::vector<Tri>& T, const V3& o, const V3& d,
                std::vector<double>& ts) {
  const double eps = 1e-8;
  ts.clear();
  if (bvh.nodes.empty() || bvh.order.empty()) return false;
  int64_t st[128];
  int sp = 0;
  st[sp++] = 0;
  while (sp) {
    const BNode& b = bvh.nodes[(size_t)st[--sp]];
    if (!ray_box(b, o, d)) continue;
    if (b.left < 0) {
      for (int64_t i = b.first; i < b.first + b.count; ++i) {
        const Tri& t = T[(size_t)bvh.order[(size_t)i]];
        double tt;
        if (ray_triangle(o, d, t.v[0], t.v[1], t.v[2], eps, tt) && tt > eps) ts.push_back(tt);
      }
    } else {
      st[sp++] = b.left;
      st[sp++] = b.right;
    }
  }
  if (ts.empty()) return false;
  std::sort(ts.begin(), ts.end());
  int64_t unique = 1;
  for (size_t i = 1; i < ts.size(); ++i)
    if (std::fabs(ts[i] - ts[i - 1]) > eps) ++unique;
  return (unique % 2) == 1;
}

// generate_ray_directions_prioritized (RaycastingSignDetection.jl:162-227).
void ray_directions(double D[36][3]) {
  const double axes[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
  const double face[12][3] = {{1, 1, 0},  {1, -1, 0},  {-1, 1, 0},  {-1, -1, 0},
                              {1, 0, 1},  {1, 0, -1},  {-1, 0, 1},  {-1, 0, -1},
                              {0, 1, 1},  {0, 1, -1},  {0, -1, 1},  {0, -1, -1}};
  const double body[8][3] = {{1, 1, 1},   {1, 1, -1},  {1, -1, 1},  {1, -1, -1},
                             {-1, 1, 1},  {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
  int r = 0;
  auto push_norm = [&](const double* v) {
    V3 u = normalize3({v[0], v[1], v[2]});
    D[r][0] = u.x; D[r][1] = u.y; D[r][2] = u.z;
    ++r;
  };
  for (auto& v : axes) push_norm(v);
  for (auto& v : face) push_norm(v);
  for (auto& v : body) push_norm(v);
  const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
  const double two_pi = 2.0 * 3.14159265358979323846;
  for (int i = 1; i <= 10; ++i) {
    const double x = (double)i * phi;
    const double fr = std::fmod(x, 1.0);  // mod(x, 1.0) for x > 0
    const double theta = two_pi * fr;
    const double z = 1.0 - 2.0 * ((double)i / 10.0);
    const double rr = std::sqrt(1.0 - z * z);
    D[r][0] = rr * std::cos(theta);
    D[r][1] = rr * std::sin(theta);
    D[r][2] = z;
    ++r;
  }
}

// generalized_winding_number (RaycastingSignDetection.jl:295-328).
double winding_sign(const std::vector<Tri>& T, const V3& p, double* wout) {
  double w = 0.0;
  for (const Tri& t : T) {
    const V3 a = normalize3(sub(t.v[0], p));
    const V3 b = normalize3(sub(t.v[1], p));
    const V3 c = normalize3(sub(t.v[2], p));
    const double num = dot3(a, cross(b, c));
    const double den = ((1.0 + dot3(a, b)) + dot3(b, c)) + dot3(c, a);
    if (std::fabs(den) > 1e-10) {
      double sa = 2.0 * std::atan2(std::fabs(num), den);
      if (num < 0) sa = -sa;
      w += sa;
    }
  }
  w = w / (4.0 * 3.14159265358979323846);
  if (wout) *wout = w;
  return std::fabs(w) > 0.5 ? 1.0 : -1.0;
}

struct Mesh {
  const double* X;
  int64_t nnp;
  const int64_t* IEN;
  int64_t nel;
  std::vector<Tri> T;
  BVH bvh;
  std::vector<std::vector<int64_t>> INE;  // node -> elements (MeshInformations.jl:39-54)
};

void mesh_init(Mesh& M, const double* X, int64_t nnp, const int64_t* IEN, int64_t nel) {
  M.X = X; M.nnp = nnp; M.IEN = IEN; M.nel = nel;
  M.T = prepare_triangles(X, nnp, IEN, nel);
  build_bvh(M.T, M.bvh);
  M.INE.assign((size_t)nnp, {});
  for (int64_t el = 0; el < nel; ++el)
    for (int k = 0; k < 3; ++k) M.INE[(size_t)(IEN[3 * el + k] - 1)].push_back(el);
}

// knn(vtx_kdtree, p, 3): the 3 nearest vertices by squared distance, ties to the lower index.
void knn3(const Mesh& M, const V3& p, double r0, int64_t out[3], int& nout) {
  // Grow a ball query over triangle boxes (which contain every vertex) until 3 vertices are
  // certified nearest.
  double r = r0 > 0.0 ? r0 : 1e-6;
  std::vector<int64_t> cand;
  while (true) {
    cand.clear();
    query_ball(M.bvh, p, r, cand);
    std::vector<std::pair<double, int64_t>> vs;
    for (int64_t el : cand)
      for (int k = 0; k < 3; ++k) {
        const int64_t vi = M.IEN[3 * el + k] - 1;
        const double dx = M.X[3 * vi] - p.x, dy = M.X[3 * vi + 1] - p.y, dz = M.X[3 * vi + 2] - p.z;
        double s = dx * dx;
        s = s + dy * dy;
        s = s + dz * dz;
        vs.push_back({s, vi});
      }
    std::sort(vs.begin(), vs.end());
    vs.erase(std::unique(vs.begin(), vs.end()), vs.end());
    const int64_t need = std::min<int64_t>(3, M.nnp);
    if ((int64_t)vs.size() >= need && vs[(size_t)need - 1].first <= r * r * (1.0 - 1e-12)) {
      nout = (int)need;
      for (int i = 0; i < nout; ++i) out[i] = vs[(size_t)i].second;
      return;
    }
    if ((int64_t)cand.size() == M.nel) {  // whole mesh already in the ball
      nout = (int)std::min<int64_t>(need, (int64_t)vs.size());
      for (int i = 0; i < nout; ++i) out[i] = vs[(size_t)i].second;
      return;
    }
    r *= 2.0;
  }
}

enum { MODE_REF_RULE = 0, MODE_EXACT = 1, MODE_UNBOUNDED = 2 };

// One node of evalDistancesOnTriMesh.  Returns the merged, un-clamped running minimum (1e10 when
// nothing improved it) and the projection.  flags: bit0 = candidate set C(p) was empty (knn
// fallback used), bit1 = result depends on the candidate order (ref-rule differs from the exact
// minimum over the same candidates).
double eval_node(const Mesh& M, const Grid& g, const V3& p, int mode, V3& proj, int& flags,
                 std::vector<int64_t>& cand) {
  flags = 0;
  double m = std::fabs(-1.0e10);
  proj = {0.0, 0.0, 0.0};
  cand.clear();
  if (mode == MODE_REF_RULE) {
    // tri_indices = inrange(tri_kdtree, p, 2.5h)  (dfOnTriangularMesh.jl:48,79)
    const double sr = 2.5 * g.h;
    const double r2 = sr * sr;
    std::vector<int64_t> boxc;
    query_ball(M.bvh, p, sr, boxc);
    for (int64_t el : boxc) {
      const Tri& t = M.T[(size_t)el];
      const double dx = t.c.x - p.x, dy = t.c.y - p.y, dz = t.c.z - p.z;
      double s = dx * dx;
      s = s + dy * dy;
      s = s + dz * dz;
      if (s <= r2) cand.push_back(el);
    }
    if (cand.empty()) {  // knn fallback (dfOnTriangularMesh.jl:82-94)
      flags |= 1;
      int64_t nn[3];
      int k = 0;
      knn3(M, p, 2.0 * g.h, nn, k);
      for (int i = 0; i < k; ++i)
        for (int64_t el : M.INE[(size_t)nn[i]]) cand.push_back(el);
    }
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    for (int64_t el : cand) tri_step(M.T[(size_t)el], p, m, proj, true);
    // Order sensitivity: compare with the true minimum over the same candidates.
    double me = std::fabs(-1.0e10);
    V3 pe{0, 0, 0};
    for (int64_t el : cand) tri_step(M.T[(size_t)el], p, me, pe, false);
    const double hclamp = g.h;
    if (std::min(m, hclamp) != std::min(me, hclamp)) flags |= 2;
    return m;
  }
  if (mode == MODE_EXACT) {
    // True minimum over every triangle within reach of the clamp; clamped by the caller.
    query_ball(M.bvh, p, g.h, cand);
    std::sort(cand.begin(), cand.end());
    for (int64_t el : cand) tri_step(M.T[(size_t)el], p, m, proj, false);
    return m;
  }
  // MODE_UNBOUNDED: the true minimum over every triangle (no clamp).  Grow a ball query.
  double r = g.h;
  while (true) {
    cand.clear();
    query_ball(M.bvh, p, r, cand);
    std::sort(cand.begin(), cand.end());
    double mm = std::fabs(-1.0e10);
    V3 pp{0, 0, 0};
    for (int64_t el : cand) tri_step(M.T[(size_t)el], p, mm, pp, false);
    if (mm <= r || (int64_t)cand.size() == M.nel) {
      proj = pp;
      return mm;
    }
    r *= 2.0;
  }
}

// adaptive_point_in_mesh_raycast (RaycastingSignDetection.jl:234-288) + the winding fallback of
// raycast_sign_detection (:376-380).  stats[0] += rays cast, stats[1] += winding fallbacks.
void sign_node(const Mesh& M, const V3& p, const double D[36][3], int min_rays, int max_rays,
               double conf_thresh, int use_winding, double& sign, double& conf, int64_t* rays_out,
               int* fb_out, double* w_out, std::vector<double>& ts) {
  int inside = 0, total = 0;
  for (int i = 0; i < min_rays; ++i) {
    const V3 d{D[i][0], D[i][1], D[i][2]};
    if (ray_inside(M.bvh, M.T, p, d, ts)) ++inside;
    ++total;
  }
  double ratio = (double)inside / (double)total;
  double c = std::max(ratio, 1.0 - ratio);
  int used = min_rays;
  while (c < 0.85 && used < max_rays) {
    const int batch = std::min(4, max_rays - used);
    for (int i = used + 1; i <= used + batch; ++i) {
      if (i <= 36) {
        const V3 d{D[i - 1][0], D[i - 1][1], D[i - 1][2]};
        if (ray_inside(M.bvh, M.T, p, d, ts)) ++inside;
        ++total;
      }
    }
    used += batch;
    ratio = (double)inside / (double)total;
    c = std::max(ratio, 1.0 - ratio);
    if (c > 0.95) break;
  }
  double s = ratio > 0.5 ? 1.0 : -1.0;
  *fb_out = 0;
  *w_out = 0.0;
  if (use_winding && c < conf_thresh) {
    s = winding_sign(M.T, p, w_out);
    c = 0.8;
    *fb_out = 1;
  }
  *rays_out = total;
  sign = s;
  conf = c;
}

bool grid_from(const double* origin, double h, const int64_t* N, Grid& g) {
  for (int a = 0; a < 3; ++a) {
    g.origin[a] = origin[a];
    g.N[a] = N[a];
    if (N[a] < 0) return false;
    g.amax[a] = origin[a] + (double)N[a] * h;
  }
  g.h = h;
  g.ngp = (N[0] + 1) * (N[1] + 1) * (N[2] + 1);
  return h > 0.0 && std::isfinite(h);
}

int nthreads_for(int requested) {
#ifdef _OPENMP
  return requested > 0 ? requested : omp_get_max_threads();
#else
  (void)requested;
  return 1;
#endif
}

}  // namespace

extern "C" {

// Grid constructor (Grid.jl:9-32).  Returns 0 on success.
int oracle_grid(const double xmin[3], const double xmax[3], int64_t n_max, int64_t margin,
                double origin[3], double amax[3], int64_t N[3], double* h, int64_t* ngp) {
  if (n_max <= 0) return 1;
  // maximum(AABB_max .- AABB_min)
  double ext = xmax[0] - xmin[0];
  for (int a = 1; a < 3; ++a) ext = std::max(ext, xmax[a] - xmin[a]);
  if (!std::isfinite(ext) || !(ext > 0.0)) return 1;
  const double cs = ext / (double)n_max;
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = xmin[a] - (double)margin * cs;
    hi[a] = xmax[a] + (double)margin * cs;
  }
  int64_t prod = 1;
  for (int a = 0; a < 3; ++a) {
    const double q = std::ceil((hi[a] - lo[a]) / cs);
    if (!std::isfinite(q) || q < 0 || q > 9.0e15) return 2;
    N[a] = (int64_t)q;
    origin[a] = lo[a];
    amax[a] = lo[a] + (double)N[a] * cs;
    prod *= (N[a] + 1);
  }
  *h = cs;
  *ngp = prod;
  return 0;
}

// noninteractive_sdf_grid_setup (Grid_setup.jl:104-124): N_new = floor(maxext / B), margin 3.
int oracle_grid_from_cell_size(const double* X, int64_t nnp, double B, double origin[3],
                               double amax[3], int64_t N[3], double* h, int64_t* ngp) {
  if (nnp <= 0 || !(B > 0.0)) return 1;
  double xmin[3] = {X[0], X[1], X[2]}, xmax[3] = {X[0], X[1], X[2]};
  for (int64_t v = 1; v < nnp; ++v)
    for (int a = 0; a < 3; ++a) {
      xmin[a] = std::min(xmin[a], X[3 * v + a]);
      xmax[a] = std::max(xmax[a], X[3 * v + a]);
    }
  double ext = xmax[0] - xmin[0];
  for (int a = 1; a < 3; ++a) ext = std::max(ext, xmax[a] - xmin[a]);
  const double q = std::floor(ext / B);
  if (!std::isfinite(q) || q < 1) return 2;
  return oracle_grid(xmin, xmax, (int64_t)q, 3, origin, amax, N, h, ngp);
}

// evalDistancesOnTriMesh over the implicit grid (origin, h, N), or over the nodes listed in
// `nodes` (linear indices, x fastest) when nodes != NULL.  dist_out/xp_out/flags_out have one
// entry (three for xp) per evaluated node.  mode: 0 ref-rule, 1 exact (clamped), 2 unbounded.
int oracle_distances(const double* X, int64_t nnp, const int64_t* IEN, int64_t nel,
                     const double origin[3], double h, const int64_t N[3], int mode,
                     const int64_t* nodes, int64_t nnodes, double* dist_out, double* xp_out,
                     int32_t* flags_out, int nthreads) {
  if (nel <= 0 || nnp <= 0) return 1;
  Grid g;
  if (!grid_from(origin, h, N, g)) return 1;
  Mesh M;
  mesh_init(M, X, nnp, IEN, nel);
  const int64_t count = nodes ? nnodes : g.ngp;
  const int nt = nthreads_for(nthreads);
#pragma omp parallel num_threads(nt)
  {
    std::vector<int64_t> cand;
#pragma omp for schedule(dynamic, 128)
    for (int64_t q = 0; q < count; ++q) {
      const int64_t lin = nodes ? nodes[q] : q;
      const V3 p = node_coord(g, lin);
      V3 proj;
      int fl = 0;
      double m = eval_node(M, g, p, mode, proj, fl, cand);
      // Thread merge keeps the minimum (dfOnTriangularMesh.jl:195-199); the clamp
      // (:202-206) sets |d| > cell_size to cell_size.
      if (mode != MODE_UNBOUNDED && std::fabs(m) > std::fabs(g.h)) m = (m > 0 ? 1.0 : -1.0) * g.h;
      dist_out[q] = m;
      if (xp_out) { xp_out[3 * q] = proj.x; xp_out[3 * q + 1] = proj.y; xp_out[3 * q + 2] = proj.z; }
      if (flags_out) flags_out[q] = fl;
    }
  }
  return 0;
}

// raycast_sign_detection over the grid or a node list.  rays_out (optional) receives the number
// of rays cast per node, fb_out (optional) 1 where the winding fallback ran, w_out (optional) the
// winding number of those nodes.
int oracle_signs(const double* X, int64_t nnp, const int64_t* IEN, int64_t nel,
                 const double origin[3], double h, const int64_t N[3], int min_rays, int max_rays,
                 double conf_thresh, int use_winding, const int64_t* nodes, int64_t nnodes,
                 double* sign_out, double* conf_out, int32_t* rays_out, int32_t* fb_out,
                 double* w_out, int nthreads) {
  if (nel <= 0 || nnp <= 0) return 1;
  if (min_rays < 1 || min_rays > 36 || max_rays < 1) return 1;
  Grid g;
  if (!grid_from(origin, h, N, g)) return 1;
  Mesh M;
  mesh_init(M, X, nnp, IEN, nel);
  double D[36][3];
  ray_directions(D);
  const int64_t count = nodes ? nnodes : g.ngp;
  const int nt = nthreads_for(nthreads);
#pragma omp parallel num_threads(nt)
  {
    std::vector<double> ts;
#pragma omp for schedule(dynamic, 64)
    for (int64_t q = 0; q < count; ++q) {
      const int64_t lin = nodes ? nodes[q] : q;
      const V3 p = node_coord(g, lin);
      double s, c, w;
      int64_t rays;
      int fb;
      sign_node(M, p, D, min_rays, max_rays, conf_thresh, use_winding, s, c, &rays, &fb, &w, ts);
      sign_out[q] = s;
      if (conf_out) conf_out[q] = c;
      if (rays_out) rays_out[q] = (int32_t)rays;
      if (fb_out) fb_out[q] = fb;
      if (w_out) w_out[q] = w;
    }
  }
  return 0;
}

// The 36 prioritized ray directions (RaycastingSignDetection.jl:162-227), 36x3 row major.
void oracle_ray_directions(double* out) {
  double D[36][3];
  ray_directions(D);
  std::memcpy(out, D, sizeof(D));
}

// Single Möller–Trumbore evaluation (for known-answer tests).  Returns 1 on hit.
int oracle_ray_triangle(const double o[3], const double d[3], const double v1[3],
                        const double v2[3], const double v3[3], double eps, double* t) {
  double tt = 0.0;
  const bool hit = ray_triangle({o[0], o[1], o[2]}, {d[0], d[1], d[2]}, {v1[0], v1[1], v1[2]},
                                {v2[0], v2[1], v2[2]}, {v3[0], v3[1], v3[2]}, eps, tt);
  *t = hit ? tt : 0.0;
  return hit ? 1 : 0;
}

// Barycentric coordinates of the projection (dfOnTriangularMesh.jl:226-251).
void oracle_barycentric(const double x1[3], const double x2[3], const double x3[3],
                        const double n[3], const double x[3], double lam[3]) {
  barycentric({x1[0], x1[1], x1[2]}, {x2[0], x2[1], x2[2]}, {x3[0], x3[1], x3[2]},
              {n[0], n[1], n[2]}, {x[0], x[1], x[2]}, lam);
}

// Generalized winding number at arbitrary points (RaycastingSignDetection.jl:295-328).
int oracle_winding(const double* X, int64_t nnp, const int64_t* IEN, int64_t nel, const double* pts,
                   int64_t npts, double* sign_out, double* w_out, int nthreads) {
  if (nel <= 0) return 1;
  std::vector<Tri> T = prepare_triangles(X, nnp, IEN, nel);
  const int nt = nthreads_for(nthreads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16)
  for (int64_t q = 0; q < npts; ++q) {
    double w;
    sign_out[q] = winding_sign(T, {pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]}, &w);
    if (w_out) w_out[q] = w;
  }
  return 0;
}

// Algorithmic work of the hot path at each listed node, independent of any implementation (the
// roofline's work model):
//   nD[q]      = |D*(p)|, triangles whose AABB lies within min(d_true(p), h) of p -- the
//                candidates no box-pruned nearest search can skip (d_true: the unbounded minimum);
//   nrow[3q+a] = triangles whose AABB meets the grid line through p along axis a (the +a and -a
//                rays of every node of that row share them);
//   nextra[q]  = triangles whose AABB the rays beyond the six axis rays hit (rays the reference's
//                adaptive vote casts at p, RaycastingSignDetection.jl:234-288);
//   rays[q]    = rays the vote casts at p.
int oracle_work_model(const double* X, int64_t nnp, const int64_t* IEN, int64_t nel,
                      const double origin[3], double h, const int64_t N[3], const int64_t* nodes,
                      int64_t nnodes, int64_t* nD, int64_t* nrow, int64_t* nextra, int32_t* rays,
                      int64_t* nD_unb, int nthreads) {
  if (nel <= 0 || nnp <= 0 || !nodes) return 1;
  Grid g;
  if (!grid_from(origin, h, N, g)) return 1;
  Mesh M;
  mesh_init(M, X, nnp, IEN, nel);
  double D[36][3];
  ray_directions(D);
  const int nt = nthreads_for(nthreads);
#pragma omp parallel num_threads(nt)
  {
    std::vector<int64_t> cand;
    std::vector<double> ts;
#pragma omp for schedule(dynamic, 64)
    for (int64_t q = 0; q < nnodes; ++q) {
      const V3 p = node_coord(g, nodes[q]);
      V3 proj;
      int fl = 0;
      const double dt = eval_node(M, g, p, MODE_UNBOUNDED, proj, fl, cand);
      // triangles whose AABB lies within radius r of p
      auto count_within = [&](double r) {
        cand.clear();
        query_ball(M.bvh, p, r, cand);
        int64_t c = 0;
        for (int64_t el : cand) {
          const Tri& t = M.T[(size_t)el];
          const double lo[3] = {t.bmin.x, t.bmin.y, t.bmin.z}, hi[3] = {t.bmax.x, t.bmax.y, t.bmax.z};
          const double pc[3] = {p.x, p.y, p.z};
          double s2 = 0.0;
          for (int a = 0; a < 3; ++a) {
            const double dd = pc[a] < lo[a] ? lo[a] - pc[a] : (pc[a] > hi[a] ? pc[a] - hi[a] : 0.0);
            s2 += dd * dd;
          }
          if (s2 <= r * r) ++c;
        }
        return c;
      };
      nD[q] = count_within(std::min(dt, g.h));
      // the unclamped form: every triangle a box-pruned search for the true minimum must look at
      if (nD_unb) nD_unb[q] = dt <= g.h ? nD[q] : count_within(dt);
      // grid lines: both coordinates other than a inside the triangle's box
      const double pc[3] = {p.x, p.y, p.z};
      for (int a = 0; a < 3; ++a) {
        const int b = (a + 1) % 3, e = (a + 2) % 3;
        int64_t cnt = 0;
        int64_t st[128];
        int sp = 0;
        st[sp++] = 0;
        while (sp) {
          const BNode& nd = M.bvh.nodes[(size_t)st[--sp]];
          if (pc[b] < nd.lo[b] || pc[b] > nd.hi[b] || pc[e] < nd.lo[e] || pc[e] > nd.hi[e]) continue;
          if (nd.left < 0) {
            for (int64_t i = nd.first; i < nd.first + nd.count; ++i) {
              const Tri& t = M.T[(size_t)M.bvh.order[(size_t)i]];
              const double lo[3] = {t.bmin.x, t.bmin.y, t.bmin.z}, hi[3] = {t.bmax.x, t.bmax.y, t.bmax.z};
              if (pc[b] >= lo[b] && pc[b] <= hi[b] && pc[e] >= lo[e] && pc[e] <= hi[e]) ++cnt;
            }
          } else {
            st[sp++] = nd.left;
            st[sp++] = nd.right;
          }
        }
        nrow[3 * q + a] = cnt;
      }
      double sg, cf, w;
      int64_t nr;
      int fb;
      sign_node(M, p, D, 6, 30, 0.6, 1, sg, cf, &nr, &fb, &w, ts);
      rays[q] = (int32_t)nr;
      int64_t ex = 0;
      for (int64_t rr = 6; rr < nr && rr < 36; ++rr) {
        const V3 d{D[rr][0], D[rr][1], D[rr][2]};
        for (const Tri& t : M.T) {
          BNode bb{};
          bb.lo[0] = t.bmin.x; bb.lo[1] = t.bmin.y; bb.lo[2] = t.bmin.z;
          bb.hi[0] = t.bmax.x; bb.hi[1] = t.bmax.y; bb.hi[2] = t.bmax.z;
          if (ray_box(bb, p, d)) ++ex;
        }
      }
      nextra[q] = ex;
    }
  }
  return 0;
}

int oracle_max_threads(void) { return nthreads_for(0); }

}  // extern "C"
