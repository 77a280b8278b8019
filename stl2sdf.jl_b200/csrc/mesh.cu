// mesh.cu -- TriangularMesh upload, per-triangle preparation and the LBVH build.
//
// Reference: TriangularMesh (src/MeshGrid/MeshInformations.jl:57-84), prepare_triangle_data
// (src/SignedDistances/dfOnTriangularMesh.jl:329-368) and the two acceleration structures the
// reference builds per call (KD-trees at dfOnTriangularMesh.jl:27,35; ImplicitBVH at
// RaycastingSignDetection.jl:35-56).  Here one LBVH over triangle boxes serves every query that
// is not grid-structured: arbitrary-direction rays, the 3-nearest-vertex fallback and the
// unbounded nearest-triangle search.
//
// LBVH (Karras 2012, "Maximizing parallelism in the construction of BVHs, octrees, and k-d
// trees"): 30-bit Morton codes of the triangle centroids with the triangle index in the low 32
// bits (unique 64-bit keys), a CUB radix sort, one thread per internal node to find its range
// and split, then a bottom-up refit with one atomic counter per internal node.
#include <cub/cub.cuh>

#include "common.cuh"

namespace sdfgpu {

namespace {

__global__ void k_vertex_bbox(const double* __restrict__ X, int64_t nnp, unsigned long long* bb) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  bool nonfinite = false;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nnp; v += (int64_t)gridDim.x * blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      const double x = X[3 * v + a];
      if (!isfinite(x)) nonfinite = true;
      lo[a] = fmin(lo[a], x);
      hi[a] = fmax(hi[a], x);
    }
  }
  for (int a = 0; a < 3; ++a) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[a] = fmin(lo[a], __shfl_down_sync(0xffffffffu, lo[a], off));
      hi[a] = fmax(hi[a], __shfl_down_sync(0xffffffffu, hi[a], off));
    }
  }
  const unsigned nf = __ballot_sync(0xffffffffu, nonfinite);
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(&bb[a], dbl_ord(lo[a]));
      atomicMax(&bb[3 + a], dbl_ord(hi[a]));
    }
    if (nf) atomicOr(&bb[6], 1ULL);
  }
}

// Per-triangle FP64 record (dfOnTriangularMesh.jl:329-368) and the barycentric factorization.
__global__ void k_prep(const double* __restrict__ X, int64_t nnp, const int64_t* __restrict__ IEN, int64_t nel,
                       TriRec64* __restrict__ rec, double4* __restrict__ cent, int64_t* counters) {
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    TriRec64 r;
    d3 v[3];
    for (int k = 0; k < 3; ++k) {
      int64_t vi = IEN[3 * el + k];
      if (vi < 1 || vi > nnp) {
        count_add(counters, C_ERR_INDEX, 1);
        vi = 1;
      }
      vi -= 1;
      v[k] = {X[3 * vi], X[3 * vi + 1], X[3 * vi + 2]};
      r.v[3 * k] = v[k].x; r.v[3 * k + 1] = v[k].y; r.v[3 * k + 2] = v[k].z;
    }
    const d3 e[3] = {v_sub(v[1], v[0]), v_sub(v[2], v[1]), v_sub(v[0], v[2])};
    for (int j = 0; j < 3; ++j) {
      r.L[j] = v_norm(e[j]);
      const d3 u = v_div(e[j], r.L[j]);
      r.u[3 * j] = u.x; r.u[3 * j + 1] = u.y; r.u[3 * j + 2] = u.z;
    }
    const d3 nn = v_cross(e[0], v_neg(e[2]));
    const d3 n = v_div(nn, v_norm(nn));
    r.n[0] = n.x; r.n[1] = n.y; r.n[2] = n.z;
    const d3 c = v_div(v_add(v_add(v[0], v[1]), v[2]), 3.0);
    r.bmin[0] = fmin(v[0].x, fmin(v[1].x, v[2].x));
    r.bmin[1] = fmin(v[0].y, fmin(v[1].y, v[2].y));
    r.bmin[2] = fmin(v[0].z, fmin(v[1].z, v[2].z));
    r.bmax[0] = fmax(v[0].x, fmax(v[1].x, v[2].x));
    r.bmax[1] = fmax(v[0].y, fmax(v[1].y, v[2].y));
    r.bmax[2] = fmax(v[0].z, fmax(v[1].z, v[2].z));
    r.pad = 0;
    factor_bary(r);
    rec[el] = r;
    cent[el] = make_double4(c.x, c.y, c.z, 0.0);
  }
}

// Mesh-local FP32 copies: vertices, centroid, outward-rounded box; and rho = max vertex
// distance from the centroid (decides whether the centroid rule can miss a triangle within h).
// v32[3*el+k].w carries the global (0-based) index of vertex k; c32[el].w is 1 when the triangle
// is well conditioned for FP32 decisions (no edge shorter than 1e-5 E, sine of the smallest
// angle above ~1e-3, distinct vertices) and 0 when every decision on it must be made in FP64.
__global__ void k_local32(const TriRec64* __restrict__ rec, const double4* __restrict__ cent,
                          const int64_t* __restrict__ IEN, int64_t nel, double cx, double cy, double cz, double E,
                          float4* __restrict__ v32, float4* __restrict__ c32, float4* __restrict__ box32,
                          unsigned long long* rho_ord) {
  double rho = 0.0;
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    const TriRec64& r = rec[el];
    const double4 c = cent[el];
    int32_t gid[3];
    for (int k = 0; k < 3; ++k) {
      gid[k] = (int32_t)(IEN[3 * el + k] - 1);
      const double x = r.v[3 * k], y = r.v[3 * k + 1], z = r.v[3 * k + 2];
      v32[3 * el + k] = make_float4((float)(x - cx), (float)(y - cy), (float)(z - cz), __int_as_float(gid[k]));
      const double dx = x - c.x, dy = y - c.y, dz = z - c.z;
      rho = fmax(rho, sqrt(dx * dx + dy * dy + dz * dz));
    }
    double L[3], lmin = 1e300, lmax = 0.0;
    for (int j = 0; j < 3; ++j) {
      const int a = j, b = (j + 1) % 3;
      const double ex = r.v[3 * b] - r.v[3 * a], ey = r.v[3 * b + 1] - r.v[3 * a + 1], ez = r.v[3 * b + 2] - r.v[3 * a + 2];
      L[j] = sqrt(ex * ex + ey * ey + ez * ez);
      lmin = fmin(lmin, L[j]);
      lmax = fmax(lmax, L[j]);
    }
    const double ax = r.v[3] - r.v[0], ay = r.v[4] - r.v[1], az = r.v[5] - r.v[2];
    const double bx = r.v[6] - r.v[0], by = r.v[7] - r.v[1], bz = r.v[8] - r.v[2];
    const double nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
    const double nn = sqrt(nx * nx + ny * ny + nz * nz);
    const bool ok = lmin > 1e-5 * E && nn > 1e-3 * lmax * lmax && gid[0] != gid[1] && gid[1] != gid[2] &&
                    gid[0] != gid[2];
    c32[el] = make_float4((float)(c.x - cx), (float)(c.y - cy), (float)(c.z - cz), ok ? 1.f : 0.f);
    box32[2 * el] = make_float4(__double2float_rd(r.bmin[0] - cx), __double2float_rd(r.bmin[1] - cy),
                                __double2float_rd(r.bmin[2] - cz), 0.f);
    box32[2 * el + 1] = make_float4(__double2float_ru(r.bmax[0] - cx), __double2float_ru(r.bmax[1] - cy),
                                    __double2float_ru(r.bmax[2] - cz), 0.f);
  }
  for (int off = 16; off > 0; off >>= 1) rho = fmax(rho, __shfl_down_sync(0xffffffffu, rho, off));
  if ((threadIdx.x & 31) == 0) atomicMax(rho_ord, dbl_ord(rho * (1.0 + 1e-12)));
}

__device__ __forceinline__ unsigned expand_bits10(unsigned v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

// 30-bit Morton code of each centroid and the triangle index; a stable sort of the codes (index as
// the value) orders the triangles exactly as the unique 64-bit keys (code << 32 | index) would, in
// half the radix passes.
__global__ void k_morton(const float4* __restrict__ c32, int64_t nel, float lox, float loy, float loz, float inv,
                         uint32_t* __restrict__ code, int32_t* __restrict__ idx) {
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x) {
    const float4 c = c32[el];
    const float fx = fminf(fmaxf((c.x - lox) * inv, 0.f), 1023.f);
    const float fy = fminf(fmaxf((c.y - loy) * inv, 0.f), 1023.f);
    const float fz = fminf(fmaxf((c.z - loz) * inv, 0.f), 1023.f);
    code[el] = (expand_bits10((unsigned)fx) << 2) | (expand_bits10((unsigned)fy) << 1) | expand_bits10((unsigned)fz);
    idx[el] = (int32_t)el;
  }
}

// The sorted unique keys (code << 32 | index) the hierarchy build splits on.
__global__ void k_pack_keys(const uint32_t* __restrict__ code, const int32_t* __restrict__ idx, int n,
                            unsigned long long* __restrict__ keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keys[i] = ((unsigned long long)code[i] << 32) | (unsigned long long)(uint32_t)idx[i];
}

__device__ __forceinline__ int kdelta(const unsigned long long* __restrict__ k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  return __clzll(k[i] ^ k[j]);
}

__global__ void k_karras(const unsigned long long* __restrict__ keys, int n, BNode* __restrict__ nodes,
                         int32_t* __restrict__ int_parent, int32_t* __restrict__ leaf_parent) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
    const int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
      if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(keys, n, i, j);
    int s = 0, t = l;
    while (true) {
      t = (t + 1) >> 1;
      if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
      if (t <= 1) break;
    }
    const int gamma = i + s * d + (d < 0 ? -1 : 0);
    const int lo = min(i, j), hi = max(i, j);
    int left, right;
    if (lo == gamma) { left = kLeafBit | gamma; leaf_parent[gamma] = i; }
    else { left = gamma; int_parent[gamma] = i; }
    if (hi == gamma + 1) { right = kLeafBit | (gamma + 1); leaf_parent[gamma + 1] = i; }
    else { right = gamma + 1; int_parent[gamma + 1] = i; }
    // d.z, d.w: the node's range of sorted leaves [lo, hi]; its left child covers [lo, gamma] and its
    // right child [gamma + 1, hi], so a parent tells the size of both children's subtrees.
    nodes[i].d = make_int4(left, right, lo, hi);
  }
}

__global__ void k_refit(const unsigned long long* __restrict__ keys, const float4* __restrict__ box32, int n,
                        BNode* nodes, const int32_t* __restrict__ int_parent, const int32_t* __restrict__ leaf_parent,
                        int32_t* flags, int32_t* __restrict__ leaf_prim) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int prim = (int)(keys[i] & 0xffffffffULL);
    leaf_prim[i] = prim;
    float4 lo = box32[2 * prim], hi = box32[2 * prim + 1];
    int child = kLeafBit | i;
    int node = leaf_parent[i];
    int guard = 0;
    while (node >= 0 && ++guard <= 128) {  // LBVH depth <= 64 for unique 64-bit keys
      float* f = reinterpret_cast<float*>(&nodes[node]);
      const int left = __ldcg(reinterpret_cast<const int*>(&nodes[node].d.x));
      const int slot = (left == child) ? 0 : 6;
      __stcg(f + slot + 0, lo.x); __stcg(f + slot + 1, lo.y); __stcg(f + slot + 2, lo.z);
      __stcg(f + slot + 3, hi.x); __stcg(f + slot + 4, hi.y); __stcg(f + slot + 5, hi.z);
      __threadfence();
      if (atomicAdd(&flags[node], 1) == 0) break;
      __threadfence();
      float b[12];
      for (int q = 0; q < 12; ++q) b[q] = __ldcg(f + q);
      lo = make_float4(fminf(b[0], b[6]), fminf(b[1], b[7]), fminf(b[2], b[8]), 0.f);
      hi = make_float4(fmaxf(b[3], b[9]), fmaxf(b[4], b[10]), fmaxf(b[5], b[11]), 0.f);
      child = node;
      node = int_parent[node];
    }
  }
}

// A single-triangle mesh: root with the leaf on the left and an empty box on the right.
__global__ void k_single_root(const float4* __restrict__ box32, BNode* nodes, int32_t* leaf_prim) {
  const float4 lo = box32[0], hi = box32[1];
  BNode nd;
  nd.a = make_float4(lo.x, lo.y, lo.z, hi.x);
  nd.b = make_float4(hi.y, hi.z, 3.0e38f, 3.0e38f);
  nd.c = make_float4(3.0e38f, -3.0e38f, -3.0e38f, -3.0e38f);
  nd.d = make_int4(kLeafBit | 0, kLeafBit | 0, 0, 0);
  nodes[0] = nd;
  leaf_prim[0] = 0;
}

// Leaf-ordered copies for the unbounded searches and the oriented-box fit, which read the
// triangles of runs of consecutive leaves: the FP32 vertices (3 x float4, as v32) and the LeafTri
// record, both of the triangle at each sorted leaf.  The record's fields are computed in FP64 from
// the triangle's vertices (mesh-local) and rounded once.
__global__ void k_leaf_order(const int32_t* __restrict__ leaf_prim, const float4* __restrict__ v32,
                             const TriRec64* __restrict__ rec, int n, double cx, double cy, double cz,
                             float4* __restrict__ lv32, LeafTri* __restrict__ ltri) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int prim = leaf_prim[i];
    lv32[3 * i] = v32[3 * prim];
    lv32[3 * i + 1] = v32[3 * prim + 1];
    lv32[3 * i + 2] = v32[3 * prim + 2];
    const double* v = rec[prim].v;
    const double ax = v[0] - cx, ay = v[1] - cy, az = v[2] - cz;
    const double e0[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
    const double e1[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
    const double e2[3] = {v[6] - v[3], v[7] - v[4], v[8] - v[5]};
    const double l0 = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
    const double l1 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const double l2 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const double nx = e0[1] * e1[2] - e0[2] * e1[1], ny = e0[2] * e1[0] - e0[0] * e1[2], nz = e0[0] * e1[1] - e0[1] * e1[0];
    const double nn = nx * nx + ny * ny + nz * nz;
    LeafTri T;
    T.a = make_float4((float)ax, (float)ay, (float)az, (float)(1.0 / l0));
    T.e0 = make_float4((float)e0[0], (float)e0[1], (float)e0[2], (float)(1.0 / l1));
    T.e1 = make_float4((float)e1[0], (float)e1[1], (float)e1[2], (float)(1.0 / l2));
    if (nn > 1e-20 * l0 * l1) {
      const double rn = 1.0 / sqrt(nn), un[3] = {nx * rn, ny * rn, nz * rn};
      // inward in-plane edge normals: n x (edge direction), edges a->b, b->c, c->a
      const double* ed[3] = {e0, e2, e1};
      const double sg[3] = {1.0, 1.0, -1.0};
      double m[3][3];
      for (int k = 0; k < 3; ++k) {
        const double* d = ed[k];
        const double mx = sg[k] * (un[1] * d[2] - un[2] * d[1]), my = sg[k] * (un[2] * d[0] - un[0] * d[2]),
                     mz = sg[k] * (un[0] * d[1] - un[1] * d[0]);
        const double r = 1.0 / sqrt(mx * mx + my * my + mz * mz);
        m[k][0] = mx * r; m[k][1] = my * r; m[k][2] = mz * r;
      }
      T.n = make_float4((float)un[0], (float)un[1], (float)un[2], __int_as_float(prim));
      T.m0 = make_float4((float)m[0][0], (float)m[0][1], (float)m[0][2], 0.f);
      T.m1 = make_float4((float)m[1][0], (float)m[1][1], (float)m[1][2],
                         (float)(e0[0] * m[1][0] + e0[1] * m[1][1] + e0[2] * m[1][2]));
      T.m2 = make_float4((float)m[2][0], (float)m[2][1], (float)m[2][2],
                         (float)(e1[0] * m[2][0] + e1[1] * m[2][1] + e1[2] * m[2][2]));
    } else {  // no area: the edges alone
      T.n = make_float4(0.f, 0.f, 0.f, __int_as_float(prim));
      T.m0 = make_float4(0.f, 0.f, 0.f, 1.f);
      T.m1 = make_float4(0.f, 0.f, 0.f, 1.f);
      T.m2 = make_float4(0.f, 0.f, 0.f, 1.f);
    }
    ltri[i] = T;
  }
}

// Eigenvectors of the symmetric 3x3 matrix A (cyclic Jacobi rotations in FP32, at most 8 sweeps):
// the columns of V, orthonormal to a few FP32 roundings.
__device__ void jacobi3f(float A[3][3], float V[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = i == j ? 1.f : 0.f;
#pragma unroll 1
  for (int sweep = 0; sweep < 8; ++sweep) {
    const float off = fabsf(A[0][1]) + fabsf(A[0][2]) + fabsf(A[1][2]);
    const float diag = fabsf(A[0][0]) + fabsf(A[1][1]) + fabsf(A[2][2]);
    if (!(off > 1e-7f * diag)) break;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int p = r == 2 ? 1 : 0, q = r == 0 ? 1 : 2;
      const float apq = A[p][q];
      if (apq == 0.f) continue;
      const float th = (A[q][q] - A[p][p]) / (2.f * apq);
      const float t = copysignf(1.f, th) / (fabsf(th) + sqrtf(fmaf(th, th, 1.f)));
      const float c = rsqrtf(fmaf(t, t, 1.f)), sn = t * c;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float akp = A[k][p], akq = A[k][q];
        A[k][p] = c * akp - sn * akq;
        A[k][q] = sn * akp + c * akq;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float apk = A[p][k], aqk = A[q][k];
        A[p][k] = c * apk - sn * aqk;
        A[q][k] = sn * apk + c * aqk;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float vkp = V[k][p], vkq = V[k][q];
        V[k][p] = c * vkp - sn * vkq;
        V[k][q] = sn * vkp + c * vkq;
      }
    }
  }
}

template <bool kWarp>
__device__ __forceinline__ double red_sum(double v) {
  if (kWarp)
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// The oriented box of the leaves [first, first + cnt) (see k_obb_small); kWarp: the 32 lanes of a
// warp share the loops over the vertices and all return the same box.
template <bool kWarp>
__device__ OBox fit_obox(const float4* __restrict__ lv32, int first, int cnt, double E, int lane) {
  const int step = kWarp ? 32 : 1, start = first + (kWarp ? lane : 0), end = first + cnt;
  const float4 r4 = lv32[3 * first];
  const double rx = r4.x, ry = r4.y, rz = r4.z;
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // sums of x, y, z, xx, xy, xz, yy, yz, zz about the first vertex
  for (int l = start; l < end; l += step)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 v = lv32[3 * l + k];
      const double x = v.x - rx, y = v.y - ry, z = v.z - rz;
      s[0] += x; s[1] += y; s[2] += z;
      s[3] = fma(x, x, s[3]); s[4] = fma(x, y, s[4]); s[5] = fma(x, z, s[5]);
      s[6] = fma(y, y, s[6]); s[7] = fma(y, z, s[7]); s[8] = fma(z, z, s[8]);
    }
#pragma unroll
  for (int k = 0; k < 9; ++k) s[k] = red_sum<kWarp>(s[k]);
  const double nv = 3.0 * cnt, mx = s[0] / nv, my = s[1] / nv, mz = s[2] / nv;
  const double c00 = s[3] / nv - mx * mx, c01 = s[4] / nv - mx * my, c02 = s[5] / nv - mx * mz;
  const double c11 = s[6] / nv - my * my, c12 = s[7] / nv - my * mz, c22 = s[8] / nv - mz * mz;
  const double tr = c00 + c11 + c22;
  double ax[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  if (tr > 0.0) {  // principal axes of the trace-normalised covariance (FP32 is enough for a direction)
    const double inv = 1.0 / tr;
    float A[3][3] = {{(float)(c00 * inv), (float)(c01 * inv), (float)(c02 * inv)},
                     {(float)(c01 * inv), (float)(c11 * inv), (float)(c12 * inv)},
                     {(float)(c02 * inv), (float)(c12 * inv), (float)(c22 * inv)}};
    float V[3][3];
    jacobi3f(A, V);
    // Gram-Schmidt in FP64: the axes are orthonormal to FP64 rounding before they are stored in FP32
    double a[3] = {V[0][0], V[1][0], V[2][0]}, b[3] = {V[0][1], V[1][1], V[2][1]};
    const double na = 1.0 / sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int k = 0; k < 3; ++k) a[k] *= na;
    const double ab = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    for (int k = 0; k < 3; ++k) b[k] -= ab * a[k];
    const double bb = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
    if (bb > 1e-12) {
      const double nb = 1.0 / sqrt(bb);
      for (int k = 0; k < 3; ++k) {
        ax[0][k] = a[k];
        ax[1][k] = b[k] * nb;
      }
      ax[2][0] = ax[0][1] * ax[1][2] - ax[0][2] * ax[1][1];
      ax[2][1] = ax[0][2] * ax[1][0] - ax[0][0] * ax[1][2];
      ax[2][2] = ax[0][0] * ax[1][1] - ax[0][1] * ax[1][0];
    }
  }
  float af[3][3];
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 3; ++k) af[a][k] = (float)ax[a][k];
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int l = start; l < end; l += step)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 v = lv32[3 * l + k];
#pragma unroll
      for (int a = 0; a < 3; ++a) {  // float x float products are exact in FP64
        const double t = (double)v.x * af[a][0] + (double)v.y * af[a][1] + (double)v.z * af[a][2];
        lo[a] = fmin(lo[a], t);
        hi[a] = fmax(hi[a], t);
      }
    }
  OBox o;
  float ce[3], ex[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (kWarp)
      for (int off = 16; off > 0; off >>= 1) {
        lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
        hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
      }
    const double c = 0.5 * (lo[a] + hi[a]);
    ce[a] = (float)c;
    // the FP64 sums above round by at most ~1e-15 E; the margin 1e-9 E covers them
    ex[a] = __double2float_ru(0.5 * (hi[a] - lo[a]) + fabs(c - (double)ce[a]) + 1e-9 * E);
  }
  o.a0 = make_float4(af[0][0], af[0][1], af[0][2], ce[0]);
  o.a1 = make_float4(af[1][0], af[1][1], af[1][2], ce[1]);
  o.a2 = make_float4(af[2][0], af[2][1], af[2][2], ce[2]);
  o.e = make_float4(ex[0], ex[1], ex[2], 0.f);
  return o;
}

// The child `side` of inner node i covers the sorted leaves [first, first + cnt): the left child
// [d.z, gamma], the right [gamma + 1, d.w].
__device__ __forceinline__ void child_range(const BNode* nodes, int i, int side, int& first, int& cnt) {
  const int4 d = nodes[i].d;
  const int gamma = d.x & 0x7fffffff;
  first = side ? gamma + 1 : d.z;
  cnt = side ? d.w - gamma : gamma - d.z + 1;
}

constexpr int kObbWarpMin = 33;  // children of this many leaves or more are fitted by a warp

// Oriented boxes of the LBVH's children (OBox, two per inner node: obb[2 i + side]).  For each child
// subtree of 2..kObbMaxLeaves leaves (a contiguous run of the Morton-sorted leaves) the principal
// axes of its vertices -- the FP64 covariance about the run's first vertex, diagonalised by Jacobi
// rotations -- and then the exact extents of its FP32 vertices along the axes as stored.  The axes
// only decide how tight the box is; the extents make it a bound for whatever axes come out.  On a
// smooth surface the smallest axis is the patch normal and the box is a thin slab around the patch,
// so a point at distance D from the surface has a lower bound close to D for every patch away from
// its nearest point (an axis-aligned box of a tilted patch is as thick as the patch is wide).
// Leaves and larger subtrees get kNoObb.  One thread per child here; children of kObbWarpMin or
// more leaves are left to k_obb_large (one warp per child).
__global__ void k_obb_small(const BNode* __restrict__ nodes, const float4* __restrict__ lv32, int n_inner, double E,
                            OBox* __restrict__ obb) {
  for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < 2 * n_inner; ci += gridDim.x * blockDim.x) {
    int first, cnt;
    child_range(nodes, ci >> 1, ci & 1, first, cnt);
    if (cnt >= kObbWarpMin && cnt <= kObbMaxLeaves) continue;
    OBox o;
    if (cnt >= 2 && cnt <= kObbMaxLeaves) {
      o = fit_obox<false>(lv32, first, cnt, E, 0);
    } else {
      o.a0 = make_float4(1.f, 0.f, 0.f, 0.f);
      o.a1 = make_float4(0.f, 1.f, 0.f, 0.f);
      o.a2 = make_float4(0.f, 0.f, 1.f, 0.f);
      o.e = make_float4(kNoObb, kNoObb, kNoObb, 0.f);
    }
    obb[ci] = o;
  }
}

__global__ void k_obb_large(const BNode* __restrict__ nodes, const float4* __restrict__ lv32, int n_inner, double E,
                            OBox* __restrict__ obb) {
  const int lane = threadIdx.x & 31, nw = (gridDim.x * blockDim.x) >> 5;
  for (int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < 2 * n_inner; ci += nw) {
    int first, cnt;
    child_range(nodes, ci >> 1, ci & 1, first, cnt);
    if (cnt < kObbWarpMin || cnt > kObbMaxLeaves) continue;
    const OBox o = fit_obox<true>(lv32, first, cnt, E, lane);
    if (lane == 0) obb[ci] = o;
  }
}

__global__ void k_ine_count(const int64_t* __restrict__ IEN, int64_t nel, int32_t* __restrict__ cnt) {
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) atomicAdd(&cnt[IEN[3 * el + k] - 1], 1);
}

__global__ void k_ine_fill(const int64_t* __restrict__ IEN, int64_t nel, const int32_t* __restrict__ off,
                           int32_t* __restrict__ cur, int32_t* __restrict__ ine) {
  for (int64_t el = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; el < nel; el += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const int64_t v = IEN[3 * el + k] - 1;
      ine[off[v] + atomicAdd(&cur[v], 1)] = (int32_t)el;
    }
}

}  // namespace

int mesh_upload_and_build(sdfgpu_ctx* ctx, const double* X, int64_t nnp, const int64_t* IEN, int64_t nel,
                          bool device_ptrs) {
  cudaStream_t st = ctx->stream;
  if (nel < 1 || nnp < 3) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "mesh needs at least 1 triangle and 3 vertices");
  if (nel > (int64_t)0x7fffffff / 4) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "too many triangles (limit 536870911)");
  if (!X || !IEN) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "X and IEN must not be NULL");
  ctx->has_mesh = false;
  ctx->mesh.ine_ready = false;
  ctx->launches = 0;
  // the previous mesh's LBVH build reads the buffers rewritten below
  SDF_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev_obb, 0));
  SDF_CUDA(ctx, cudaEventRecord(ctx->ev[4], st));

  double* dX;
  int64_t* dIEN;
  SDF_TRY(scratch_t(ctx, "X64", (size_t)nnp * 3, &dX));
  SDF_TRY(scratch_t(ctx, "IEN64", (size_t)nel * 3, &dIEN));
  const cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  SDF_CUDA(ctx, cudaMemcpyAsync(dX, X, sizeof(double) * 3 * nnp, kind, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(dIEN, IEN, sizeof(int64_t) * 3 * nel, kind, st));

  TriRec64* rec;
  double4* cent;
  float4 *v32, *c32, *box32;
  unsigned long long* bb;
  SDF_TRY(scratch_t(ctx, "rec", (size_t)nel, &rec));
  SDF_TRY(scratch_t(ctx, "cent64", (size_t)nel, &cent));
  SDF_TRY(scratch_t(ctx, "v32", (size_t)nel * 3, &v32));
  SDF_TRY(scratch_t(ctx, "c32", (size_t)nel, &c32));
  SDF_TRY(scratch_t(ctx, "box32", (size_t)nel * 2, &box32));
  SDF_TRY(scratch_t(ctx, "bbox", 8, &bb));

  unsigned long long init[8];
  for (int a = 0; a < 3; ++a) { init[a] = ~0ULL; init[3 + a] = 0ULL; }
  init[6] = 0ULL;
  init[7] = 0ULL;  // rho (ordered encoding of 0.0 is > 0; reset below)
  SDF_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, sizeof(int64_t) * C_NUM, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(bb, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_vertex_bbox<<<grid_for(nnp, 256, 148 * 8), 256, 0, st>>>(dX, nnp, bb);
  SDF_KERNEL(ctx);
  k_prep<<<grid_for(nel, 128), 128, 0, st>>>(dX, nnp, dIEN, nel, rec, cent, ctx->d_counters);
  SDF_KERNEL(ctx);
  unsigned long long hbb[8];
  int64_t hcnt[C_NUM];
  SDF_CUDA(ctx, cudaMemcpyAsync(hbb, bb, sizeof(hbb), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(hcnt, ctx->d_counters, sizeof(hcnt), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  if (hbb[6]) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "mesh vertices must be finite");
  if (hcnt[C_ERR_INDEX]) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "IEN holds an index outside 1..nnp");

  MeshDev& M = ctx->mesh;
  M.nnp = nnp;
  M.nel = nel;
  double E = 0.0;
  for (int a = 0; a < 3; ++a) {
    M.bmin[a] = ord_dbl(hbb[a]);
    M.bmax[a] = ord_dbl(hbb[3 + a]);
    M.center[a] = 0.5 * (M.bmin[a] + M.bmax[a]);
    E = std::max(E, std::max(M.bmax[a] - M.center[a], M.center[a] - M.bmin[a]));
  }
  M.E = E;

  unsigned long long rho0 = 0ULL;  // below the encoding of every non-negative double
  SDF_CUDA(ctx, cudaMemcpyAsync(bb + 7, &rho0, sizeof(rho0), cudaMemcpyHostToDevice, st));
  k_local32<<<grid_for(nel, 128), 128, 0, st>>>(rec, cent, dIEN, nel, M.center[0], M.center[1], M.center[2], M.E, v32,
                                                 c32, box32, bb + 7);
  SDF_KERNEL(ctx);

  // LBVH, on its own stream: only the unbounded search, the 3-nearest-vertex fallback and the
  // adaptive rays read it, and they wait for ev_bvh (the unbounded search for ev_obb, which also
  // covers the oriented boxes); the tile lists and the fold do not, so the build overlaps the
  // distance stage of the next call.
  SDF_CUDA(ctx, cudaEventRecord(ctx->ev_mesh, st));
  cudaStream_t sb = ctx->bvh_stream;
  SDF_CUDA(ctx, cudaStreamWaitEvent(sb, ctx->ev_mesh, 0));
  const int n = (int)nel;
  unsigned long long* keys2;
  BNode* nodes;
  int32_t *int_parent, *leaf_parent, *flags, *leaf_prim;
  SDF_TRY(scratch_t(ctx, "keys2", (size_t)n, &keys2));
  SDF_TRY(scratch_t(ctx, "nodes", (size_t)std::max(1, n - 1), &nodes));
  SDF_TRY(scratch_t(ctx, "int_parent", (size_t)n, &int_parent));
  SDF_TRY(scratch_t(ctx, "leaf_parent", (size_t)n, &leaf_parent));
  SDF_TRY(scratch_t(ctx, "flags", (size_t)n, &flags));
  SDF_TRY(scratch_t(ctx, "leaf_prim", (size_t)n, &leaf_prim));
  if (n == 1) {
    k_single_root<<<1, 1, 0, sb>>>(box32, nodes, leaf_prim);
    SDF_KERNEL(ctx);
  } else {
    const float lox = (float)(M.bmin[0] - M.center[0]), loy = (float)(M.bmin[1] - M.center[1]),
                loz = (float)(M.bmin[2] - M.center[2]);
    const double ext = std::max(M.bmax[0] - M.bmin[0], std::max(M.bmax[1] - M.bmin[1], M.bmax[2] - M.bmin[2]));
    const float inv = ext > 0 ? (float)(1024.0 / ext) : 1.0f;
    uint32_t *code, *code2;
    int32_t *idx, *idx2;
    SDF_TRY(scratch_t(ctx, "mcode", (size_t)n, &code));
    SDF_TRY(scratch_t(ctx, "mcode2", (size_t)n, &code2));
    SDF_TRY(scratch_t(ctx, "midx", (size_t)n, &idx));
    SDF_TRY(scratch_t(ctx, "midx2", (size_t)n, &idx2));
    k_morton<<<grid_for(nel, 256), 256, 0, sb>>>(c32, nel, lox, loy, loz, inv, code, idx);
    SDF_KERNEL(ctx);
    size_t tmp_bytes = 0;
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, code, code2, idx, idx2, n, 0, 30, sb));
    void* tmp;
    SDF_TRY(scratch(ctx, "cub_tmp_bvh", tmp_bytes, &tmp));
    SDF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, code, code2, idx, idx2, n, 0, 30, sb));
    k_pack_keys<<<grid_for(n, 256), 256, 0, sb>>>(code2, idx2, n, keys2);
    SDF_KERNEL(ctx);
    SDF_CUDA(ctx, cudaMemsetAsync(int_parent, 0xff, sizeof(int32_t) * n, sb));
    SDF_CUDA(ctx, cudaMemsetAsync(flags, 0, sizeof(int32_t) * n, sb));
    k_karras<<<grid_for(n - 1, 256), 256, 0, sb>>>(keys2, n, nodes, int_parent, leaf_parent);
    SDF_KERNEL(ctx);
    k_refit<<<grid_for(n, 256), 256, 0, sb>>>(keys2, box32, n, nodes, int_parent, leaf_parent, flags, leaf_prim);
    SDF_KERNEL(ctx);
  }
  float4* lv32;
  LeafTri* ltri;
  SDF_TRY(scratch_t(ctx, "lv32", (size_t)n * 3, &lv32));
  SDF_TRY(scratch_t(ctx, "ltri", (size_t)n, &ltri));
  k_leaf_order<<<grid_for(n, 256), 256, 0, sb>>>(leaf_prim, v32, rec, n, M.center[0], M.center[1], M.center[2], lv32,
                                                 ltri);
  SDF_KERNEL(ctx);
  // the rays and the 3-nearest-vertex fallback need only the tree; the unbounded searches wait for
  // the oriented boxes as well
  SDF_CUDA(ctx, cudaEventRecord(ctx->ev_bvh, sb));
  OBox* obb;
  const int n_inner = std::max(1, n - 1);
  SDF_TRY(scratch_t(ctx, "obb", (size_t)2 * n_inner, &obb));
  k_obb_small<<<grid_for(2 * n_inner, 256), 256, 0, sb>>>(nodes, lv32, n_inner, M.E, obb);
  SDF_KERNEL(ctx);
  k_obb_large<<<grid_for(2 * n_inner, 8, 148 * 16), 256, 0, sb>>>(nodes, lv32, n_inner, M.E, obb);
  SDF_KERNEL(ctx);
  SDF_CUDA(ctx, cudaEventRecord(ctx->ev_obb, sb));
  unsigned long long hrho = 0;
  SDF_CUDA(ctx, cudaMemcpyAsync(&hrho, bb + 7, sizeof(hrho), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaEventRecord(ctx->ev[5], st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  M.rho_max = ord_dbl(hrho);
  float ms = 0.f;
  SDF_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]));
  ctx->stats.ms_mesh = ms;
  ctx->stats.mesh_launches = ctx->launches;
  ctx->stats.nel = nel;
  ctx->stats.rho_max = M.rho_max;
  ctx->has_mesh = true;
  return 0;
}

int ensure_ine(sdfgpu_ctx* ctx) {
  MeshDev& M = ctx->mesh;
  if (M.ine_ready) return 0;
  cudaStream_t st = ctx->stream;
  int32_t *cnt, *off, *cur, *ine;
  SDF_TRY(scratch_t(ctx, "ine_cnt", (size_t)M.nnp + 1, &cnt));
  SDF_TRY(scratch_t(ctx, "ine_off", (size_t)M.nnp + 1, &off));
  SDF_TRY(scratch_t(ctx, "ine_cur", (size_t)M.nnp + 1, &cur));
  SDF_TRY(scratch_t(ctx, "ine", (size_t)M.nel * 3, &ine));
  const int64_t* dIEN = buf<int64_t>(ctx, "IEN64");
  SDF_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (M.nnp + 1), st));
  SDF_CUDA(ctx, cudaMemsetAsync(cur, 0, sizeof(int32_t) * (M.nnp + 1), st));
  k_ine_count<<<grid_for(M.nel, 256), 256, 0, st>>>(dIEN, M.nel, cnt);
  SDF_KERNEL(ctx);
  SDF_TRY(cub_scan_i32(ctx, cnt, off, M.nnp + 1));
  k_ine_fill<<<grid_for(M.nel, 256), 256, 0, st>>>(dIEN, M.nel, off, cur, ine);
  SDF_KERNEL(ctx);
  M.ine_ready = true;
  return 0;
}

int cub_scan_i32(sdfgpu_ctx* ctx, const int32_t* in, int32_t* out, int64_t n, cudaStream_t st, const char* tmp_name) {
  if (!st) st = ctx->stream;
  size_t bytes = 0;
  SDF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, st));
  void* tmp;
  SDF_TRY(scratch(ctx, tmp_name, bytes, &tmp));
  SDF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, st));
  return 0;
}

int cub_scan_i64(sdfgpu_ctx* ctx, const int64_t* in, int64_t* out, int64_t n) {
  size_t bytes = 0;
  SDF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, ctx->stream));
  void* tmp;
  SDF_TRY(scratch(ctx, "cub_tmp_scan", bytes, &tmp));
  SDF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, ctx->stream));
  return 0;
}

}  // namespace sdfgpu
