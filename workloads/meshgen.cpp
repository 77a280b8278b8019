// meshgen.cpp -- closed synthetic meshes for the SignedDistances workloads (libmeshgen.so).
//
// Marching cubes over a scalar field s(x) on an n^3 lattice; "inside" is s > 0.  The case table
// is derived at start-up from the cube's faces rather than tabulated by hand: on every face the
// runs of consecutive inside corners (in counter-clockwise order seen from outside the cube) are
// cut off by one segment each, from the crossing on the edge that leaves the run to the crossing
// on the edge that enters it.  A face with two diagonal inside corners therefore separates them,
// and since that choice depends only on the face's own four corners, the two cells sharing a face
// always agree, which makes the surface closed.  The segments of a cell chain into loops (every
// crossing edge ends one segment and starts another), and each loop is fanned into triangles,
// reversed so normals point from inside to outside.
//
// Vertices are shared through global lattice-edge ids (interpolated at t = s0/(s0 - s1), clamped
// to [1e-3, 1 - 1e-3] of the edge so no two vertices coincide), so the output is an indexed,
// watertight mesh.  The lattice is processed one z-slab at a time with the field evaluated per
// slice (OpenMP), so memory stays at a few lattice planes.  Output order is deterministic.
//
// Fields:
//   blobs:  s = sum_b exp(-|x - c_b|^2 / (2 sigma_b^2)) - iso   (separable per axis)
//   gyroid: s = thickness - |sin x cos y + sin y cos z + sin z cos x|, forced to -1 on the
//           lattice border so the sheet is capped and closed.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

struct Table {
  // per configuration: triangles as triples of cube-edge ids (0..11), -1 terminated
  std::array<std::array<int8_t, 16 * 3>, 256> tri;
  int edge_corner[12][2];
};

int corner_bit(int c, int a) { return (c >> a) & 1; }

Table build_table() {
  Table T;
  int ne = 0;
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 8; ++c)
      if (!corner_bit(c, a)) {
        T.edge_corner[ne][0] = c;
        T.edge_corner[ne][1] = c | (1 << a);
        ++ne;
      }
  auto edge_of = [&](int c0, int c1) {
    for (int e = 0; e < 12; ++e)
      if ((T.edge_corner[e][0] == c0 && T.edge_corner[e][1] == c1) ||
          (T.edge_corner[e][0] == c1 && T.edge_corner[e][1] == c0))
        return e;
    return -1;
  };
  // faces: corners in counter-clockwise order seen from outside
  std::vector<std::array<int, 4>> faces;
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s) {
      std::vector<int> cs;
      for (int c = 0; c < 8; ++c)
        if (corner_bit(c, a) == s) cs.push_back(c);
      const int u = (a + 1) % 3, v = (a + 2) % 3;
      // cyclic order in the (u, v) plane
      std::array<int, 4> cyc;
      const int order[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
      for (int q = 0; q < 4; ++q)
        for (int c : cs)
          if (corner_bit(c, u) == order[q][0] && corner_bit(c, v) == order[q][1]) cyc[q] = c;
      // (e_u x e_v) = e_a; outward normal is +e_a for s = 1, -e_a for s = 0
      if (s == 0) std::swap(cyc[1], cyc[3]);
      faces.push_back(cyc);
    }
  for (int cfg = 0; cfg < 256; ++cfg) {
    auto inside = [&](int c) { return (cfg >> c) & 1; };
    int next_of[12];
    for (int e = 0; e < 12; ++e) next_of[e] = -1;
    for (auto& f : faces) {
      int nin = 0;
      for (int q = 0; q < 4; ++q) nin += inside(f[q]);
      if (nin == 0 || nin == 4) continue;
      for (int q = 0; q < 4; ++q) {
        // a run starts at f[q] when f[q] is inside and its predecessor is outside
        if (!inside(f[q]) || inside(f[(q + 3) % 4])) continue;
        int r = q;
        while (inside(f[(r + 1) % 4])) r = (r + 1) % 4;
        const int entry = edge_of(f[(q + 3) % 4], f[q]);
        const int exit = edge_of(f[r], f[(r + 1) % 4]);
        next_of[exit] = entry;  // segment exit -> entry
      }
    }
    int nt = 0;
    bool used[12] = {};
    for (int e0 = 0; e0 < 12; ++e0) {
      if (next_of[e0] < 0 || used[e0]) continue;
      std::vector<int> loop;
      int e = e0;
      while (!used[e]) {
        used[e] = true;
        loop.push_back(e);
        e = next_of[e];
      }
      // the loop runs counter-clockwise around the inside part of the cube surface: reverse the
      // fan so triangle normals point outward (away from the inside region)
      for (size_t k = 1; k + 1 < loop.size(); ++k) {
        T.tri[cfg][3 * nt + 0] = (int8_t)loop[0];
        T.tri[cfg][3 * nt + 1] = (int8_t)loop[k + 1];
        T.tri[cfg][3 * nt + 2] = (int8_t)loop[k];
        ++nt;
      }
    }
    for (int q = 3 * nt; q < 16 * 3; ++q) T.tri[cfg][q] = -1;
  }
  return T;
}

struct Field {
  virtual void slice(int k, std::vector<double>& out) const = 0;  // (n x n), x fastest
  virtual ~Field() {}
};

struct Blobs : Field {
  int n;
  double lo, step, iso;
  int nb;
  std::vector<double> ex, ey, ez;  // nb x n each
  Blobs(const double* c, const double* s, int nb_, double iso_, int n_, double lo_, double hi_)
      : n(n_), lo(lo_), step((hi_ - lo_) / (n_ - 1)), iso(iso_), nb(nb_) {
    ex.resize((size_t)nb * n); ey.resize((size_t)nb * n); ez.resize((size_t)nb * n);
    for (int b = 0; b < nb; ++b) {
      const double inv = 1.0 / (2.0 * s[b] * s[b]);
      for (int i = 0; i < n; ++i) {
        const double x = lo + step * i;
        ex[(size_t)b * n + i] = std::exp(-(x - c[3 * b]) * (x - c[3 * b]) * inv);
        ey[(size_t)b * n + i] = std::exp(-(x - c[3 * b + 1]) * (x - c[3 * b + 1]) * inv);
        ez[(size_t)b * n + i] = std::exp(-(x - c[3 * b + 2]) * (x - c[3 * b + 2]) * inv);
      }
    }
  }
  void slice(int k, std::vector<double>& out) const override {
    out.assign((size_t)n * n, 0.0);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double f = 0.0;
        for (int b = 0; b < nb; ++b)
          f += ex[(size_t)b * n + i] * ey[(size_t)b * n + j] * ez[(size_t)b * n + k];
        out[(size_t)j * n + i] = f - iso;
      }
  }
};

struct Gyroid : Field {
  int n;
  double thick;
  std::vector<double> sn, cs;
  Gyroid(int n_, double lo, double hi, double thick_) : n(n_), thick(thick_) {
    const double step = (hi - lo) / (n - 1);
    sn.resize(n); cs.resize(n);
    for (int i = 0; i < n; ++i) { sn[i] = std::sin(lo + step * i); cs[i] = std::cos(lo + step * i); }
  }
  void slice(int k, std::vector<double>& out) const override {
    out.assign((size_t)n * n, 0.0);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double s = -1.0;
        if (i > 0 && j > 0 && k > 0 && i < n - 1 && j < n - 1 && k < n - 1) {
          const double g = sn[i] * cs[j] + sn[j] * cs[k] + sn[k] * cs[i];
          s = thick - std::fabs(g);
        }
        out[(size_t)j * n + i] = s;
      }
  }
};

int64_t march(const Field& F, int n, double lo, double hi, std::vector<double>& V, std::vector<int64_t>& T) {
  static const Table TB = build_table();
  const double step = (hi - lo) / (n - 1);
  std::vector<double> s0, s1;
  F.slice(0, s0);
  const size_t nn = (size_t)n * n;
  // vertex id of every lattice edge of the current slab: x- and y-edges of planes k and k+1,
  // z-edges between them
  std::vector<int64_t> xe0(nn, -1), ye0(nn, -1), xe1(nn, -1), ye1(nn, -1), ze(nn, -1);
  auto vid = [&](std::vector<int64_t>& slot, size_t idx, double x0, double y0, double z0, int axis, double a, double b) {
    if (slot[idx] >= 0) return slot[idx];
    double t = a / (a - b);
    t = std::min(std::max(t, 1e-3), 1.0 - 1e-3);
    double p[3] = {x0, y0, z0};
    p[axis] += t * step;
    V.push_back(p[0]); V.push_back(p[1]); V.push_back(p[2]);
    slot[idx] = (int64_t)(V.size() / 3) - 1;
    return slot[idx];
  };
  for (int k = 0; k + 1 < n; ++k) {
    F.slice(k + 1, s1);
    std::fill(xe1.begin(), xe1.end(), -1);
    std::fill(ye1.begin(), ye1.end(), -1);
    std::fill(ze.begin(), ze.end(), -1);
    const double z0 = lo + step * k;
    for (int j = 0; j + 1 < n; ++j)
      for (int i = 0; i + 1 < n; ++i) {
        double c[8];
        for (int q = 0; q < 8; ++q) {
          const size_t idx = (size_t)(j + ((q >> 1) & 1)) * n + (i + (q & 1));
          c[q] = (q & 4) ? s1[idx] : s0[idx];
        }
        int cfg = 0;
        for (int q = 0; q < 8; ++q)
          if (c[q] > 0.0) cfg |= 1 << q;
        if (cfg == 0 || cfg == 255) continue;
        int64_t ev[12];
        for (int e = 0; e < 12; ++e) ev[e] = -1;
        for (int e = 0; e < 12; ++e) {
          const int ca = TB.edge_corner[e][0], cb = TB.edge_corner[e][1];
          if (((cfg >> ca) & 1) == ((cfg >> cb) & 1)) continue;
          const int axis = e / 4;
          const int di = ca & 1, dj = (ca >> 1) & 1, dk = (ca >> 2) & 1;
          const size_t idx = (size_t)(j + dj) * n + (i + di);
          const double x0 = lo + step * (i + di), y0 = lo + step * (j + dj), zz = z0 + step * dk;
          // interpolate from the inside-or-outside corner a towards b along +axis
          if (axis == 0) ev[e] = vid(dk ? xe1 : xe0, idx, x0, y0, zz, 0, c[ca], c[cb]);
          else if (axis == 1) ev[e] = vid(dk ? ye1 : ye0, idx, x0, y0, zz, 1, c[ca], c[cb]);
          else ev[e] = vid(ze, idx, x0, y0, zz, 2, c[ca], c[cb]);
        }
        const auto& tr = TB.tri[cfg];
        for (int q = 0; q < 16 && tr[3 * q] >= 0; ++q) {
          T.push_back(ev[tr[3 * q]] + 1);
          T.push_back(ev[tr[3 * q + 1]] + 1);
          T.push_back(ev[tr[3 * q + 2]] + 1);
        }
      }
    std::swap(s0, s1);
    std::swap(xe0, xe1);
    std::swap(ye0, ye1);
  }
  return (int64_t)(T.size() / 3);
}

struct Result {
  std::vector<double> V;
  std::vector<int64_t> T;
};

}  // namespace

extern "C" {

// Gaussian-blob isosurface: returns a handle; read it with mg_sizes / mg_copy, free with mg_free.
void* mg_blobs(const double* centers, const double* sigmas, int nb, double iso, int n, double lo, double hi) {
  Result* r = new Result();
  Blobs F(centers, sigmas, nb, iso, n, lo, hi);
  march(F, n, lo, hi, r->V, r->T);
  return r;
}

void* mg_gyroid(int n, double lo, double hi, double thickness) {
  Result* r = new Result();
  Gyroid F(n, lo, hi, thickness);
  march(F, n, lo, hi, r->V, r->T);
  return r;
}

void mg_sizes(void* h, int64_t* nv, int64_t* nt) {
  Result* r = (Result*)h;
  *nv = (int64_t)(r->V.size() / 3);
  *nt = (int64_t)(r->T.size() / 3);
}

void mg_copy(void* h, double* V, int64_t* T) {
  Result* r = (Result*)h;
  std::memcpy(V, r->V.data(), r->V.size() * sizeof(double));
  std::memcpy(T, r->T.data(), r->T.size() * sizeof(int64_t));
}

void mg_free(void* h) { delete (Result*)h; }

// The derived case table (256 x 16 x 3 edge ids, -1 padded) and edge corners, for tests.
void mg_table(int8_t* tri, int32_t* edge_corner) {
  static const Table TB = build_table();
  for (int c = 0; c < 256; ++c) std::memcpy(tri + 48 * c, TB.tri[c].data(), 48);
  for (int e = 0; e < 12; ++e) { edge_corner[2 * e] = TB.edge_corner[e][0]; edge_corner[2 * e + 1] = TB.edge_corner[e][1]; }
}

}  // extern "C"
