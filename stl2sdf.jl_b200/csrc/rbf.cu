// rbf.cu -- RBFs_smoothing (src/SdfSmoothing/RBFs4Smoothing.jl:275-320) on the GPU.
//
// The reference interpolates the SDF of the coarse grid with Gaussian RBFs of width sigma = cell
// size cut off below `threshold` (exp(-(r/sigma)^2) > threshold, i.e. r < sigma sqrt(-ln thr)),
// solving K w = sdf with conjugate gradients (interpolation) or taking w = sdf (approximation),
// and evaluates sum_j w_j exp(-(|p - c_j| / sigma)^2) on a grid refined `smooth` times.
//
// On a regular grid K is a fixed 3-D stencil, so nothing is assembled: the matrix-vector product
// reads the 5 x 5 x 5 neighbourhood of each node (the cut-off keeps the 81 nodes with
// |offset|^2 <= 6 cells^2 at the default threshold) with per-axis Gaussian factors taken from the
// nodes' actual Float32 coordinates, K = Kx Ky Kz (FP64 product, rounded to FP32 as the
// reference stores K).  CG follows IterativeSolvers.cg: x0 = 0, u = r + (|r|^2/|r_prev|^2) u,
// c = K u, alpha = |r|^2 / (u . c), stop when |r| <= sqrt(eps(Float32)) |b| or after n
// iterations; FP32 vectors, dot products accumulated in FP64 in a fixed order (deterministic).
// The new search direction is formed on the fly inside the product (double-buffered), so one CG
// iteration is two passes over the vectors.  The loop runs as a CUDA graph of kGraphIters
// iterations: the scalar kernel raises a device flag when the stopping rule holds, every kernel
// after it returns at once, so the result is that of stopping exactly there, and the host reads
// the flag once per graph launch instead of once per iteration.  The fine evaluation sums, per fine point, every
// coarse node within the cut-off distance (the reference's 124-nearest query always contains
// them all), with FP32 distances as the reference's KD-tree computes them and FP64 terms.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace sdfgpu {
namespace {

constexpr int kRbfMaxR = 4;      // stencil radius in cells (threshold >= exp(-16) ~ 1.1e-7)
constexpr int kRbfBlocks = 592;  // fixed grid of the reduction kernels (4 per SM): fixed sum order
constexpr int kRbfThreads = 256;
constexpr int kGraphIters = 16;  // CG iterations per graph launch (even: the u buffers swap back)

// Scalars of the CG loop (device): rr = |r|^2, beta, alpha, rr_prev, the stop flag (0/1), the
// iteration count and the stopping bound on rr.
enum CgScalar : int { CG_RR = 0, CG_BETA, CG_ALPHA, CG_RR_PREV, CG_DONE, CG_ITERS, CG_TOL2, CG_MAXIT, CG_NUM };

struct Axis3 {
  const float* x[3];
  int64_t n[3];
};

// process_vector (RBFs4Smoothing.jl:15-22), pass 1: max |v| over |v| < 1e9 (as ordered bits).
__global__ void k_rbf_absmax(const double* __restrict__ d, int64_t n, unsigned* out) {
  float m = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = fabsf((float)d[i]);
    if (v < 1.0e9f) m = fmaxf(m, v);
  }
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // m >= 0: bit order = value order
}

// pass 2: Float32 values, |v| ~ 1e10 (isapprox, rtol sqrt(eps(Float32))) -> sign(v) max.
__global__ void k_rbf_process(const double* __restrict__ d, int64_t n, const unsigned* mx, float* __restrict__ b) {
  const float big = 1.0e10f, rtol = 3.4526698e-4f, m = __uint_as_float(*mx);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = (float)d[i];
    const float a = fabsf(v);
    const bool near = fabsf(a - big) <= rtol * fmaxf(a, big);
    b[i] = near ? copysignf(m, v) : v;
  }
}

// c = K u_new with u_new = r + beta u_old formed on the fly; writes u_new of the own node and the
// block's partial sum of u_new . c.
__global__ void __launch_bounds__(kRbfThreads) k_rbf_matvec(Axis3 ax, const double* __restrict__ kt, int R,
                                                            double thr, const float* __restrict__ r,
                                                            const float* __restrict__ u_old, float* __restrict__ u_new,
                                                            float* __restrict__ c, const double* __restrict__ sc,
                                                            double* __restrict__ partial) {
  if (sc[CG_DONE] != 0.0) return;  // converged in an earlier iteration of this graph
  const int64_t nx = ax.n[0], ny = ax.n[1], nz = ax.n[2], nxy = nx * ny, ngp = nxy * nz;
  const int W = 2 * R + 1;
  const float beta = (float)sc[CG_BETA];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ngp; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = i % nx, y = (i / nx) % ny, z = i / nxy;
    const double* tx = kt + (size_t)x * W;
    const double* ty = kt + (size_t)(nx + y) * W;
    const double* tz = kt + (size_t)(nx + ny + z) * W;
    float s = 0.f;
    for (int oz = -R; oz <= R; ++oz) {
      const int64_t zz = z + oz;
      if (zz < 0 || zz >= nz) continue;
      const double fz = tz[oz + R];
      for (int oy = -R; oy <= R; ++oy) {
        const int64_t yy = y + oy;
        if (yy < 0 || yy >= ny) continue;
        const double fzy = fz * ty[oy + R];
        if (!(fzy > thr)) continue;
        const int64_t row = zz * nxy + yy * nx;
        for (int ox = -R; ox <= R; ++ox) {
          const int64_t xx = x + ox;
          if (xx < 0 || xx >= nx) continue;
          const double k = fzy * tx[ox + R];
          if (!(k > thr)) continue;
          const int64_t j = row + xx;
          const float uj = fmaf(beta, u_old[j], r[j]);
          s = fmaf((float)k, uj, s);
        }
      }
    }
    const float ui = fmaf(beta, u_old[i], r[i]);
    u_new[i] = ui;
    c[i] = s;
    acc += (double)ui * (double)s;
  }
  __shared__ double red[kRbfThreads / 32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kRbfThreads / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
}

// x += alpha u, r -= alpha c, partial |r|^2.
__global__ void __launch_bounds__(kRbfThreads) k_rbf_update(int64_t n, const double* __restrict__ sc,
                                                            const float* __restrict__ u, const float* __restrict__ c,
                                                            float* __restrict__ x, float* __restrict__ r,
                                                            double* __restrict__ partial) {
  if (sc[CG_DONE] != 0.0) return;
  const float alpha = (float)sc[CG_ALPHA];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = fmaf(alpha, u[i], x[i]);
    const float ri = fmaf(-alpha, c[i], r[i]);
    r[i] = ri;
    acc += (double)ri * (double)ri;
  }
  __shared__ double red[kRbfThreads / 32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kRbfThreads / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
}

// which = 0: alpha = rr / (u . c); which = 1: new rr, the next beta = rr_new / rr_old, one more
// iteration counted and the stop flag raised when rr <= tol^2 or the iteration cap is reached;
// which = 2: the initial rr = |b|^2 (no iteration, stop when b = 0).  One block, fixed order.
__global__ void k_rbf_scalar(const double* __restrict__ partial, int count, double* sc, int which) {
  if (which != 2 && sc[CG_DONE] != 0.0) return;
  __shared__ double red[kRbfThreads];
  double t = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) t += partial[i];
  red[threadIdx.x] = t;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double sum = red[0];
    if (which == 0) {
      sc[CG_ALPHA] = sc[CG_RR] / sum;
    } else if (which == 1) {
      sc[CG_RR_PREV] = sc[CG_RR];
      sc[CG_RR] = sum;
      sc[CG_BETA] = sum / sc[CG_RR_PREV];
      sc[CG_ITERS] += 1.0;
      if (!(sum > sc[CG_TOL2]) || sc[CG_ITERS] >= sc[CG_MAXIT]) sc[CG_DONE] = 1.0;
    } else {
      // IterativeSolvers: prev_residual = 1 at the start, so the first beta is |b|^2 (u is 0)
      sc[CG_RR] = sum;
      sc[CG_RR_PREV] = 1.0;
      sc[CG_BETA] = sum;
      sc[CG_TOL2] = (double)FLT_EPSILON * sum;  // (sqrt(eps(Float32)) |b|)^2
      if (!(sum > sc[CG_TOL2])) sc[CG_DONE] = 1.0;
    }
  }
}

// Fine grid: every coarse node within maxd (FP32 distance) of the fine point, FP64 terms.
__global__ void k_rbf_eval(Axis3 fine, Axis3 coarse, double h, double sigma, float maxd, int R,
                           const float* __restrict__ w, float* __restrict__ out) {
  const int64_t nx = fine.n[0], ny = fine.n[1], nz = fine.n[2], ngp = nx * ny * nz;
  const double inv_s2 = 1.0 / (sigma * sigma);
  const float x0c = coarse.x[0][0], y0c = coarse.x[1][0], z0c = coarse.x[2][0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ngp; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t fx = i % nx, fy = (i / nx) % ny, fz = i / (nx * ny);
    const float px = fine.x[0][fx], py = fine.x[1][fy], pz = fine.x[2][fz];
    int64_t lo[3], hi[3];
    const float pc[3] = {px, py, pz}, c0[3] = {x0c, y0c, z0c};
    for (int a = 0; a < 3; ++a) {
      const int64_t m = (int64_t)floor(((double)pc[a] - (double)c0[a]) / h);
      lo[a] = std::max<int64_t>(0, m - R - 1);
      hi[a] = std::min<int64_t>(coarse.n[a] - 1, m + R + 2);
    }
    double acc = 0.0;
    for (int64_t cz = lo[2]; cz <= hi[2]; ++cz) {
      const float dz = __fsub_rn(pz, coarse.x[2][cz]);
      const float dz2 = __fmul_rn(dz, dz);
      if (dz2 > maxd * maxd * 1.0001f) continue;
      for (int64_t cy = lo[1]; cy <= hi[1]; ++cy) {
        const float dy = __fsub_rn(py, coarse.x[1][cy]);
        const float dy2 = __fmul_rn(dy, dy);
        if (dy2 > maxd * maxd * 1.0001f) continue;
        for (int64_t cx = lo[0]; cx <= hi[0]; ++cx) {
          const float dx = __fsub_rn(px, coarse.x[0][cx]);
          const float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), dy2), dz2);
          const float dist = __fsqrt_rn(s);
          if (!(dist <= maxd)) continue;
          const double t = (double)dist;
          acc += (double)w[(cz * coarse.n[1] + cy) * coarse.n[0] + cx] * exp(-(t * t) * inv_s2);
        }
      }
    }
    out[i] = (float)acc;
  }
}

}  // namespace
}  // namespace sdfgpu

using namespace sdfgpu;

extern "C" int sdfgpu_rbf_smoothing(sdfgpu_ctx* ctx, const double aabb_min[3], const double aabb_max[3],
                                    const int64_t N[3], double cell_size, const double* dist, int32_t interpolation,
                                    int32_t smooth, double threshold, float* fine_out, float* weights_out,
                                    int32_t* cg_iterations, double* cg_residual) {
  SDF_TRY(begin_call(ctx));
  if (!aabb_min || !aabb_max || !N || !dist || !fine_out)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "rbf_smoothing: NULL argument");
  if (!(cell_size > 0.0) || !std::isfinite(cell_size) || smooth < 1 || smooth > 16 || !(threshold > 1.2e-7) ||
      !(threshold < 1.0))
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT,
                "rbf_smoothing: need cell_size > 0, 1 <= smooth <= 16 and exp(-16) < threshold < 1");
  double cells = 1.0, fcells = 1.0;
  int64_t nc[3], nf[3];
  for (int a = 0; a < 3; ++a) {
    if (N[a] < 1) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "rbf_smoothing: every N must be >= 1");
    nc[a] = N[a] + 1;
    nf[a] = N[a] * smooth + 1;
    cells *= (double)nc[a];
    fcells *= (double)nf[a];
  }
  if (fcells > 2147483647.0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "rbf_smoothing: fine grid too large");
  const int64_t n = (int64_t)cells, m = (int64_t)fcells;
  const double sigma = cell_size;
  const double rcut = std::sqrt(-std::log(threshold));  // cut-off radius in units of sigma
  const int R = std::min(kRbfMaxR, (int)std::ceil(rcut));
  const float maxd = (float)std::sqrt(-std::log(threshold) * sigma * sigma);
  // Coordinates (Float32) on the host: coarse = range(min, max, length = N+1); fine = min + i dx
  // with dx = (xmax - xmin) / (nx - 1) from the x axis, in Float32 arithmetic.
  std::vector<float> hc, hf;
  for (int a = 0; a < 3; ++a) {
    const double lo = (double)(float)aabb_min[a], hi = (double)(float)aabb_max[a];  // Float32 end points
    for (int64_t i = 0; i < nc[a]; ++i) hc.push_back((float)(lo + (hi - lo) * (double)i / (double)N[a]));
  }
  volatile float fx0 = (float)aabb_min[0], fx1 = (float)aabb_max[0];
  volatile float span = fx1 - fx0;
  volatile float dxf = span / (float)(nf[0] - 1);
  for (int a = 0; a < 3; ++a) {
    const float f0 = (float)aabb_min[a];
    for (int64_t i = 0; i < nf[a]; ++i) {
      volatile float step = (float)i * dxf;
      hf.push_back(f0 + step);
    }
  }
  // Per-axis Gaussian factors exp(-(dx/sigma)^2) of the coarse stencil (0 outside the grid).
  const int W = 2 * R + 1;
  std::vector<double> hk((size_t)(nc[0] + nc[1] + nc[2]) * W, 0.0);
  {
    size_t base = 0, off = 0;
    for (int a = 0; a < 3; ++a) {
      for (int64_t i = 0; i < nc[a]; ++i)
        for (int o = -R; o <= R; ++o) {
          const int64_t j = i + o;
          if (j < 0 || j >= nc[a]) continue;
          volatile float d = hc[off + j] - hc[off + i];
          const double t = (double)d / sigma;
          hk[base + (size_t)i * W + (o + R)] = std::exp(-t * t);
        }
      base += (size_t)nc[a] * W;
      off += (size_t)nc[a];
    }
  }
  cudaStream_t st = ctx->stream;
  float *dc, *df, *b, *x, *r, *u0, *u1, *c, *out;
  double *kt, *dd, *part, *sc;
  unsigned* mx;
  SDF_TRY(scratch_t(ctx, "rbf_cx", hc.size(), &dc));
  SDF_TRY(scratch_t(ctx, "rbf_fx", hf.size(), &df));
  SDF_TRY(scratch_t(ctx, "rbf_kt", hk.size(), &kt));
  SDF_TRY(scratch_t(ctx, "rbf_dist", (size_t)n, &dd));
  SDF_TRY(scratch_t(ctx, "rbf_b", (size_t)n, &b));
  SDF_TRY(scratch_t(ctx, "rbf_x", (size_t)n, &x));
  SDF_TRY(scratch_t(ctx, "rbf_r", (size_t)n, &r));
  SDF_TRY(scratch_t(ctx, "rbf_u0", (size_t)n, &u0));
  SDF_TRY(scratch_t(ctx, "rbf_u1", (size_t)n, &u1));
  SDF_TRY(scratch_t(ctx, "rbf_c", (size_t)n, &c));
  SDF_TRY(scratch_t(ctx, "rbf_out", (size_t)m, &out));
  SDF_TRY(scratch_t(ctx, "rbf_part", kRbfBlocks, &part));
  SDF_TRY(scratch_t(ctx, "rbf_sc", CG_NUM, &sc));
  SDF_TRY(scratch_t(ctx, "rbf_mx", 1, &mx));
  SDF_CUDA(ctx, cudaMemcpyAsync(dc, hc.data(), sizeof(float) * hc.size(), cudaMemcpyHostToDevice, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(df, hf.data(), sizeof(float) * hf.size(), cudaMemcpyHostToDevice, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(kt, hk.data(), sizeof(double) * hk.size(), cudaMemcpyHostToDevice, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(dd, dist, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  SDF_CUDA(ctx, cudaMemsetAsync(mx, 0, sizeof(unsigned), st));
  const unsigned g = grid_for(n, kRbfThreads, 148 * 8);
  k_rbf_absmax<<<g, kRbfThreads, 0, st>>>(dd, n, mx);
  SDF_KERNEL(ctx);
  k_rbf_process<<<g, kRbfThreads, 0, st>>>(dd, n, mx, b);
  SDF_KERNEL(ctx);
  Axis3 ac{{dc, dc + nc[0], dc + nc[0] + nc[1]}, {nc[0], nc[1], nc[2]}};
  Axis3 af{{df, df + nf[0], df + nf[0] + nf[1]}, {nf[0], nf[1], nf[2]}};
  const float* weights = b;
  int iters = 0;
  double res = 0.0;
  if (interpolation) {
    // x = 0, r = b, u = 0; |b|^2 through the update's reduction with alpha = 0 (x and r unchanged)
    SDF_CUDA(ctx, cudaMemsetAsync(x, 0, sizeof(float) * n, st));
    SDF_CUDA(ctx, cudaMemsetAsync(u0, 0, sizeof(float) * n, st));
    SDF_CUDA(ctx, cudaMemcpyAsync(r, b, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    double h_sc[CG_NUM] = {0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, (double)n};
    SDF_CUDA(ctx, cudaMemcpyAsync(sc, h_sc, sizeof(h_sc), cudaMemcpyHostToDevice, st));
    k_rbf_update<<<kRbfBlocks, kRbfThreads, 0, st>>>(n, sc, u0, u0, x, r, part);
    SDF_KERNEL(ctx);
    k_rbf_scalar<<<1, kRbfThreads, 0, st>>>(part, kRbfBlocks, sc, 2);
    SDF_KERNEL(ctx);
    // kGraphIters iterations captured once: matvec (u0 -> u1), alpha, update, rr; then u1 -> u0.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto release = [&]() {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
    };
    SDF_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    bool cap_ok = true;
    for (int k = 0; k < kGraphIters && cap_ok; ++k) {
      float* ua = (k & 1) ? u1 : u0;
      float* ub = (k & 1) ? u0 : u1;
      k_rbf_matvec<<<kRbfBlocks, kRbfThreads, 0, st>>>(ac, kt, R, threshold, r, ua, ub, c, sc, part);
      k_rbf_scalar<<<1, kRbfThreads, 0, st>>>(part, kRbfBlocks, sc, 0);
      k_rbf_update<<<kRbfBlocks, kRbfThreads, 0, st>>>(n, sc, ub, c, x, r, part);
      k_rbf_scalar<<<1, kRbfThreads, 0, st>>>(part, kRbfBlocks, sc, 1);
      cap_ok = cudaGetLastError() == cudaSuccess;
    }
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (!cap_ok || ce != cudaSuccess) {
      release();
      return fail(ctx, SDFGPU_ERR_CUDA, std::string("rbf_smoothing: CG graph capture failed: ") + cudaGetErrorString(ce));
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
      release();
      return fail(ctx, SDFGPU_ERR_CUDA, std::string("rbf_smoothing: cudaGraphInstantiate: ") + cudaGetErrorString(ce));
    }
    ctx->launches += 4 * kGraphIters;
    static_assert((int)CG_NUM <= (int)S_NUM, "the CG scalars are read back through the context's page-locked slots");
    double* h_out = reinterpret_cast<double*>(ctx->h_scalars);  // page-locked: read back per launch
    const int64_t max_launches = n / kGraphIters + 2;
    for (int64_t l = 0;; ++l) {
      ce = cudaGraphLaunch(exec, st);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(h_out, sc, sizeof(double) * CG_NUM, cudaMemcpyDeviceToHost, st);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
      if (ce != cudaSuccess) {
        release();
        return fail(ctx, SDFGPU_ERR_CUDA, std::string("rbf_smoothing: CG graph: ") + cudaGetErrorString(ce));
      }
      if (!std::isfinite(h_out[CG_RR])) {
        release();
        return fail(ctx, SDFGPU_ERR_CUDA, "rbf_smoothing: CG diverged (non-finite residual)");
      }
      if (h_out[CG_DONE] != 0.0 || l >= max_launches) break;
    }
    release();
    iters = (int)h_out[CG_ITERS];
    const double rr = h_out[CG_RR];
    res = std::sqrt(rr);
    weights = x;
  }
  k_rbf_eval<<<grid_for(m, kRbfThreads, 148 * 16), kRbfThreads, 0, st>>>(af, ac, cell_size, sigma, maxd, R, weights,
                                                                            out);
  SDF_KERNEL(ctx);
  SDF_CUDA(ctx, cudaMemcpyAsync(fine_out, out, sizeof(float) * m, cudaMemcpyDeviceToHost, st));
  if (weights_out) SDF_CUDA(ctx, cudaMemcpyAsync(weights_out, weights, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  if (cg_iterations) *cg_iterations = iters;
  if (cg_residual) *cg_residual = res;
  return SDFGPU_OK;
}
