// radius.cu -- the learned search radius: a small Fourier-feature MLP that predicts, per node, a
// radius r(p) that bounds the nearest-triangle search of SDFGPU_MODE_UNBOUNDED.
//
// Network (FP16 weights, FP32 accumulate), on normalised coordinates x = (p - c) / s:
//   f  = [x, sin(2^k pi x), cos(2^k pi x) for k = 0..3, 0 x 5]    (32 features)
//   h0 = half(f)
//   h1 = half(relu(W1 h0 + b1))      W1: 64 x 32
//   h2 = half(relu(W2 h1 + b2))      W2: 64 x 64
//   a3 = relu(W3 h2 + b3)            W3: 64 x 64   (FP32)
//   y  = w4 . a3 + b4,  dhat = softplus(y)   (normalised distance)
// Weights are rounded to FP16 wherever they are used; the FP32 master copy is what Adam updates.
// The loss is mean((log(dhat + eps) - log(d + eps))^2), eps = 1e-3, on exact unbounded distances d
// of a coarse grid of the same mesh computed by the library's own exact kernel.
//
// Training kernels run on CUDA cores (batched: per-sample forward and backward, per-row weight
// gradients with a fixed summation order, Adam).  Inference uses mma.sync m16n8k16 (FP16 in, FP32
// accumulate): a warp evaluates 32 nodes, and each layer's FP32 accumulator fragments are converted
// in registers into the next layer's A fragments (the accumulator layout of two adjacent n8 tiles
// is the A layout of one k16 tile), so activations never leave registers.
//
// Use: radius r = (dhat (1 + alpha) + beta) * s.  The unbounded search prunes with r; a nearest hit
// with d <= r is certified exact (every triangle nearer than it lies within r and was visited);
// otherwise the node falls back to the unbounded search.
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "radius.cuh"

namespace sdfgpu {

namespace {

__device__ __forceinline__ float h16(float x) { return __half2float(__float2half_rn(x)); }

__device__ __forceinline__ void features(float x0, float x1, float x2, float f[kIn]) {
  f[0] = x0; f[1] = x1; f[2] = x2;
  const float xs[3] = {x0, x1, x2};
#pragma unroll
  for (int k = 0; k < kFreq; ++k)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float s, c;
      sincospif(xs[a] * (float)(1 << k), &s, &c);
      f[3 + 6 * k + 2 * a] = s;
      f[3 + 6 * k + 2 * a + 1] = c;
    }
#pragma unroll
  for (int q = kFeat; q < kIn; ++q) f[q] = 0.f;
}

__device__ __forceinline__ float softplus(float y) { return y > 20.f ? y : log1pf(expf(y)); }
__device__ __forceinline__ float sigmoid(float y) { return 1.f / (1.f + expf(-y)); }

// ---- training -----------------------------------------------------------------------------

// Per-sample forward (the definition above) storing what the backward needs, plus the loss term
// and dL/dy of every sample.
__global__ void k_train_fwd(const float* __restrict__ P, const float* __restrict__ X, const float* __restrict__ T,
                            int64_t B, float* __restrict__ H0, float* __restrict__ H1, float* __restrict__ H2,
                            float* __restrict__ A3, float* __restrict__ GY, float* __restrict__ LOSS,
                            float* __restrict__ YHAT) {
  __shared__ float W[kParams];
  for (int q = threadIdx.x; q < kParams; q += blockDim.x) W[q] = (q < kOffB1 || (q >= kOffW2 && q < kOffB2) ||
                                                                   (q >= kOffW3 && q < kOffB3) || (q >= kOffW4 && q < kOffB4))
                                                                      ? h16(P[q]) : P[q];
  __syncthreads();
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
    float f[kIn];
    features(X[3 * b], X[3 * b + 1], X[3 * b + 2], f);
    float h0[kIn], h1[kHid], h2[kHid], a3[kHid];
    for (int j = 0; j < kIn; ++j) { h0[j] = h16(f[j]); H0[b * kIn + j] = h0[j]; }
    for (int i = 0; i < kHid; ++i) {
      float z = W[kOffB1 + i];
      for (int j = 0; j < kIn; ++j) z = fmaf(W[kOffW1 + i * kIn + j], h0[j], z);
      h1[i] = h16(fmaxf(z, 0.f));
      H1[b * kHid + i] = h1[i];
    }
    for (int i = 0; i < kHid; ++i) {
      float z = W[kOffB2 + i];
      for (int j = 0; j < kHid; ++j) z = fmaf(W[kOffW2 + i * kHid + j], h1[j], z);
      h2[i] = h16(fmaxf(z, 0.f));
      H2[b * kHid + i] = h2[i];
    }
    for (int i = 0; i < kHid; ++i) {
      float z = W[kOffB3 + i];
      for (int j = 0; j < kHid; ++j) z = fmaf(W[kOffW3 + i * kHid + j], h2[j], z);
      a3[i] = fmaxf(z, 0.f);
      A3[b * kHid + i] = a3[i];
    }
    float y = W[kOffB4];
    for (int j = 0; j < kHid; ++j) y = fmaf(W[kOffW4 + j], a3[j], y);
    const float dh = softplus(y);
    if (YHAT) YHAT[b] = dh;
    if (T) {
      const float r = logf(dh + kLogEps) - logf(T[b] + kLogEps);
      LOSS[b] = r * r;
      GY[b] = 2.f * r / (dh + kLogEps) * sigmoid(y) / (float)B;
    }
  }
}

// Per-sample backward through the layers: DZ3, DZ2, DZ1 (the relu masks use the stored
// activations: a unit is active when its stored output is > 0).
__global__ void k_train_bwd(const float* __restrict__ P, int64_t B, const float* __restrict__ H1,
                            const float* __restrict__ H2, const float* __restrict__ A3, const float* __restrict__ GY,
                            float* __restrict__ DZ1, float* __restrict__ DZ2, float* __restrict__ DZ3) {
  __shared__ float W[kParams];
  for (int q = threadIdx.x; q < kParams; q += blockDim.x) W[q] = q < kOffB4 ? h16(P[q]) : P[q];
  __syncthreads();
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
    const float gy = GY[b];
    float dz3[kHid], dz2[kHid];
    for (int i = 0; i < kHid; ++i) {
      dz3[i] = A3[b * kHid + i] > 0.f ? gy * W[kOffW4 + i] : 0.f;
      DZ3[b * kHid + i] = dz3[i];
    }
    for (int j = 0; j < kHid; ++j) {
      float s = 0.f;
      for (int i = 0; i < kHid; ++i) s = fmaf(W[kOffW3 + i * kHid + j], dz3[i], s);
      dz2[j] = H2[b * kHid + j] > 0.f ? s : 0.f;
      DZ2[b * kHid + j] = dz2[j];
    }
    for (int j = 0; j < kHid; ++j) {
      float s = 0.f;
      for (int i = 0; i < kHid; ++i) s = fmaf(W[kOffW2 + i * kHid + j], dz2[i], s);
      DZ1[b * kHid + j] = H1[b * kHid + j] > 0.f ? s : 0.f;
    }
  }
}

// Weight gradients: one CTA per output row of a layer; thread j sums DZ[b][row] * H[b][j] over
// the batch in order (deterministic); thread 0 also sums the bias gradient.
__global__ void k_train_wgrad(int64_t B, const float* __restrict__ H0, const float* __restrict__ H1,
                              const float* __restrict__ H2, const float* __restrict__ A3, const float* __restrict__ GY,
                              const float* __restrict__ DZ1, const float* __restrict__ DZ2,
                              const float* __restrict__ DZ3, float* __restrict__ G) {
  const int row = blockIdx.x;  // 0..63 layer 1, 64..127 layer 2, 128..191 layer 3, 192 layer 4
  const int layer = row / kHid;
  const int i = row % kHid;
  const float* H;
  const float* DZ;
  int K, offW, offB;
  if (layer == 0) { H = H0; DZ = DZ1; K = kIn; offW = kOffW1; offB = kOffB1; }
  else if (layer == 1) { H = H1; DZ = DZ2; K = kHid; offW = kOffW2; offB = kOffB2; }
  else if (layer == 2) { H = H2; DZ = DZ3; K = kHid; offW = kOffW3; offB = kOffB3; }
  else { H = A3; DZ = GY; K = kHid; offW = kOffW4; offB = kOffB4; }
  const int dzs = layer == 3 ? 1 : kHid;
  const int dzo = layer == 3 ? 0 : i;
  const int j = threadIdx.x;
  if (j < K) {
    float s = 0.f;
    for (int64_t b = 0; b < B; ++b) s = fmaf(DZ[b * dzs + dzo], H[b * K + j], s);
    G[offW + (layer == 3 ? j : i * K + j)] = s;
  }
  if (j == kHid) {
    float s = 0.f;
    for (int64_t b = 0; b < B; ++b) s += DZ[b * dzs + dzo];
    G[offB + (layer == 3 ? 0 : i)] = s;
  }
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M1,
                       float* __restrict__ M2, int n, float lr, float b1t, float b2t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float g = G[q];
  const float m = 0.9f * M1[q] + 0.1f * g;
  const float v = 0.999f * M2[q] + 0.001f * g * g;
  M1[q] = m;
  M2[q] = v;
  P[q] -= lr * (m / (1.f - b1t)) / (sqrtf(v / (1.f - b2t)) + 1e-8f);
}

__global__ void k_reduce_loss(const float* __restrict__ L, int64_t B, float* out) {
  __shared__ float red[256];
  float s = 0.f;
  for (int64_t b = threadIdx.x; b < B; b += blockDim.x) s += L[b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0] / (float)B;
}

// Training samples: nodes of the coarse grid (normalised) and their exact distances (normalised).
__global__ void k_make_samples(const double* __restrict__ dist, GridP g, double cx, double cy, double cz, double s,
                               float* __restrict__ X, float* __restrict__ T) {
  for (int64_t lin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; lin < g.ngp; lin += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = lin % g.n[0], j = (lin / g.n[0]) % g.n[1], k = lin / (g.n[0] * g.n[1]);
    const d3 p = gnode(g, i, j, k);
    X[3 * lin] = (float)((p.x - cx) / s);
    X[3 * lin + 1] = (float)((p.y - cy) / s);
    X[3 * lin + 2] = (float)((p.z - cz) / s);
    T[lin] = (float)(dist[lin] / s);
  }
}

__global__ void k_gather_batch(const float* __restrict__ X, const float* __restrict__ T,
                               const int32_t* __restrict__ perm, int64_t off, int64_t B, float* __restrict__ XB,
                               float* __restrict__ TB) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
    const int32_t q = perm[off + b];
    XB[3 * b] = X[3 * q]; XB[3 * b + 1] = X[3 * q + 1]; XB[3 * b + 2] = X[3 * q + 2];
    TB[b] = T[q];
  }
}

__global__ void k_to_half(const float* __restrict__ P, __half* __restrict__ WH) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < kParams) WH[q] = __float2half_rn(P[q]);
}

// ---- inference (mma.sync m16n8k16, FP16 x FP16 -> FP32) ---------------------------------------

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
  __half2 v = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// One layer for one 16-row m tile: acc[nt][4] = bias + A x W^T, W (64 x K) FP16 row-major in smem.
template <int KT>
__device__ __forceinline__ void mma_layer(const uint32_t a[KT][4], const __half* W, int K, const float* bias,
                                          float acc[8][4], int g, int t) {
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias[8 * nt + 2 * t], b1 = bias[8 * nt + 2 * t + 1];
    acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
#pragma unroll
    for (int kc = 0; kc < KT; ++kc) {
      const __half* w = W + (8 * nt + g) * K + 16 * kc + 2 * t;
      const uint32_t bf[2] = {*reinterpret_cast<const uint32_t*>(w), *reinterpret_cast<const uint32_t*>(w + 8)};
      mma16816(acc[nt], a[kc], bf);
    }
  }
}

// relu(acc) of two adjacent n8 tiles -> the A fragment of one k16 tile of the next layer.
__device__ __forceinline__ void acc_to_a(const float acc[8][4], uint32_t a[4][4]) {
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    a[kc][0] = pack_h2(fmaxf(acc[2 * kc][0], 0.f), fmaxf(acc[2 * kc][1], 0.f));
    a[kc][1] = pack_h2(fmaxf(acc[2 * kc][2], 0.f), fmaxf(acc[2 * kc][3], 0.f));
    a[kc][2] = pack_h2(fmaxf(acc[2 * kc + 1][0], 0.f), fmaxf(acc[2 * kc + 1][1], 0.f));
    a[kc][3] = pack_h2(fmaxf(acc[2 * kc + 1][2], 0.f), fmaxf(acc[2 * kc + 1][3], 0.f));
  }
}

struct RadiusArgs {
  GridP g;          // grid of the query (ngp nodes) -- or npts explicit normalised points
  const float* pts; // nullable: B x 3 normalised points instead of grid nodes
  int64_t count;
  double cx, cy, cz, s;
  float alpha, beta;  // r = (dhat (1 + alpha) + beta) * s; alpha < 0: write dhat itself
  const __half* WH;
  const float* P;     // FP32 params (biases)
  float* out;
};

// A warp evaluates 32 nodes; the CTA stages the FP16 weights and the FP32 biases once.
__global__ void __launch_bounds__(128) k_radius(RadiusArgs A) {
  __shared__ __align__(16) __half W[kOffB4];
  __shared__ float Bs[3 * kHid + kHid + 1];  // b1 b2 b3, w4, b4 (FP32; w4 rounded to half)
  __shared__ __align__(16) __half F[4][32][kIn + 8];  // per warp: features of its 32 nodes
  __shared__ float Y[4][32];
  for (int q = threadIdx.x; q < kOffB4; q += blockDim.x) W[q] = A.WH[q];
  for (int q = threadIdx.x; q < kHid; q += blockDim.x) {
    Bs[q] = A.P[kOffB1 + q];
    Bs[kHid + q] = A.P[kOffB2 + q];
    Bs[2 * kHid + q] = A.P[kOffB3 + q];
    Bs[3 * kHid + q] = __half2float(A.WH[kOffW4 + q]);
  }
  if (threadIdx.x == 0) Bs[4 * kHid] = A.P[kOffB4];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const GridP& G = A.g;
  for (int64_t base = ((int64_t)blockIdx.x * 4 + warp) * 32; base < A.count; base += (int64_t)gridDim.x * 128) {
    const int64_t q = base + lane;
    float x0 = 0.f, x1 = 0.f, x2 = 0.f;
    if (q < A.count) {
      if (A.pts) {
        x0 = A.pts[3 * q]; x1 = A.pts[3 * q + 1]; x2 = A.pts[3 * q + 2];
      } else {
        const int64_t i = q % G.n[0], j = (q / G.n[0]) % G.n[1], k = q / (G.n[0] * G.n[1]);
        const d3 p = node_coord(G.o, G.h, i, j, k);
        x0 = (float)((p.x - A.cx) / A.s); x1 = (float)((p.y - A.cy) / A.s); x2 = (float)((p.z - A.cz) / A.s);
      }
    }
    float f[kIn];
    features(x0, x1, x2, f);
#pragma unroll
    for (int j = 0; j < kIn; ++j) F[warp][lane][j] = __float2half_rn(f[j]);
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      uint32_t a1[2][4];
#pragma unroll
      for (int kc = 0; kc < 2; ++kc) {
        const __half* r0 = &F[warp][16 * mt + g][16 * kc + 2 * t];
        const __half* r1 = &F[warp][16 * mt + g + 8][16 * kc + 2 * t];
        a1[kc][0] = *reinterpret_cast<const uint32_t*>(r0);
        a1[kc][1] = *reinterpret_cast<const uint32_t*>(r1);
        a1[kc][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
        a1[kc][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
      }
      float acc[8][4];
      uint32_t a2[4][4];
      mma_layer<2>(a1, W + kOffW1, kIn, Bs, acc, g, t);
      acc_to_a(acc, a2);
      mma_layer<4>(a2, W + kOffW2, kHid, Bs + kHid, acc, g, t);
      acc_to_a(acc, a2);
      mma_layer<4>(a2, W + kOffW3, kHid, Bs + 2 * kHid, acc, g, t);
      // last layer on CUDA cores: rows g and g+8, columns 8 nt + 2t, +1
      float y0 = 0.f, y1 = 0.f;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const float w0 = Bs[3 * kHid + 8 * nt + 2 * t], w1 = Bs[3 * kHid + 8 * nt + 2 * t + 1];
        y0 = fmaf(w0, fmaxf(acc[nt][0], 0.f), fmaf(w1, fmaxf(acc[nt][1], 0.f), y0));
        y1 = fmaf(w0, fmaxf(acc[nt][2], 0.f), fmaf(w1, fmaxf(acc[nt][3], 0.f), y1));
      }
      y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
      y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
      y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
      y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
      if (t == 0) {
        Y[warp][16 * mt + g] = y0 + Bs[4 * kHid];
        Y[warp][16 * mt + g + 8] = y1 + Bs[4 * kHid];
      }
    }
    __syncwarp();
    if (q < A.count) {
      const float dh = softplus(Y[warp][lane]);
      A.out[q] = A.alpha < 0.f ? dh : (float)((dh * (1.f + A.alpha) + A.beta) * A.s);
    }
    __syncwarp();
  }
}

}  // namespace

int radius_params_init(sdfgpu_ctx* ctx, uint64_t seed) {
  // He-style uniform initialisation from a 64-bit LCG (deterministic per seed).
  std::vector<float> P(kParams, 0.f);
  uint64_t st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  auto rnd = [&]() {
    st = st * 6364136223846793005ULL + 1442695040888963407ULL;
    return ((st >> 40) & 0xFFFFFF) / 16777216.0f * 2.f - 1.f;
  };
  auto fill = [&](int off, int rows, int cols) {
    const float lim = std::sqrt(6.f / (float)cols);
    for (int q = 0; q < rows * cols; ++q) P[off + q] = lim * rnd();
  };
  fill(kOffW1, kHid, kFeat);  // padded feature columns stay zero
  for (int i = 0; i < kHid; ++i)
    for (int j = kFeat; j < kIn; ++j) P[kOffW1 + i * kIn + j] = 0.f;
  fill(kOffW2, kHid, kHid);
  fill(kOffW3, kHid, kHid);
  fill(kOffW4, 1, kHid);
  for (int q = 0; q < kHid; ++q) P[kOffW4 + q] *= 0.1f;
  float* dP;
  SDF_TRY(scratch_t(ctx, "mlp_p", kParams, &dP));
  SDF_CUDA(ctx, cudaMemcpyAsync(dP, P.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, ctx->stream));
  return 0;
}

// Forward (+ backward) of the training definition over B host samples; for gradient checks.
int mlp_eval_host(sdfgpu_ctx* ctx, const float* params, const float* xn, const float* target, int64_t B, float* yhat,
                  float* loss, float* grad) {
  cudaStream_t st = ctx->stream;
  float *dP, *dX, *dT, *H0, *H1, *H2, *A3, *GY, *LS, *YH, *DZ1, *DZ2, *DZ3, *G, *dl;
  SDF_TRY(scratch_t(ctx, "mlpe_p", kParams, &dP));
  SDF_TRY(scratch_t(ctx, "mlpe_x", (size_t)B * 3, &dX));
  SDF_TRY(scratch_t(ctx, "mlpe_t", (size_t)B, &dT));
  SDF_TRY(scratch_t(ctx, "mlpe_h0", (size_t)B * kIn, &H0));
  SDF_TRY(scratch_t(ctx, "mlpe_h1", (size_t)B * kHid, &H1));
  SDF_TRY(scratch_t(ctx, "mlpe_h2", (size_t)B * kHid, &H2));
  SDF_TRY(scratch_t(ctx, "mlpe_a3", (size_t)B * kHid, &A3));
  SDF_TRY(scratch_t(ctx, "mlpe_gy", (size_t)B, &GY));
  SDF_TRY(scratch_t(ctx, "mlpe_ls", (size_t)B, &LS));
  SDF_TRY(scratch_t(ctx, "mlpe_yh", (size_t)B, &YH));
  SDF_TRY(scratch_t(ctx, "mlpe_dz1", (size_t)B * kHid, &DZ1));
  SDF_TRY(scratch_t(ctx, "mlpe_dz2", (size_t)B * kHid, &DZ2));
  SDF_TRY(scratch_t(ctx, "mlpe_dz3", (size_t)B * kHid, &DZ3));
  SDF_TRY(scratch_t(ctx, "mlpe_g", kParams, &G));
  SDF_TRY(scratch_t(ctx, "mlpe_l", 1, &dl));
  SDF_CUDA(ctx, cudaMemcpyAsync(dP, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(dX, xn, sizeof(float) * 3 * B, cudaMemcpyHostToDevice, st));
  if (target) SDF_CUDA(ctx, cudaMemcpyAsync(dT, target, sizeof(float) * B, cudaMemcpyHostToDevice, st));
  k_train_fwd<<<grid_for(B, 128), 128, 0, st>>>(dP, dX, target ? dT : nullptr, B, H0, H1, H2, A3, GY, LS, YH);
  SDF_KERNEL(ctx);
  if (target) {
    k_reduce_loss<<<1, 256, 0, st>>>(LS, B, dl);
    SDF_KERNEL(ctx);
    if (grad) {
      k_train_bwd<<<grid_for(B, 128), 128, 0, st>>>(dP, B, H1, H2, A3, GY, DZ1, DZ2, DZ3);
      SDF_KERNEL(ctx);
      k_train_wgrad<<<3 * kHid + 1, 96, 0, st>>>(B, H0, H1, H2, A3, GY, DZ1, DZ2, DZ3, G);
      SDF_KERNEL(ctx);
      SDF_CUDA(ctx, cudaMemcpyAsync(grad, G, sizeof(float) * kParams, cudaMemcpyDeviceToHost, st));
    }
    if (loss) SDF_CUDA(ctx, cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, st));
  }
  if (yhat) SDF_CUDA(ctx, cudaMemcpyAsync(yhat, YH, sizeof(float) * B, cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  return 0;
}

// Trains the radius network on the exact unbounded distances of a coarse grid of the mesh.
int train_radius(sdfgpu_ctx* ctx, int coarse_n, int steps, int batch, float lr, uint64_t seed, float* final_loss) {
  cudaStream_t st = ctx->stream;
  const MeshDev& M = ctx->mesh;
  // coarse grid: Grid(Xmin, Xmax, coarse_n - 7, 3), the rule of the workloads' grids
  double o[3], amax[3], h;
  int64_t N[3], ngp;
  {
    const double ext = std::max(M.bmax[0] - M.bmin[0], std::max(M.bmax[1] - M.bmin[1], M.bmax[2] - M.bmin[2]));
    h = ext / (double)(coarse_n - 7);
    ngp = 1;
    for (int a = 0; a < 3; ++a) {
      o[a] = M.bmin[a] - 3.0 * h;
      N[a] = (int64_t)std::ceil((M.bmax[a] + 3.0 * h - o[a]) / h);
      amax[a] = o[a] + (double)N[a] * h;
      ngp *= N[a] + 1;
    }
  }
  GridP g;
  SDF_TRY(make_grid(ctx, o, h, N, g));
  double* dd;
  SDF_TRY(scratch_t(ctx, "mlp_dist", (size_t)ngp, &dd));
  SDF_TRY(run_distances(ctx, g, SDFGPU_MODE_UNBOUNDED, 0, dd, nullptr));
  RadiusNorm& R = ctx->radius;
  R.c[0] = 0.5 * (o[0] + amax[0]);
  R.c[1] = 0.5 * (o[1] + amax[1]);
  R.c[2] = 0.5 * (o[2] + amax[2]);
  R.s = 0.5 * std::max(amax[0] - o[0], std::max(amax[1] - o[1], amax[2] - o[2]));
  R.coarse_h = h;
  float *X, *T;
  SDF_TRY(scratch_t(ctx, "mlp_X", (size_t)ngp * 3, &X));
  SDF_TRY(scratch_t(ctx, "mlp_T", (size_t)ngp, &T));
  k_make_samples<<<grid_for(ngp, 256), 256, 0, st>>>(dd, g, R.c[0], R.c[1], R.c[2], R.s, X, T);
  SDF_KERNEL(ctx);
  // deterministic shuffles (host LCG), uploaded once
  const int64_t B = std::min<int64_t>(batch, ngp);
  const int64_t per_epoch = ngp / B;
  std::vector<int32_t> perm((size_t)ngp);
  for (int64_t q = 0; q < ngp; ++q) perm[q] = (int32_t)q;
  uint64_t s64 = seed ^ 0x9E3779B97F4A7C15ULL;
  for (int64_t q = ngp - 1; q > 0; --q) {
    s64 = s64 * 6364136223846793005ULL + 1442695040888963407ULL;
    const int64_t r = (int64_t)((s64 >> 33) % (uint64_t)(q + 1));
    std::swap(perm[q], perm[r]);
  }
  int32_t* dperm;
  SDF_TRY(scratch_t(ctx, "mlp_perm", (size_t)ngp, &dperm));
  SDF_CUDA(ctx, cudaMemcpyAsync(dperm, perm.data(), sizeof(int32_t) * ngp, cudaMemcpyHostToDevice, st));
  SDF_TRY(radius_params_init(ctx, seed));
  float *P, *M1, *M2, *XB, *TB, *H0, *H1, *H2, *A3, *GY, *LS, *DZ1, *DZ2, *DZ3, *G, *dl;
  P = buf<float>(ctx, "mlp_p");
  SDF_TRY(scratch_t(ctx, "mlp_m1", kParams, &M1));
  SDF_TRY(scratch_t(ctx, "mlp_m2", kParams, &M2));
  SDF_TRY(scratch_t(ctx, "mlp_xb", (size_t)B * 3, &XB));
  SDF_TRY(scratch_t(ctx, "mlp_tb", (size_t)B, &TB));
  SDF_TRY(scratch_t(ctx, "mlp_h0", (size_t)B * kIn, &H0));
  SDF_TRY(scratch_t(ctx, "mlp_h1", (size_t)B * kHid, &H1));
  SDF_TRY(scratch_t(ctx, "mlp_h2", (size_t)B * kHid, &H2));
  SDF_TRY(scratch_t(ctx, "mlp_a3", (size_t)B * kHid, &A3));
  SDF_TRY(scratch_t(ctx, "mlp_gy", (size_t)B, &GY));
  SDF_TRY(scratch_t(ctx, "mlp_ls", (size_t)B, &LS));
  SDF_TRY(scratch_t(ctx, "mlp_dz1", (size_t)B * kHid, &DZ1));
  SDF_TRY(scratch_t(ctx, "mlp_dz2", (size_t)B * kHid, &DZ2));
  SDF_TRY(scratch_t(ctx, "mlp_dz3", (size_t)B * kHid, &DZ3));
  SDF_TRY(scratch_t(ctx, "mlp_g", kParams, &G));
  SDF_TRY(scratch_t(ctx, "mlp_l", 1, &dl));
  SDF_CUDA(ctx, cudaMemsetAsync(M1, 0, sizeof(float) * kParams, st));
  SDF_CUDA(ctx, cudaMemsetAsync(M2, 0, sizeof(float) * kParams, st));
  float b1t = 1.f, b2t = 1.f;
  for (int it = 0; it < steps; ++it) {
    const int64_t off = (it % per_epoch) * B;
    k_gather_batch<<<grid_for(B, 256), 256, 0, st>>>(X, T, dperm, off, B, XB, TB);
    SDF_KERNEL(ctx);
    k_train_fwd<<<grid_for(B, 128), 128, 0, st>>>(P, XB, TB, B, H0, H1, H2, A3, GY, LS, nullptr);
    SDF_KERNEL(ctx);
    k_train_bwd<<<grid_for(B, 128), 128, 0, st>>>(P, B, H1, H2, A3, GY, DZ1, DZ2, DZ3);
    SDF_KERNEL(ctx);
    k_train_wgrad<<<3 * kHid + 1, 96, 0, st>>>(B, H0, H1, H2, A3, GY, DZ1, DZ2, DZ3, G);
    SDF_KERNEL(ctx);
    b1t *= 0.9f;
    b2t *= 0.999f;
    const float lr_t = lr * 0.5f * (1.f + std::cos(3.14159265f * (float)it / (float)steps));  // cosine decay
    k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(P, G, M1, M2, kParams, lr_t, b1t, b2t);
    SDF_KERNEL(ctx);
  }
  // final loss over the first batch of the shuffle
  k_gather_batch<<<grid_for(B, 256), 256, 0, st>>>(X, T, dperm, 0, B, XB, TB);
  SDF_KERNEL(ctx);
  k_train_fwd<<<grid_for(B, 128), 128, 0, st>>>(P, XB, TB, B, H0, H1, H2, A3, GY, LS, nullptr);
  SDF_KERNEL(ctx);
  k_reduce_loss<<<1, 256, 0, st>>>(LS, B, dl);
  SDF_KERNEL(ctx);
  __half* WH;
  SDF_TRY(scratch_t(ctx, "mlp_wh", kParams, &WH));
  k_to_half<<<(kParams + 255) / 256, 256, 0, st>>>(P, WH);
  SDF_KERNEL(ctx);
  float l = 0.f;
  SDF_CUDA(ctx, cudaMemcpyAsync(&l, dl, sizeof(float), cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  R.trained = true;
  R.loss = l;
  if (final_loss) *final_loss = l;
  return 0;
}

int set_radius_params(sdfgpu_ctx* ctx, const float* params, const double norm[4]) {
  cudaStream_t st = ctx->stream;
  float* P;
  __half* WH;
  SDF_TRY(scratch_t(ctx, "mlp_p", kParams, &P));
  SDF_TRY(scratch_t(ctx, "mlp_wh", kParams, &WH));
  SDF_CUDA(ctx, cudaMemcpyAsync(P, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, st));
  k_to_half<<<(kParams + 255) / 256, 256, 0, st>>>(P, WH);
  SDF_KERNEL(ctx);
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  RadiusNorm& R = ctx->radius;
  R.c[0] = norm[0]; R.c[1] = norm[1]; R.c[2] = norm[2]; R.s = norm[3];
  R.trained = true;
  return 0;
}

int get_radius_params(sdfgpu_ctx* ctx, float* params, double norm[4]) {
  const RadiusNorm& R = ctx->radius;
  if (!R.trained) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "no radius network: call sdfgpu_train_radius first");
  SDF_CUDA(ctx, cudaMemcpyAsync(params, buf<float>(ctx, "mlp_p"), sizeof(float) * kParams, cudaMemcpyDeviceToHost,
                                ctx->stream));
  SDF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  norm[0] = R.c[0]; norm[1] = R.c[1]; norm[2] = R.c[2]; norm[3] = R.s;
  return 0;
}

// Radii (or raw dhat when alpha < 0) of the grid nodes, or of explicit normalised points.
int run_radius(sdfgpu_ctx* ctx, const GridP* g, const float* d_pts, int64_t count, float alpha, float beta, float* d_out) {
  const RadiusNorm& R = ctx->radius;
  if (!R.trained) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "no radius network: call sdfgpu_train_radius first");
  RadiusArgs A;
  if (g) A.g = *g;
  else std::memset(&A.g, 0, sizeof(A.g));
  A.pts = d_pts;
  A.count = count;
  A.cx = R.c[0]; A.cy = R.c[1]; A.cz = R.c[2]; A.s = R.s;
  A.alpha = alpha;
  A.beta = beta;
  A.WH = buf<__half>(ctx, "mlp_wh");
  A.P = buf<float>(ctx, "mlp_p");
  A.out = d_out;
  k_radius<<<grid_for(count, 128, 148 * 16), 128, 0, ctx->stream>>>(A);
  SDF_KERNEL(ctx);
  return 0;
}

}  // namespace sdfgpu
