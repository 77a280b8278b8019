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

// ---- training (mma.sync m16n8k16, FP16 operands, FP32 accumulate) ------------------------------
//
// One step = k_train_step + k_train_reduce.  k_train_step: every CTA takes kTS samples of the
// step's batch (4 warps x 32).  A warp runs the forward of its 32 samples as three 64-wide GEMM
// layers on the tensor cores (the inference kernel's fragments), the loss and dL/dy, then the
// backward input gradients dZ3 -> dZ2 -> dZ1 as two more GEMMs (dH = dZ W, W read transposed from
// shared memory), staging every activation and every dZ in shared memory as FP16.  Then each warp
// forms a 16-row slice of every weight gradient dW = dZ^T H as GEMMs over the CTA's kTS samples,
// and the CTA writes its partial gradient (and partial loss) to global memory.  k_train_reduce sums
// the partials of all CTAs in a fixed order (deterministic), rescales, and applies Adam.
//
// dL/dy is carried scaled by kGyScale instead of 1/B so the FP16 dZ stay in range; the reduce
// multiplies by 1 / (kGyScale B).  dZ beyond the FP16 range are clamped (only possible far from a
// trained state; the gradient then stays finite).
constexpr int kTS = 128;                 // samples per CTA
constexpr float kGyScale = 1.f / 256.f;  // per-sample dL/dy scale inside the step
constexpr int kLd1 = kIn + 8;            // shared-memory row strides in halves (padding against bank conflicts)
constexpr int kLdH = kHid + 8;
constexpr int kPart = kParams + 1;       // partial gradient of one CTA + its loss sum

struct TrainSmem {
  __half W1[kHid * kLd1];  // row major [out][in], FP16-rounded weights
  __half W2[kHid * kLdH];
  __half W3[kHid * kLdH];
  float b1[kHid], b2[kHid], b3[kHid], w4[kHid];
  float b4;
  __half H0[kTS * kLd1];   // per sample: features, h1, h2 (the forward's FP16 activations)
  __half H1[kTS * kLdH];
  __half H2[kTS * kLdH];
  __half D1[kTS * kLdH];   // per sample: dZ1, dZ2, dZ3 (scaled by kGyScale)
  __half D2[kTS * kLdH];
  __half D3[kTS * kLdH];
  float gw4[4][kHid];
  float red[4][2];         // per warp: sum of dL/dy (b4) and of the loss terms
};

__device__ __forceinline__ uint32_t pack_hh(__half lo, __half hi) {
  __half2 v = __halves2half2(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float hclamp(float x) { return fminf(fmaxf(x, -60000.f), 60000.f); }

// Accumulators of two adjacent n8 tiles -> the A fragment of one k16 tile (no activation).
__device__ __forceinline__ void acc_to_a_raw(const float acc[8][4], uint32_t a[4][4]) {
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    a[kc][0] = pack_h2(hclamp(acc[2 * kc][0]), hclamp(acc[2 * kc][1]));
    a[kc][1] = pack_h2(hclamp(acc[2 * kc][2]), hclamp(acc[2 * kc][3]));
    a[kc][2] = pack_h2(hclamp(acc[2 * kc + 1][0]), hclamp(acc[2 * kc + 1][1]));
    a[kc][3] = pack_h2(hclamp(acc[2 * kc + 1][2]), hclamp(acc[2 * kc + 1][3]));
  }
}

// Store an accumulator fragment (rows r0 and r0 + 8 of the tile) as FP16 into a row-major array.
__device__ __forceinline__ void store_acc(__half* M, int ld, int r0, const uint32_t a[4][4], int t) {
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    *reinterpret_cast<uint32_t*>(M + r0 * ld + 16 * kc + 2 * t) = a[kc][0];
    *reinterpret_cast<uint32_t*>(M + (r0 + 8) * ld + 16 * kc + 2 * t) = a[kc][1];
    *reinterpret_cast<uint32_t*>(M + r0 * ld + 16 * kc + 8 + 2 * t) = a[kc][2];
    *reinterpret_cast<uint32_t*>(M + (r0 + 8) * ld + 16 * kc + 8 + 2 * t) = a[kc][3];
  }
}

// acc = dZ (16 x 64, A fragments) x W (64 x 64 row major [out][in]): dH[s][in] = sum_out dZ[s][out] W[out][in].
__device__ __forceinline__ void mma_back(const uint32_t a[4][4], const __half* W, float acc[8][4], int g, int t) {
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      const int k0 = 16 * kc + 2 * t, n = 8 * nt + g;
      const uint32_t bf[2] = {pack_hh(W[k0 * kLdH + n], W[(k0 + 1) * kLdH + n]),
                              pack_hh(W[(k0 + 8) * kLdH + n], W[(k0 + 9) * kLdH + n])};
      mma16816(acc[nt], a[kc], bf);
    }
  }
}

// dZ masked by the activation of the forward (unit active when its stored FP16 output is > 0).
__device__ __forceinline__ void mask_by(float acc[8][4], const __half* H, int r0, int t) {
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int c = 8 * nt + 2 * t;
    if (!(__half2float(H[r0 * kLdH + c]) > 0.f)) acc[nt][0] = 0.f;
    if (!(__half2float(H[r0 * kLdH + c + 1]) > 0.f)) acc[nt][1] = 0.f;
    if (!(__half2float(H[(r0 + 8) * kLdH + c]) > 0.f)) acc[nt][2] = 0.f;
    if (!(__half2float(H[(r0 + 8) * kLdH + c + 1]) > 0.f)) acc[nt][3] = 0.f;
  }
}

// dW rows [16 w, 16 w + 16) of one layer: sum over the CTA's kTS samples of dZ[s][out] H[s][in]
// (A = dZ^T, B = H), written to the CTA's partial at offW (row stride K).
template <int NT>
__device__ __forceinline__ void wgrad_rows(const __half* D, const __half* H, int ldh, int K, int w, int g, int t,
                                           float* out) {
  float acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
  const int o = 16 * w + g;
#pragma unroll 2
  for (int kk = 0; kk < kTS / 16; ++kk) {
    const int s0 = 16 * kk + 2 * t;
    const uint32_t a[4] = {pack_hh(D[s0 * kLdH + o], D[(s0 + 1) * kLdH + o]),
                           pack_hh(D[s0 * kLdH + o + 8], D[(s0 + 1) * kLdH + o + 8]),
                           pack_hh(D[(s0 + 8) * kLdH + o], D[(s0 + 9) * kLdH + o]),
                           pack_hh(D[(s0 + 8) * kLdH + o + 8], D[(s0 + 9) * kLdH + o + 8])};
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int n = 8 * nt + g;
      const uint32_t bf[2] = {pack_hh(H[s0 * ldh + n], H[(s0 + 1) * ldh + n]),
                              pack_hh(H[(s0 + 8) * ldh + n], H[(s0 + 9) * ldh + n])};
      mma16816(acc[nt], a, bf);
    }
  }
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int c = 8 * nt + 2 * t;
    out[o * K + c] = acc[nt][0];
    out[o * K + c + 1] = acc[nt][1];
    out[(o + 8) * K + c] = acc[nt][2];
    out[(o + 8) * K + c + 1] = acc[nt][3];
  }
}

// Forward, loss and backward of kTS samples per CTA; writes the CTA's partial gradient.  Sample q of
// the step is X[perm[off + q]] (perm may be NULL: X[q]); samples q >= B contribute nothing.
// dhat_out / loss_out (nullable) receive the per-sample network output and loss term.
__global__ void __launch_bounds__(128) k_train_step(const float* __restrict__ P, const float* __restrict__ X,
                                                    const float* __restrict__ T, const int32_t* __restrict__ perm,
                                                    int64_t off, int64_t B, float* __restrict__ partial,
                                                    float* __restrict__ dhat_out, float* __restrict__ loss_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
  for (int q = threadIdx.x; q < kHid * kIn; q += blockDim.x)
    S.W1[(q / kIn) * kLd1 + q % kIn] = __float2half_rn(P[kOffW1 + q]);
  for (int q = threadIdx.x; q < kHid * kHid; q += blockDim.x) {
    S.W2[(q / kHid) * kLdH + q % kHid] = __float2half_rn(P[kOffW2 + q]);
    S.W3[(q / kHid) * kLdH + q % kHid] = __float2half_rn(P[kOffW3 + q]);
  }
  for (int q = threadIdx.x; q < kHid; q += blockDim.x) {
    S.b1[q] = P[kOffB1 + q];
    S.b2[q] = P[kOffB2 + q];
    S.b3[q] = P[kOffB3 + q];
    S.w4[q] = h16(P[kOffW4 + q]);
  }
  if (threadIdx.x == 0) S.b4 = P[kOffB4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int64_t cbase = (int64_t)blockIdx.x * kTS;
  {  // features of this warp's 32 samples
    const int sl = 32 * warp + lane;
    const int64_t q = cbase + sl;
    float x0 = 0.f, x1 = 0.f, x2 = 0.f;
    if (q < B) {
      const int64_t src = perm ? (int64_t)perm[off + q] : q;
      x0 = X[3 * src]; x1 = X[3 * src + 1]; x2 = X[3 * src + 2];
    }
    float f[kIn];
    features(x0, x1, x2, f);
#pragma unroll
    for (int j = 0; j < kIn; ++j) S.H0[sl * kLd1 + j] = __float2half_rn(f[j]);
  }
  __syncthreads();
  float gw4[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) gw4[nt][0] = gw4[nt][1] = 0.f;
  float gb4 = 0.f, lsum = 0.f;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = 32 * warp + 16 * mt + g;  // this thread's rows r0 and r0 + 8 (CTA-local samples)
    uint32_t a1[2][4];
#pragma unroll
    for (int kc = 0; kc < 2; ++kc) {
      const __half* p0 = &S.H0[r0 * kLd1 + 16 * kc + 2 * t];
      const __half* p1 = &S.H0[(r0 + 8) * kLd1 + 16 * kc + 2 * t];
      a1[kc][0] = *reinterpret_cast<const uint32_t*>(p0);
      a1[kc][1] = *reinterpret_cast<const uint32_t*>(p1);
      a1[kc][2] = *reinterpret_cast<const uint32_t*>(p0 + 8);
      a1[kc][3] = *reinterpret_cast<const uint32_t*>(p1 + 8);
    }
    float acc[8][4];
    uint32_t a2[4][4];
    mma_layer<2>(a1, S.W1, kLd1, S.b1, acc, g, t);
    acc_to_a(acc, a2);
    store_acc(S.H1, kLdH, r0, a2, t);
    mma_layer<4>(a2, S.W2, kLdH, S.b2, acc, g, t);
    acc_to_a(acc, a2);
    store_acc(S.H2, kLdH, r0, a2, t);
    mma_layer<4>(a2, S.W3, kLdH, S.b3, acc, g, t);
    // a3 = relu(acc); y = w4 . a3 + b4 for rows r0 (y0) and r0 + 8 (y1)
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[nt][e] = fmaxf(acc[nt][e], 0.f);
      const float w0 = S.w4[8 * nt + 2 * t], w1 = S.w4[8 * nt + 2 * t + 1];
      y0 = fmaf(w0, acc[nt][0], fmaf(w1, acc[nt][1], y0));
      y1 = fmaf(w0, acc[nt][2], fmaf(w1, acc[nt][3], y1));
    }
    y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
    y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
    float gy[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float y = (h == 0 ? y0 : y1) + S.b4;
      const int64_t q = cbase + r0 + 8 * h;
      float gq = 0.f;
      if (q < B) {
        const float dh = softplus(y);
        if (dhat_out && t == 0) dhat_out[q] = dh;
        if (T) {  // without targets (outputs only) nothing flows back
          const float tq = T[perm ? (int64_t)perm[off + q] : q];
          const float r = logf(dh + kLogEps) - logf(tq + kLogEps);
          gq = 2.f * r / (dh + kLogEps) * sigmoid(y) * kGyScale;
          if (t == 0) {
            lsum += r * r;
            gb4 += gq;
            if (loss_out) loss_out[q] = r * r;
          }
        }
      }
      gy[h] = gq;
    }
    // dZ3 = [a3 > 0] gy w4, and the w4 gradient gy a3
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float w0 = S.w4[8 * nt + 2 * t], w1 = S.w4[8 * nt + 2 * t + 1];
      gw4[nt][0] = fmaf(gy[0], acc[nt][0], fmaf(gy[1], acc[nt][2], gw4[nt][0]));
      gw4[nt][1] = fmaf(gy[0], acc[nt][1], fmaf(gy[1], acc[nt][3], gw4[nt][1]));
      acc[nt][0] = acc[nt][0] > 0.f ? gy[0] * w0 : 0.f;
      acc[nt][1] = acc[nt][1] > 0.f ? gy[0] * w1 : 0.f;
      acc[nt][2] = acc[nt][2] > 0.f ? gy[1] * w0 : 0.f;
      acc[nt][3] = acc[nt][3] > 0.f ? gy[1] * w1 : 0.f;
    }
    uint32_t ad[4][4];
    acc_to_a_raw(acc, ad);
    store_acc(S.D3, kLdH, r0, ad, t);
    __syncwarp();
    mma_back(ad, S.W3, acc, g, t);  // dH2
    mask_by(acc, S.H2, r0, t);      // dZ2
    acc_to_a_raw(acc, ad);
    store_acc(S.D2, kLdH, r0, ad, t);
    mma_back(ad, S.W2, acc, g, t);  // dH1
    mask_by(acc, S.H1, r0, t);      // dZ1
    acc_to_a_raw(acc, ad);
    store_acc(S.D1, kLdH, r0, ad, t);
  }
  // w4 gradient: sum over the 8 row groups g of the warp, then over the warps
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      float v = gw4[nt][e];
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 8);
      v += __shfl_xor_sync(0xffffffffu, v, 16);
      if (g == 0) S.gw4[warp][8 * nt + 2 * t + e] = v;
    }
  for (int off2 = 16; off2 > 0; off2 >>= 1) {
    gb4 += __shfl_xor_sync(0xffffffffu, gb4, off2);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, off2);
  }
  if (lane == 0) {
    S.red[warp][0] = gb4;
    S.red[warp][1] = lsum;
  }
  __syncthreads();
  float* out = partial + (int64_t)blockIdx.x * kPart;
  wgrad_rows<8>(S.D3, S.H2, kLdH, kHid, warp, g, t, out + kOffW3);
  wgrad_rows<8>(S.D2, S.H1, kLdH, kHid, warp, g, t, out + kOffW2);
  wgrad_rows<4>(S.D1, S.H0, kLd1, kIn, warp, g, t, out + kOffW1);
  for (int q = threadIdx.x; q < 3 * kHid; q += blockDim.x) {  // bias gradients: sums of dZ over the samples
    const int layer = q / kHid, o = q % kHid;
    const __half* D = layer == 0 ? S.D1 : (layer == 1 ? S.D2 : S.D3);
    float s = 0.f;
    for (int sl = 0; sl < kTS; ++sl) s += __half2float(D[sl * kLdH + o]);
    out[(layer == 0 ? kOffB1 : (layer == 1 ? kOffB2 : kOffB3)) + o] = s;
  }
  if (threadIdx.x < kHid)
    out[kOffW4 + threadIdx.x] =
        S.gw4[0][threadIdx.x] + S.gw4[1][threadIdx.x] + S.gw4[2][threadIdx.x] + S.gw4[3][threadIdx.x];
  if (threadIdx.x == 0) {
    out[kOffB4] = S.red[0][0] + S.red[1][0] + S.red[2][0] + S.red[3][0];
    out[kParams] = S.red[0][1] + S.red[1][1] + S.red[2][1] + S.red[3][1];
  }
}

// Sums the CTAs' partials in CTA order, scales them to dL/dP, and (adam = 1) applies one Adam step
// at learning rate lr with the bias corrections b1t = 0.9^t, b2t = 0.999^t; G (nullable) receives
// the gradient and *loss (nullable) the mean loss of the step.
__global__ void k_train_reduce(const float* __restrict__ partial, int nparts, int64_t B, float* __restrict__ P,
                               float* __restrict__ M1, float* __restrict__ M2, int adam, float lr, float b1t,
                               float b2t, float* __restrict__ G, float* __restrict__ loss) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q > kParams) return;
  float s = 0.f;
  for (int c = 0; c < nparts; ++c) s += partial[(int64_t)c * kPart + q];
  if (q == kParams) {
    if (loss) *loss = s / (float)B;
    return;
  }
  const float gq = s / (kGyScale * (float)B);
  if (G) G[q] = gq;
  if (!adam) return;
  const float m = 0.9f * M1[q] + 0.1f * gq;
  const float v = 0.999f * M2[q] + 0.001f * gq * gq;
  M1[q] = m;
  M2[q] = v;
  P[q] -= lr * (m / (1.f - b1t)) / (sqrtf(v / (1.f - b2t)) + 1e-8f);
}

struct RadiusArgs {
  GridP g;          // grid of the query (ngp nodes) -- or npts explicit normalised points
  const float* pts; // nullable: B x 3 normalised points instead of grid nodes
  int32_t b[3];     // b[0] > 0: the query is the centre of each warp brick of b nodes (nb per axis)
  int64_t nb[3];
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
        d3 p;
        if (A.b[0] > 0) {
          p = brick_center(G, A.b, q % A.nb[0], (q / A.nb[0]) % A.nb[1], q / (A.nb[0] * A.nb[1]));
        } else {
          p = gnode(G, q % G.n[0], (q / G.n[0]) % G.n[1], q / (G.n[0] * G.n[1]));
        }
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

// k_train_step's shared memory (~128 KB) is above the default 48 KB limit.
int train_smem_attr(sdfgpu_ctx* ctx) {
  SDF_CUDA(ctx, cudaFuncSetAttribute(k_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem)));
  return 0;
}

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

// The training step's forward (+ backward) over B host samples at host params, without the update;
// for checking the GPU gradients against a CPU implementation.
int mlp_eval_host(sdfgpu_ctx* ctx, const float* params, const float* xn, const float* target, int64_t B, float* yhat,
                  float* loss, float* grad) {
  cudaStream_t st = ctx->stream;
  float *dP, *dX, *dT = nullptr, *YH, *G, *dl, *part;
  const int nparts = (int)cdiv(B, kTS);
  SDF_TRY(scratch_t(ctx, "mlpe_p", kParams, &dP));
  SDF_TRY(scratch_t(ctx, "mlpe_x", (size_t)B * 3, &dX));
  if (target) SDF_TRY(scratch_t(ctx, "mlpe_t", (size_t)B, &dT));
  SDF_TRY(scratch_t(ctx, "mlpe_yh", (size_t)B, &YH));
  SDF_TRY(scratch_t(ctx, "mlpe_g", kParams, &G));
  SDF_TRY(scratch_t(ctx, "mlpe_l", 1, &dl));
  SDF_TRY(scratch_t(ctx, "mlpe_part", (size_t)nparts * kPart, &part));
  SDF_CUDA(ctx, cudaMemcpyAsync(dP, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(dX, xn, sizeof(float) * 3 * B, cudaMemcpyHostToDevice, st));
  if (target) SDF_CUDA(ctx, cudaMemcpyAsync(dT, target, sizeof(float) * B, cudaMemcpyHostToDevice, st));
  SDF_TRY(train_smem_attr(ctx));
  k_train_step<<<nparts, 128, sizeof(TrainSmem), st>>>(dP, dX, dT, nullptr, 0, B, part, YH, nullptr);
  SDF_KERNEL(ctx);
  k_train_reduce<<<(kPart + 255) / 256, 256, 0, st>>>(part, nparts, B, dP, nullptr, nullptr, 0, 0.f, 0.f, 0.f, G, dl);
  SDF_KERNEL(ctx);
  if (target && grad) SDF_CUDA(ctx, cudaMemcpyAsync(grad, G, sizeof(float) * kParams, cudaMemcpyDeviceToHost, st));
  if (target && loss) SDF_CUDA(ctx, cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, st));
  if (yhat) SDF_CUDA(ctx, cudaMemcpyAsync(yhat, YH, sizeof(float) * B, cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  return 0;
}

// Trains the radius network on the exact unbounded distances of a coarse grid of the mesh.
int train_radius(sdfgpu_ctx* ctx, int coarse_n, int steps, int batch, float lr, uint64_t seed, float* final_loss) {
  cudaStream_t st = ctx->stream;
  const MeshDev& M = ctx->mesh;
  // coarse grid: coarse_n - 1 cells on the longest axis of the mesh box, padded by one cell (the
  // workloads' grids pad by 3 of their own, much finer, cells); nodes far outside the box would only
  // make the training targets expensive
  double o[3], amax[3], h;
  int64_t N[3], ngp;
  {
    const double ext = std::max(M.bmax[0] - M.bmin[0], std::max(M.bmax[1] - M.bmin[1], M.bmax[2] - M.bmin[2]));
    h = ext / (double)(coarse_n - 3);
    ngp = 1;
    for (int a = 0; a < 3; ++a) {
      o[a] = M.bmin[a] - h;
      N[a] = (int64_t)std::ceil((M.bmax[a] + h - o[a]) / h);
      amax[a] = o[a] + (double)N[a] * h;
      ngp *= N[a] + 1;
    }
  }
  GridP g;
  SDF_TRY(make_grid(ctx, o, h, N, g));
  double* dd;
  SDF_TRY(scratch_t(ctx, "mlp_dist", (size_t)ngp, &dd));
  // the exact unbounded distances of the coarse grid (sparse nodes: one nearest-first walk per node)
  SDF_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev_obb, 0));
  SDF_TRY(run_nearest_points(ctx, g, dd));
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
  float *P, *M1, *M2, *part, *dl;
  const int nparts = (int)cdiv(B, kTS);
  P = buf<float>(ctx, "mlp_p");
  SDF_TRY(scratch_t(ctx, "mlp_m1", kParams, &M1));
  SDF_TRY(scratch_t(ctx, "mlp_m2", kParams, &M2));
  SDF_TRY(scratch_t(ctx, "mlp_part", (size_t)nparts * kPart, &part));
  SDF_TRY(scratch_t(ctx, "mlp_l", 1, &dl));
  SDF_CUDA(ctx, cudaMemsetAsync(M1, 0, sizeof(float) * kParams, st));
  SDF_CUDA(ctx, cudaMemsetAsync(M2, 0, sizeof(float) * kParams, st));
  SDF_TRY(train_smem_attr(ctx));
  float b1t = 1.f, b2t = 1.f;
  for (int it = 0; it < steps; ++it) {
    const int64_t off = (it % per_epoch) * B;
    k_train_step<<<nparts, 128, sizeof(TrainSmem), st>>>(P, X, T, dperm, off, B, part, nullptr, nullptr);
    SDF_KERNEL(ctx);
    b1t *= 0.9f;
    b2t *= 0.999f;
    const float lr_t = lr * 0.5f * (1.f + std::cos(3.14159265f * (float)it / (float)steps));  // cosine decay
    k_train_reduce<<<(kPart + 255) / 256, 256, 0, st>>>(part, nparts, B, P, M1, M2, 1, lr_t, b1t, b2t, nullptr,
                                                         nullptr);
    SDF_KERNEL(ctx);
  }
  // final loss over the first batch of the shuffle
  k_train_step<<<nparts, 128, sizeof(TrainSmem), st>>>(P, X, T, dperm, 0, B, part, nullptr, nullptr);
  SDF_KERNEL(ctx);
  k_train_reduce<<<(kPart + 255) / 256, 256, 0, st>>>(part, nparts, B, P, nullptr, nullptr, 0, 0.f, 0.f, 0.f, nullptr,
                                                       dl);
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
int run_radius(sdfgpu_ctx* ctx, const GridP* g, const float* d_pts, int64_t count, float alpha, float beta, float* d_out,
               const int32_t* brick) {
  const RadiusNorm& R = ctx->radius;
  if (!R.trained) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "no radius network: call sdfgpu_train_radius first");
  RadiusArgs A;
  if (g) A.g = *g;
  else std::memset(&A.g, 0, sizeof(A.g));
  A.pts = d_pts;
  A.count = count;
  for (int a = 0; a < 3; ++a) {
    A.b[a] = brick ? brick[a] : 0;
    A.nb[a] = brick && g ? cdiv(g->n[a], brick[a]) : 0;
  }
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
