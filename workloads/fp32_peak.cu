// fp32_peak.cu -- measured FP32 CUDA-core throughput of the device, the denominator of the hot
// path's FP32 roofline (nodes/s bound = FP32 FLOP/s / algorithmic FLOPs per node).  A measurement
// probe of the benchmark, built into workloads/_build/libfp32peak.so, not part of libsdfgpu.so.
//
// Every thread runs kChains independent FMA chains (enough to cover the FMA pipe's latency) for
// `iters` iterations; the grid fills every SM at full occupancy.  FLOPs = 2 per FMA.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_fma_peak(float seed, int iters, float* sink) {
  float a[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) a[c] = seed + (float)(threadIdx.x + c);
  const float x = 0.999999f, y = 1.0e-7f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int c = 0; c < kChains; ++c) a[c] = fmaf(a[c], x, y);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += a[c];
  if (s == 1234.5678f) sink[blockIdx.x] = s;  // keeps the chains live; never true in practice
}

}  // namespace

// 0 = ok, 1 = bad argument, 2 = no such device, 3 = a CUDA call failed.
extern "C" int fp32_peak_tflops(int32_t device, double* tflops) {
  if (!tflops) return 1;
  *tflops = 0.0;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return 2;
  int sms = 0, per_sm = 0;
  int rc = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float* sink = nullptr;
  const int iters = 2048;
  do {
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_peak, kThreads, 0) != cudaSuccess) {
      rc = 3;
      break;
    }
    const int blocks = sms * std::max(per_sm, 1);
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaMalloc(&sink, sizeof(float) * blocks) != cudaSuccess) {
      rc = 3;
      break;
    }
    float best = 1e30f;
    for (int rep = 0; rep < 6 && rc == 0; ++rep) {  // first launch is a warm-up
      cudaEventRecord(e0, st);
      k_fma_peak<<<blocks, kThreads, 0, st>>>(1.0f, iters, sink);
      cudaEventRecord(e1, st);
      float ms = 0.f;
      if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = 3;
        break;
      }
      if (rep > 0) best = std::min(best, ms);
    }
    if (rc == 0) {
      const double flops = 2.0 * (double)blocks * kThreads * (double)iters * 16.0 * kChains;
      *tflops = flops / (best * 1e-3) / 1e12;
    }
  } while (false);
  if (sink) cudaFree(sink);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaSetDevice(prev);
  return rc;
}
