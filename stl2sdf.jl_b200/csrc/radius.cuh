// radius.cuh -- parameter layout of the learned-radius network (see radius.cu).
#pragma once

#include <stdint.h>

namespace sdfgpu {

constexpr int kFreq = 4;                   // Fourier octaves
constexpr int kFeat = 3 + 6 * kFreq;       // 27 features
constexpr int kIn = 32;                    // features padded to two k16 tiles
constexpr int kHid = 64;                   // width of the three hidden layers
constexpr int kOffW1 = 0;                  // W1: kHid x kIn, row major (out x in)
constexpr int kOffB1 = kOffW1 + kHid * kIn;
constexpr int kOffW2 = kOffB1 + kHid;      // W2: kHid x kHid
constexpr int kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;      // W3: kHid x kHid
constexpr int kOffB3 = kOffW3 + kHid * kHid;
constexpr int kOffW4 = kOffB3 + kHid;      // w4: kHid
constexpr int kOffB4 = kOffW4 + kHid;      // b4: 1
constexpr int kParams = kOffB4 + 1;        // 10497
constexpr float kLogEps = 1e-3f;           // loss: (log(dhat + eps) - log(d + eps))^2

// Normalisation x = (p - c) / s of the trained network and its training-grid spacing.
struct RadiusNorm {
  double c[3] = {0, 0, 0};
  double s = 1.0;
  double coarse_h = 0.0;
  float loss = 0.f;
  bool trained = false;
  float alpha = 0.5f;  // radius margin: r = (dhat (1 + alpha) + beta coarse_h / s) s; the fastest
  float beta = 4.0f;   // measured (tighter margins leave nodes uncertified, and those search twice)
  // options of the last training (what a SDFGPU_MODE_LEARNED batch trains every mesh with)
  int train_coarse = 24, train_steps = 50, train_batch = 2048;
  float train_lr = 5e-3f;
  uint64_t train_seed = 0;
};

}  // namespace sdfgpu
