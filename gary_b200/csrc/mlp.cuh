// Cost-model network shape and parameter-block layout (mlp.cu).
#pragma once

namespace gary {
constexpr int kMlpIn = 6, kMlpH1 = 64, kMlpH2 = 64, kMlpOut = 4;
constexpr int kMlpMuX = 0, kMlpSdX = 6, kMlpMuY = 12, kMlpSdY = 16;
constexpr int kMlpW1 = 20;
constexpr int kMlpB1 = kMlpW1 + kMlpH1 * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpH1;
constexpr int kMlpB2 = kMlpW2 + kMlpH2 * kMlpH1;
constexpr int kMlpW3 = kMlpB2 + kMlpH2;
constexpr int kMlpB3 = kMlpW3 + kMlpOut * kMlpH2;
constexpr int kMlpParams = kMlpB3 + kMlpOut;      // 4888
constexpr int kMlpWeights = kMlpParams - kMlpW1;  // 4868 trainable

// One sample through the network (standardised units).  P: parameter block.
__device__ __forceinline__ void mlp_forward_one(const float *__restrict__ P, const float *x, float *h1,
                                                float *h2, float *y) {
  const float *W1 = P + kMlpW1, *b1 = P + kMlpB1, *W2 = P + kMlpW2, *b2 = P + kMlpB2,
              *W3 = P + kMlpW3, *b3 = P + kMlpB3;
  for (int i = 0; i < kMlpH1; ++i) {
    float a = b1[i];
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) a = fmaf(W1[i * kMlpIn + f], x[f], a);
    h1[i] = a > 0.f ? a : 0.f;
  }
  for (int j = 0; j < kMlpH2; ++j) {
    float a = b2[j];
#pragma unroll 8
    for (int i = 0; i < kMlpH1; ++i) a = fmaf(W2[j * kMlpH1 + i], h1[i], a);
    h2[j] = a > 0.f ? a : 0.f;
  }
#pragma unroll
  for (int k = 0; k < kMlpOut; ++k) {
    float a = b3[k];
#pragma unroll 8
    for (int j = 0; j < kMlpH2; ++j) a = fmaf(W3[k * kMlpH2 + j], h2[j], a);
    y[k] = a;
  }
}
}  // namespace gary
