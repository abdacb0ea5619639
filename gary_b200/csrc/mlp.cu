// The cost model: a 6 -> 64 -> 64 -> 4 multilayer perceptron (ReLU hidden
// layers, linear output), FP32, trained and run by the kernels below.
//
// Parameter block (floats), the layout every kernel and the file share:
//   [0, 20)        normalisation: mu_x[6], sd_x[6], mu_y[4], sd_y[4]
//   then W1[64][6], b1[64], W2[64][64], b2[64], W3[4][64], b3[4]
// The network maps standardised features x' = (x - mu_x) / sd_x to
// standardised targets y' = (y - mu_y) / sd_y; callers apply the scaling.
//
// Training kernels: one thread per sample runs the forward pass and the
// backward deltas into shared memory, then every thread accumulates the
// gradient of a stride of the weights over the block's samples and adds it
// to the global gradient once (one atomic per weight per block).  The loss
// is the mean squared error over the (sample, output) cells a mask selects:
// a sample carries a target only for the variant that was run on it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "internal.cuh"
#include "mlp.cuh"
#include "warp_ops.cuh"

namespace gary {
namespace {

constexpr int kGradSamples = 64;  // samples per block in the gradient kernel
constexpr int kGradThreads = 128;

// y[n][4] = network(x[n][6]) in standardised units (normalisation applied
// here when `scale` is set: x is raw, y is returned raw).
__global__ void k_mlp_forward(const float *__restrict__ params, const float *__restrict__ x,
                              uint64_t n, int scale, float *__restrict__ y) {
  __shared__ float P[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  float h1[kMlpH1], h2[kMlpH2];
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n;
       s += (uint64_t)gridDim.x * blockDim.x) {
    float xi[kMlpIn], yo[kMlpOut];
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) {
      const float v = x[s * kMlpIn + f];
      xi[f] = scale ? (v - P[kMlpMuX + f]) / P[kMlpSdX + f] : v;
    }
    mlp_forward_one(P, xi, h1, h2, yo);
#pragma unroll
    for (int k = 0; k < kMlpOut; ++k)
      y[s * kMlpOut + k] = scale ? yo[k] * P[kMlpSdY + k] + P[kMlpMuY + k] : yo[k];
  }
}

// Gradient of sum over masked cells of (y - t)^2 / norm, standardised units.
__global__ void __launch_bounds__(kGradThreads)
    k_mlp_grad(const float *__restrict__ params, const float *__restrict__ x,
               const float *__restrict__ t, const uint8_t *__restrict__ mask, uint64_t n,
               float norm, float *__restrict__ grad, float *__restrict__ loss) {
  extern __shared__ float sm[];
  float *P = sm;                                  // kMlpParams
  float *X = P + kMlpParams;                      // [S][6]
  float *H1 = X + kGradSamples * kMlpIn;          // [S][64]
  float *H2 = H1 + kGradSamples * kMlpH1;         // [S][64]
  float *D1 = H2 + kGradSamples * kMlpH2;         // [S][64] delta at layer-1 pre-activation
  float *D2 = D1 + kGradSamples * kMlpH1;         // [S][64]
  float *DY = D2 + kGradSamples * kMlpH2;         // [S][4]
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  const uint64_t s0 = (uint64_t)blockIdx.x * kGradSamples;
  const int ns = (int)(n - s0 < (uint64_t)kGradSamples ? n - s0 : (uint64_t)kGradSamples);
  float lsum = 0.f;
  if (threadIdx.x < kGradSamples) {
    const int s = threadIdx.x;
    float *xs = X + s * kMlpIn, *h1 = H1 + s * kMlpH1, *h2 = H2 + s * kMlpH2;
    float *d1 = D1 + s * kMlpH1, *d2 = D2 + s * kMlpH2, *dy = DY + s * kMlpOut;
    if (s < ns) {
      float y[kMlpOut];
#pragma unroll
      for (int f = 0; f < kMlpIn; ++f) xs[f] = x[(s0 + s) * kMlpIn + f];
      mlp_forward_one(P, xs, h1, h2, y);
      const uint8_t m = mask[s0 + s];
#pragma unroll
      for (int k = 0; k < kMlpOut; ++k) {
        const float e = ((m >> k) & 1) ? y[k] - t[(s0 + s) * kMlpOut + k] : 0.f;
        lsum += e * e;
        dy[k] = 2.f * e / norm;
      }
      const float *W3 = P + kMlpW3, *W2 = P + kMlpW2;
      for (int j = 0; j < kMlpH2; ++j) {
        float a = 0.f;
#pragma unroll
        for (int k = 0; k < kMlpOut; ++k) a = fmaf(W3[k * kMlpH2 + j], dy[k], a);
        d2[j] = h2[j] > 0.f ? a : 0.f;
      }
      for (int i = 0; i < kMlpH1; ++i) {
        float a = 0.f;
        for (int j = 0; j < kMlpH2; ++j) a = fmaf(W2[j * kMlpH1 + i], d2[j], a);
        d1[i] = h1[i] > 0.f ? a : 0.f;
      }
    } else {
      for (int f = 0; f < kMlpIn; ++f) xs[f] = 0.f;
      for (int i = 0; i < kMlpH1; ++i) h1[i] = d1[i] = 0.f;
      for (int j = 0; j < kMlpH2; ++j) h2[j] = d2[j] = 0.f;
      for (int k = 0; k < kMlpOut; ++k) dy[k] = 0.f;
    }
  }
  __syncthreads();
  // weight gradients: thread w sums over the block's samples
  for (int w = threadIdx.x; w < kMlpWeights; w += blockDim.x) {
    float g = 0.f;
    if (w < kMlpB1 - kMlpW1) {  // W1[i][f]
      const int i = w / kMlpIn, f = w % kMlpIn;
      for (int s = 0; s < kGradSamples; ++s) g = fmaf(D1[s * kMlpH1 + i], X[s * kMlpIn + f], g);
    } else if (w < kMlpW2 - kMlpW1) {  // b1[i]
      const int i = w - (kMlpB1 - kMlpW1);
      for (int s = 0; s < kGradSamples; ++s) g += D1[s * kMlpH1 + i];
    } else if (w < kMlpB2 - kMlpW1) {  // W2[j][i]
      const int r = w - (kMlpW2 - kMlpW1), j = r / kMlpH1, i = r % kMlpH1;
      for (int s = 0; s < kGradSamples; ++s) g = fmaf(D2[s * kMlpH2 + j], H1[s * kMlpH1 + i], g);
    } else if (w < kMlpW3 - kMlpW1) {  // b2[j]
      const int j = w - (kMlpB2 - kMlpW1);
      for (int s = 0; s < kGradSamples; ++s) g += D2[s * kMlpH2 + j];
    } else if (w < kMlpB3 - kMlpW1) {  // W3[k][j]
      const int r = w - (kMlpW3 - kMlpW1), k = r / kMlpH2, j = r % kMlpH2;
      for (int s = 0; s < kGradSamples; ++s) g = fmaf(DY[s * kMlpOut + k], H2[s * kMlpH2 + j], g);
    } else {  // b3[k]
      const int k = w - (kMlpB3 - kMlpW1);
      for (int s = 0; s < kGradSamples; ++s) g += DY[s * kMlpOut + k];
    }
    atomicAdd(&grad[kMlpW1 + w], g);
  }
  if (loss && threadIdx.x < kGradSamples) {
    lsum = warp_sum_f32(lsum);
    if ((threadIdx.x & 31) == 0 && lsum != 0.f) atomicAdd(loss, lsum);
  }
}

// Adam (Kingma & Ba 2015) on the weights (not the normalisation block).
__global__ void k_mlp_adam(float *__restrict__ params, const float *__restrict__ grad,
                           float *__restrict__ m, float *__restrict__ v, float lr, float b1, float b2,
                           float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpWeights; i += gridDim.x * blockDim.x) {
    const int w = kMlpW1 + i;
    const float g = grad[w];
    const float mi = b1 * m[w] + (1.f - b1) * g;
    const float vi = b2 * v[w] + (1.f - b2) * g * g;
    m[w] = mi;
    v[w] = vi;
    params[w] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

}  // namespace
}  // namespace gary

using namespace gary;

extern "C" int gary_mlp_param_count(void) { return kMlpParams; }

extern "C" int gary_mlp_init(uint64_t seed, float *params) {
  GARY_CHECK_ARG(params != nullptr, "params is NULL");
  std::mt19937_64 rng(seed);
  auto uni = [&](float bound) {
    return (float)((double)(rng() >> 11) / 9007199254740992.0 * 2.0 - 1.0) * bound;
  };
  for (int f = 0; f < kMlpIn; ++f) {
    params[kMlpMuX + f] = 0.f;
    params[kMlpSdX + f] = 1.f;
  }
  for (int k = 0; k < kMlpOut; ++k) {
    params[kMlpMuY + k] = 0.f;
    params[kMlpSdY + k] = 1.f;
  }
  // He-uniform for the ReLU layers, Glorot-uniform for the output layer
  const float g1 = std::sqrt(6.f / kMlpIn), g2 = std::sqrt(6.f / kMlpH1),
              g3 = std::sqrt(6.f / (kMlpH2 + kMlpOut));
  for (int i = 0; i < kMlpH1 * kMlpIn; ++i) params[kMlpW1 + i] = uni(g1);
  for (int i = 0; i < kMlpH1; ++i) params[kMlpB1 + i] = 0.f;
  for (int i = 0; i < kMlpH2 * kMlpH1; ++i) params[kMlpW2 + i] = uni(g2);
  for (int i = 0; i < kMlpH2; ++i) params[kMlpB2 + i] = 0.f;
  for (int i = 0; i < kMlpOut * kMlpH2; ++i) params[kMlpW3 + i] = uni(g3);
  for (int i = 0; i < kMlpOut; ++i) params[kMlpB3 + i] = 0.f;
  return GARY_OK;
}

extern "C" int gary_mlp_forward(const float *d_params, const float *d_x, uint64_t n, int scale,
                                float *d_y, void *stream) {
  GARY_CHECK_ARG(n == 0 || (d_params && d_x && d_y), "NULL argument");
  if (!n) return GARY_OK;
  const uint64_t blocks = (n + 127) / 128, cap = (uint64_t)sm_count() * 8;
  k_mlp_forward<<<(unsigned)(blocks < cap ? blocks : cap), 128, 0, as_stream(stream)>>>(
      d_params, d_x, n, scale, d_y);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

extern "C" int gary_mlp_grad(const float *d_params, const float *d_x, const float *d_t,
                             const uint8_t *d_mask, uint64_t n, float norm, float *d_grad,
                             float *d_loss, void *stream) {
  GARY_CHECK_ARG(d_params && d_grad, "NULL argument");
  GARY_CHECK_ARG(n == 0 || (d_x && d_t && d_mask), "NULL argument");
  GARY_CHECK_ARG(norm > 0.f, "norm must be positive");
  cudaStream_t s = as_stream(stream);
  GARY_CUDA(cudaMemsetAsync(d_grad, 0, kMlpParams * sizeof(float), s));
  if (d_loss) GARY_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
  if (!n) return GARY_OK;
  const size_t smem = (size_t)(kMlpParams + kGradSamples * (kMlpIn + 2 * kMlpH1 + 2 * kMlpH2 + kMlpOut)) * 4;
  static bool attr[64] = {false};
  const int dev = device_ordinal();
  if (dev < 64 && !attr[dev]) {
    GARY_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr[dev] = true;
  }
  const unsigned blocks = (unsigned)((n + kGradSamples - 1) / kGradSamples);
  k_mlp_grad<<<blocks, kGradThreads, smem, s>>>(d_params, d_x, d_t, d_mask, n, norm, d_grad, d_loss);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

extern "C" int gary_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v,
                             uint32_t step, float lr, void *stream) {
  GARY_CHECK_ARG(d_params && d_grad && d_m && d_v, "NULL argument");
  GARY_CHECK_ARG(step >= 1, "step counts from 1");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - (float)std::pow((double)b1, (double)step);
  const float c2 = 1.f - (float)std::pow((double)b2, (double)step);
  k_mlp_adam<<<(kMlpWeights + 255) / 256, 256, 0, as_stream(stream)>>>(d_params, d_grad, d_m, d_v,
                                                                       lr, b1, b2, eps, c1, c2);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

// File format (little-endian): "GARYMLP1", uint32 {1, 6, 64, 64, 4},
// then kMlpParams float32 (normalisation block first, as in memory).
extern "C" int gary_mlp_save(const char *path, const float *params) {
  GARY_CHECK_ARG(path && params, "NULL argument");
  FILE *f = std::fopen(path, "wb");
  if (!f) {
    set_error("cannot open %s for writing", path);
    return GARY_ERR_INVALID;
  }
  const uint32_t hdr[5] = {1, kMlpIn, kMlpH1, kMlpH2, kMlpOut};
  bool ok = std::fwrite("GARYMLP1", 1, 8, f) == 8 && std::fwrite(hdr, 4, 5, f) == 5 &&
            std::fwrite(params, 4, kMlpParams, f) == (size_t)kMlpParams;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    set_error("short write to %s", path);
    return GARY_ERR_INVALID;
  }
  return GARY_OK;
}

extern "C" int gary_mlp_load(const char *path, float *params) {
  GARY_CHECK_ARG(path && params, "NULL argument");
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    set_error("cannot open %s", path);
    return GARY_ERR_INVALID;
  }
  char magic[8];
  uint32_t hdr[5];
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "GARYMLP1", 8) == 0 &&
            std::fread(hdr, 4, 5, f) == 5 && hdr[0] == 1 && hdr[1] == kMlpIn && hdr[2] == kMlpH1 &&
            hdr[3] == kMlpH2 && hdr[4] == kMlpOut &&
            std::fread(params, 4, kMlpParams, f) == (size_t)kMlpParams;
  std::fclose(f);
  if (!ok) {
    set_error("%s is not a 6-64-64-4 GARYMLP1 cost model", path);
    return GARY_ERR_INVALID;
  }
  return GARY_OK;
}
