// The learned planner's network: 280 -> 128 -> 128 -> 5, ReLU hidden
// layers, bf16 weights, fp32 biases, activations and accumulation.
//
// Outputs: out[0] = predicted log2(1 + distinct keys) / 32, out[1..4] =
// logits of the four grouping strategies (dense index, shared-memory hash,
// global hash, sort).  Training uses fp32 master parameters, Adam, and a
// bf16 copy of the weight matrices that the forward and backward passes
// read.  Batch-1 inference at planning time is the block forward of
// mlp_core.cuh (which also holds the parameter layout), run by the key
// sketch's last CTA.
//
// The matrices are small (at most 280 x 128), so the layers are plain
// tiled CUDA-core GEMMs with fp32 accumulation: a training step at batch
// 4096 is about 2e8 multiply-adds per pass.
#include <cuda_bf16.h>

#include <algorithm>

#include "groupby_host.h"
#include "mlp_core.cuh"

namespace nfc {
namespace {

constexpr int kIn = kMlpIn, kH = kMlpH, kOut = kMlpOut;
constexpr int64_t kOffW1 = kMlpOffW1, kOffB1 = kMlpOffB1, kOffW2 = kMlpOffW2, kOffB2 = kMlpOffB2, kOffW3 = kMlpOffW3,
                  kOffB3 = kMlpOffB3, kNParams = kMlpNParams;
constexpr int64_t kWOffW1 = kMlpWOffW1, kWOffW2 = kMlpWOffW2, kWOffW3 = kMlpWOffW3, kNWeights = kMlpNWeights;

constexpr int kRows = 16;  // batch rows per CTA in the row-tiled kernels

NFC_DEV float bf(const __nv_bfloat16* w, int64_t i) { return __bfloat162float(w[i]); }

// Y[b][j] = act(b[j] + sum_i Xn[b][i] W[i][j]) for kRows rows per CTA;
// Xn = (X - mu) / sd when mu is given (layer 1), else X.
__global__ void __launch_bounds__(256) k_layer_fwd(const float* __restrict__ X, int64_t B, int I, int O,
                                                   const float* __restrict__ mu, const float* __restrict__ sd,
                                                   const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias,
                                                   bool relu, float* __restrict__ Y) {
  __shared__ float xs[kRows][kIn];
  const int64_t r0 = (int64_t)blockIdx.x * kRows;
  for (int t = threadIdx.x; t < kRows * I; t += blockDim.x) {
    const int r = t / I, i = t % I;
    float x = r0 + r < B ? X[(r0 + r) * I + i] : 0.f;
    if (mu) x = (x - mu[i]) / sd[i];
    xs[r][i] = x;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kRows * O; t += blockDim.x) {
    const int r = t / O, j = t % O;
    if (r0 + r >= B) continue;
    float acc = bias[j];
    for (int i = 0; i < I; ++i) acc = fmaf(xs[r][i], bf(W, (int64_t)i * O + j), acc);
    Y[(r0 + r) * O + j] = relu ? fmaxf(acc, 0.f) : acc;
  }
}

// dX[b][i] = (sum_j dY[b][j] W[i][j]) * (Xact[b][i] > 0)   (hidden layers)
__global__ void __launch_bounds__(256) k_layer_bwd_dx(const float* __restrict__ dY, int64_t B, int I, int O,
                                                      const __nv_bfloat16* __restrict__ W,
                                                      const float* __restrict__ Xact, float* __restrict__ dX) {
  __shared__ float ds[kRows][kH];
  const int64_t r0 = (int64_t)blockIdx.x * kRows;
  for (int t = threadIdx.x; t < kRows * O; t += blockDim.x) {
    const int r = t / O, j = t % O;
    ds[r][j] = r0 + r < B ? dY[(r0 + r) * O + j] : 0.f;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kRows * I; t += blockDim.x) {
    const int r = t / I, i = t % I;
    if (r0 + r >= B) continue;
    float acc = 0.f;
    for (int j = 0; j < O; ++j) acc = fmaf(ds[r][j], bf(W, (int64_t)i * O + j), acc);
    dX[(r0 + r) * I + i] = Xact[(r0 + r) * I + i] > 0.f ? acc : 0.f;
  }
}

// dW[i][j] = sum_b Xn[b][i] dY[b][j]; db[j] = sum_b dY[b][j].  One thread per
// (i, j) over the whole batch, staged 64 rows at a time in shared memory.
__global__ void __launch_bounds__(256) k_layer_bwd_dw(const float* __restrict__ X, const float* __restrict__ dY,
                                                      int64_t B, int I, int O, const float* __restrict__ mu,
                                                      const float* __restrict__ sd, float* __restrict__ dW,
                                                      float* __restrict__ db) {
  constexpr int kB = 64;
  __shared__ float xs[kB][32];
  __shared__ float gs[kB][32];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const int ti = threadIdx.x / 32, tj = threadIdx.x % 32;  // 8 x 32 threads, 4 i per thread
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  float bacc = 0.f;
  for (int64_t b0 = 0; b0 < B; b0 += kB) {
    for (int t = threadIdx.x; t < kB * 32; t += blockDim.x) {
      const int r = t / 32, c = t % 32;
      const int64_t b = b0 + r;
      float x = 0.f, g = 0.f;
      if (b < B && i0 + c < I) {
        x = X[b * I + i0 + c];
        if (mu) x = (x - mu[i0 + c]) / sd[i0 + c];
      }
      if (b < B && j0 + c < O) g = dY[b * O + j0 + c];
      xs[r][c] = x;
      gs[r][c] = g;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < kB; ++r) {
      const float g = gs[r][tj];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fmaf(xs[r][ti * 4 + q], g, acc[q]);
      if (blockIdx.x == 0 && ti == 0) bacc += g;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = i0 + ti * 4 + q, j = j0 + tj;
    if (i < I && j < O) dW[(int64_t)i * O + j] = acc[q];
  }
  if (blockIdx.x == 0 && ti == 0 && j0 + tj < O) db[j0 + tj] = bacc;
}

// Loss per row: card_w * (out0 - y)^2 + cls_w * w_b * cross-entropy(out[1..4],
// label) (label < 0: no class term; w_b = sample_weight[b], or 1 when absent).
// Writes dOut and adds the batch-mean loss.
__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ y, const int32_t* __restrict__ label,
                       const float* __restrict__ sw, int64_t B, float card_w, float cls_w_all,
                       float* __restrict__ dout, float* loss_sum) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
    const float* o = out + b * kOut;
    float* d = dout + b * kOut;
    const float e = o[0] - y[b];
    float loss = card_w * e * e;
    d[0] = 2.f * card_w * e / (float)B;
    const int lb = label[b];
    const float cls_w = sw ? cls_w_all * sw[b] : cls_w_all;
    float mx = o[1];
    for (int k = 2; k < kOut; ++k) mx = fmaxf(mx, o[k]);
    float se = 0.f;
    for (int k = 1; k < kOut; ++k) se += expf(o[k] - mx);
    for (int k = 1; k < kOut; ++k) {
      const float p = expf(o[k] - mx) / se;
      d[k] = lb >= 0 ? cls_w * (p - (k - 1 == lb ? 1.f : 0.f)) / (float)B : 0.f;
    }
    if (lb >= 0) loss += cls_w * (logf(se) + mx - o[1 + lb]);
    atomicAdd(loss_sum, loss / (float)B);
  }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float wd, float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
  }
}

// bf16 working copy of the three weight matrices.
__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < kNWeights; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t src;
    if (i < kWOffW2) src = kOffW1 + i;
    else if (i < kWOffW3) src = kOffW2 + (i - kWOffW2);
    else src = kOffW3 + (i - kWOffW3);
    w[i] = __float2bfloat16_rn(p[src]);
  }
}

unsigned rows_grid(int64_t B) { return (unsigned)std::max<int64_t>(1, (B + kRows - 1) / kRows); }

}  // namespace
}  // namespace nfc

using namespace nfc;


extern "C" int32_t nfc_mlp_to_bf16(const float* params, uint16_t* weights_bf16, void* stream) {
  if (!params || !weights_bf16) return NFC_ERR_NULL;
  k_to_bf16<<<64, 256, 0, static_cast<cudaStream_t>(stream)>>>(params,
                                                                reinterpret_cast<__nv_bfloat16*>(weights_bf16));
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_mlp_forward(const float* x, int64_t batch, const float* feat_mu, const float* feat_sd,
                                   const uint16_t* weights_bf16, const float* params, float* h1, float* h2,
                                   float* out, void* stream) {
  if (batch < 0) return NFC_ERR_MALFORMED;
  if (batch == 0) return NFC_OK;
  if (!x || !weights_bf16 || !params || !h1 || !h2 || !out) return NFC_ERR_NULL;
  if ((feat_mu == nullptr) != (feat_sd == nullptr)) return NFC_ERR_MALFORMED;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const __nv_bfloat16* w = reinterpret_cast<const __nv_bfloat16*>(weights_bf16);
  k_layer_fwd<<<rows_grid(batch), 256, 0, s>>>(x, batch, kIn, kH, feat_mu, feat_sd, w + kWOffW1, params + kOffB1,
                                              true, h1);
  k_layer_fwd<<<rows_grid(batch), 256, 0, s>>>(h1, batch, kH, kH, nullptr, nullptr, w + kWOffW2, params + kOffB2, true,
                                              h2);
  k_layer_fwd<<<rows_grid(batch), 256, 0, s>>>(h2, batch, kH, kOut, nullptr, nullptr, w + kWOffW3, params + kOffB3,
                                              false, out);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_mlp_backward(const float* x, int64_t batch, const float* feat_mu, const float* feat_sd,
                                    const uint16_t* weights_bf16, const float* h1, const float* h2,
                                    const float* dout, float* dh1, float* dh2, float* grad, void* stream) {
  if (batch <= 0) return NFC_ERR_MALFORMED;
  if (!x || !weights_bf16 || !h1 || !h2 || !dout || !dh1 || !dh2 || !grad) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const __nv_bfloat16* w = reinterpret_cast<const __nv_bfloat16*>(weights_bf16);
  // Layer 3.
  k_layer_bwd_dw<<<dim3((kH + 31) / 32, (kOut + 31) / 32), 256, 0, s>>>(h2, dout, batch, kH, kOut, nullptr, nullptr,
                                                                        grad + kOffW3, grad + kOffB3);
  k_layer_bwd_dx<<<rows_grid(batch), 256, 0, s>>>(dout, batch, kH, kOut, w + kWOffW3, h2, dh2);
  // Layer 2.
  k_layer_bwd_dw<<<dim3((kH + 31) / 32, (kH + 31) / 32), 256, 0, s>>>(h1, dh2, batch, kH, kH, nullptr, nullptr,
                                                                      grad + kOffW2, grad + kOffB2);
  k_layer_bwd_dx<<<rows_grid(batch), 256, 0, s>>>(dh2, batch, kH, kH, w + kWOffW2, h1, dh1);
  // Layer 1.
  k_layer_bwd_dw<<<dim3((kIn + 31) / 32, (kH + 31) / 32), 256, 0, s>>>(x, dh1, batch, kIn, kH, feat_mu, feat_sd,
                                                                       grad + kOffW1, grad + kOffB1);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_mlp_loss(const float* out, const float* y_card, const int32_t* label,
                                const float* sample_weight, int64_t batch, float card_weight, float class_weight,
                                float* dout, float* loss_sum, void* stream) {
  if (batch <= 0) return NFC_ERR_MALFORMED;
  if (!out || !y_card || !label || !dout || !loss_sum) return NFC_ERR_NULL;
  const unsigned g = (unsigned)std::min<int64_t>((batch + 255) / 256, 1024);
  k_loss<<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(out, y_card, label, sample_weight, batch, card_weight,
                                                           class_weight, dout, loss_sum);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_mlp_adam(float* params, const float* grad, float* m, float* v, uint16_t* weights_bf16,
                                int64_t step, float lr, float beta1, float beta2, float eps, float weight_decay,
                                void* stream) {
  if (!params || !grad || !m || !v || !weights_bf16) return NFC_ERR_NULL;
  if (step < 1) return NFC_ERR_MALFORMED;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_adam<<<(unsigned)((kNParams + 255) / 256), 256, 0, s>>>(params, grad, m, v, kNParams, lr, beta1, beta2, eps,
                                                            weight_decay, c1, c2);
  k_to_bf16<<<64, 256, 0, s>>>(params, reinterpret_cast<__nv_bfloat16*>(weights_bf16));
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}
