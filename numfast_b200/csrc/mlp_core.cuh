// The planner network's parameter layout and a batch-1 forward pass that one
// block of 256 threads runs from shared memory (used by the sketch's last
// CTA, so planning costs no separate inference launch).
//
// Packed float32 parameter layout (NFC_MLP_NPARAMS floats):
//   W1[280][128] b1[128] W2[128][128] b2[128] W3[128][5] b3[5]
// bf16 weights (NFC_MLP_NWEIGHTS): W1, W2, W3 in the same order.
// Matrices are [in][out]: y[j] = b[j] + sum_i x[i] * W[i][j].
#pragma once

#include <cuda_bf16.h>

#include "nfc_common.cuh"

namespace nfc {

constexpr int kMlpIn = NFC_MLP_IN, kMlpH = NFC_MLP_H, kMlpOut = NFC_MLP_OUT;
constexpr int64_t kMlpOffW1 = 0, kMlpOffB1 = kMlpOffW1 + kMlpIn * kMlpH, kMlpOffW2 = kMlpOffB1 + kMlpH,
                  kMlpOffB2 = kMlpOffW2 + kMlpH * kMlpH, kMlpOffW3 = kMlpOffB2 + kMlpH,
                  kMlpOffB3 = kMlpOffW3 + kMlpH * kMlpOut, kMlpNParams = kMlpOffB3 + kMlpOut;
constexpr int64_t kMlpWOffW1 = 0, kMlpWOffW2 = kMlpIn * kMlpH, kMlpWOffW3 = kMlpWOffW2 + kMlpH * kMlpH,
                  kMlpNWeights = kMlpWOffW3 + kMlpH * kMlpOut;
static_assert(kMlpNParams == NFC_MLP_NPARAMS, "parameter layout");
static_assert(kMlpNWeights == NFC_MLP_NWEIGHTS, "weight layout");
static_assert(kMlpWOffW2 % 4 == 0 && kMlpWOffW3 % 4 == 0, "8-byte aligned weight rows");

// Network weights for inference at planning time.
struct MlpRef {
  const float* mu;               // feature standardisation (null: none)
  const float* sd;
  const __nv_bfloat16* w;        // bf16 weight matrices
  const float* p;                // fp32 parameters (biases read here)
  float* out;                    // NFC_MLP_OUT outputs (may be mapped host memory)
};

struct alignas(16) MlpSmem {  // part is written as float4
  float x[kMlpIn];
  float h[kMlpH];
  float part[8][kMlpH];
};

// Partial dot products of one hidden layer: thread (quad q, slice sl) sums
// inputs [sl * I/8, (sl + 1) * I/8) for outputs 4q..4q+3, reading each
// weight row's four bf16 as one 8-byte load (independent loads, unrolled).
template <int I>
NFC_DEV void mlp_layer_part(const float* xin, const __nv_bfloat16* __restrict__ W, int q, int sl,
                            float (*part)[kMlpH]) {
  static_assert(I % 8 == 0 && kMlpH == 128, "slicing");
  constexpr int per = I / 8;
  const uint2* wp = reinterpret_cast<const uint2*>(W) + q;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
  for (int ii = 0; ii < per; ++ii) {
    const int i = sl * per + ii;
    const uint2 u = __ldg(wp + (int64_t)i * (kMlpH / 4));
    const float xi = xin[i];
    const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
    const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
    a0 = fmaf(xi, lo.x, a0);
    a1 = fmaf(xi, lo.y, a1);
    a2 = fmaf(xi, hi.x, a2);
    a3 = fmaf(xi, hi.y, a3);
  }
  *reinterpret_cast<float4*>(&part[sl][4 * q]) = make_float4(a0, a1, a2, a3);
}

// Forward pass of features x (global memory, written by this block before
// the call) by a block of exactly 256 threads; every thread calls it.  The
// bf16 weights must be 8-byte aligned (the layout's offsets keep them so).
NFC_DEV void mlp_forward_block256(const float* x, const MlpRef& m, MlpSmem& sm) {
  const int t = threadIdx.x, q = t & 31, sl = t >> 5;  // 32 output quads x 8 input slices
  for (int i = t; i < kMlpIn; i += 256) sm.x[i] = m.mu ? (x[i] - m.mu[i]) / m.sd[i] : x[i];
  __syncthreads();
  mlp_layer_part<kMlpIn>(sm.x, m.w + kMlpWOffW1, q, sl, sm.part);
  __syncthreads();
  if (t < kMlpH) {
    float a = m.p[kMlpOffB1 + t];
#pragma unroll
    for (int k = 0; k < 8; ++k) a += sm.part[k][t];
    sm.h[t] = fmaxf(a, 0.f);
  }
  __syncthreads();
  mlp_layer_part<kMlpH>(sm.h, m.w + kMlpWOffW2, q, sl, sm.part);
  __syncthreads();
  if (t < kMlpH) {
    float a = m.p[kMlpOffB2 + t];
#pragma unroll
    for (int k = 0; k < 8; ++k) a += sm.part[k][t];
    sm.h[t] = fmaxf(a, 0.f);  // layer 2 read sm.h before the barrier above
  }
  __syncthreads();
  // Layer 3: warp o < 5 reduces 128 products for output o.
  const int warp = t >> 5, lane = t & 31;
  if (warp < kMlpOut) {
    float acc = 0.f;
#pragma unroll
    for (int i = lane; i < kMlpH; i += 32)
      acc = fmaf(sm.h[i], __bfloat162float(m.w[kMlpWOffW3 + (int64_t)i * kMlpOut + warp]), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) m.out[warp] = acc + m.p[kMlpOffB3 + warp];
  }
}

}  // namespace nfc
