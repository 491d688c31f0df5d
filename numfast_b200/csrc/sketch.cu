// Key sketch for the learned planner: 280 features from the first 65,536
// rows of a key column, in two passes of 64 CTAs (range, first valid key and
// HyperLogLog registers; then the pairwise counters, whose last CTA writes
// the features).
//
//   features[0..255]   HyperLogLog registers (p = 8): for each valid key,
//                      h = mix64(key); register h >> 56 keeps the maximum of
//                      (leading zeros of h << 8) + 1, capped at 57; stored
//                      as rank / 16
//   features[256..279] run / range statistics (st[0..23] at the end of
//                      k_sketch_pass2)
//
// The reference has no sketch: its planner sees only n, sortedness and the
// key span (src/Runtime/Planner/_lib/planner.py:200-262).  These features
// add what that rule cannot see -- the distinct count, runs, clustering and
// skew -- at the cost of one read of 256 KB.
#include <math.h>

#include <algorithm>

#include "groupby_host.h"
#include "mlp_core.cuh"

namespace nfc {
namespace {

constexpr int kSketchRows = 65536;
constexpr int kHllRegs = 256;

NFC_DEV uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

NFC_DEV bool key_valid(const uint8_t* bm, int64_t i) { return !bm || ((bm[i >> 3] >> (i & 7)) & 1u); }

NFC_DEV float slog2(double x) { return (float)(x >= 0 ? log2(1.0 + x) : -log2(1.0 - x)); }

// Global scratch of one sketch (zeroed before pass 1; every field's zero is
// its identity): max ordered key, max of ~ordered key (= min), max of
// ~first valid row, HLL registers, pass-2 counters, pass-2 CTA ticket.
struct SketchScratch {
  uint32_t kmax_o, kmin_c, first_c, done;
  uint32_t reg[kHllRegs];
  unsigned long long c[16];
};

constexpr int kSkCtaRows = 1024;  // rows per CTA in both passes (256 threads x 4); kSketchRows / kSkCtaRows CTAs

__global__ void __launch_bounds__(256) k_sketch_pass1(const int32_t* __restrict__ keys, const uint8_t* __restrict__ bm,
                                                     int64_t m, SketchScratch* sk) {
  __shared__ uint32_t reg[kHllRegs];
  __shared__ uint32_t s_min, s_max, s_first;
  reg[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    s_min = 0xFFFFFFFFu;
    s_max = 0u;
    s_first = 0xFFFFFFFFu;
  }
  __syncthreads();
  uint32_t mn = 0xFFFFFFFFu, mx = 0u, fi = 0xFFFFFFFFu;
  const int64_t base = (int64_t)blockIdx.x * kSkCtaRows;
#pragma unroll
  for (int j = 0; j < kSkCtaRows / 256; ++j) {
    const int64_t i = base + j * 256 + threadIdx.x;
    if (i >= m || !key_valid(bm, i)) continue;
    const int32_t k = keys[i];
    const uint32_t o = (uint32_t)k ^ 0x80000000u;
    mn = min(mn, o);
    mx = max(mx, o);
    fi = min(fi, (uint32_t)i);
    const uint64_t h = mix64((uint64_t)(uint32_t)k);
    const uint32_t r = min((uint32_t)__clzll((long long)((h << 8) | 0x80ull)) + 1u, 57u);
    atomicMax(&reg[h >> 56], r);
  }
  atomicMin(&s_min, mn);
  atomicMax(&s_max, mx);
  atomicMin(&s_first, fi);
  __syncthreads();
  if (reg[threadIdx.x]) atomicMax(&sk->reg[threadIdx.x], reg[threadIdx.x]);
  if (threadIdx.x == 0 && s_first != 0xFFFFFFFFu) {
    atomicMax(&sk->kmax_o, s_max);
    atomicMax(&sk->kmin_c, ~s_min);
    atomicMax(&sk->first_c, ~s_first);
  }
}

// Pass 2: pairwise and positional counters; the last CTA writes the features.
// With mlp.w set, the last CTA also runs the network on the features and
// leaves the scratch zeroed for the next sketch (no memset before it).
__global__ void __launch_bounds__(256) k_sketch_pass2(const int32_t* __restrict__ keys, const uint8_t* __restrict__ bm,
                                                     int64_t n, int64_t m, SketchScratch* sk, float* __restrict__ feat,
                                                     MlpRef mlp) {
  __shared__ unsigned long long sred[8 * 16];
  __shared__ unsigned long long tot[16];
  __shared__ bool s_last;
  const bool has = sk->first_c != 0u;
  const int64_t kmin = (int64_t)(int32_t)((~sk->kmin_c) ^ 0x80000000u);
  const int64_t kmax = (int64_t)(int32_t)(sk->kmax_o ^ 0x80000000u);
  const double span = has ? (double)(kmax - kmin) + 1.0 : 0.0;
  const int32_t first = has ? keys[~sk->first_c] : 0;
  unsigned long long c[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) c[j] = 0;
  const int64_t base = (int64_t)blockIdx.x * kSkCtaRows;
#pragma unroll
  for (int jj = 0; jj < kSkCtaRows / 256; ++jj) {
    const int64_t i = base + jj * 256 + threadIdx.x;
    if (i >= m || !key_valid(bm, i)) continue;
    const int32_t k = keys[i];
    c[0] += 1;                                                      // valid rows
    c[1] += (k == first);                                           // rows equal to the first key
    const double pos = span > 0 ? ((double)k - (double)kmin) / span : 0.0;
    c[2] += pos < 0.5;                                              // lower half of the range
    c[3] += pos < 0.0625;                                           // first sixteenth
    if (i + 1 < m && key_valid(bm, i + 1)) {
      const int32_t k1 = keys[i + 1];
      const int64_t d = (int64_t)k1 - (int64_t)k;
      const uint64_t ad = (uint64_t)(d < 0 ? -d : d);
      c[4] += 1;                                                    // adjacent valid pairs
      c[5] += (d == 0);
      c[6] += (d > 0);
      c[7] += (d < 0);
      c[8] += ad < 1024;
      c[9] += ad < 65536;
      c[10] += ((uint32_t)k >> 16) == ((uint32_t)k1 >> 16);
      c[11] += (ad < (1ull << 40) ? ad : (1ull << 40)) >> 8;         // sum |d| / 256 (bounded)
    }
    if (i + 8 < m && key_valid(bm, i + 8)) {
      c[12] += 1;
      c[13] += keys[i + 8] == k;
    }
    if (i > 0 && key_valid(bm, i - 1)) c[14] += keys[i - 1] != k;  // run heads after a valid row
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    unsigned long long x = c[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane_id() == 0) sred[(threadIdx.x >> 5) * 16 + j] = x;
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    unsigned long long t = 0;
    for (int w = 0; w < 8; ++w) t += sred[w * 16 + threadIdx.x];
    if (t) atomicAdd(&sk->c[threadIdx.x], t);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&sk->done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  __shared__ uint32_t sreg[kHllRegs];
  if (threadIdx.x < 16) tot[threadIdx.x] = atomicAdd(&sk->c[threadIdx.x], 0ull);
  const uint32_t rg = atomicAdd(&sk->reg[threadIdx.x], 0u);
  sreg[threadIdx.x] = rg;
  feat[threadIdx.x] = (float)rg / 16.f;
  __syncthreads();
  if (threadIdx.x == 0) {
    // HLL estimate (raw estimator with linear counting for small cardinality).
    double z = 0.0;
    int zeros = 0;
    for (int r = 0; r < kHllRegs; ++r) {
      const uint32_t v = sreg[r];
      z += ldexp(1.0, -(int)v);
      zeros += v == 0;
    }
    const double mm = (double)kHllRegs;
    double est = 0.7182725932 * mm * mm / z;  // alpha_256 = 0.7213 / (1 + 1.079 / 256)
    if (est <= 2.5 * mm && zeros > 0) est = mm * log(mm / (double)zeros);
    const double valid = (double)tot[0];
    const double pairs = tot[4] > 0 ? (double)tot[4] : 1.0;
    const double heads = (double)tot[14] + 1.0;
    float* st = feat + kHllRegs;
    st[0] = (float)(log2(1.0 + (double)n) / 32.0);
    st[1] = (float)(log2(1.0 + (double)m) / 17.0);
    st[2] = m > 0 ? (float)(valid / (double)m) : 0.f;
    st[3] = (float)(log2(1.0 + est) / 32.0);
    st[4] = (float)zeros / (float)kHllRegs;
    st[5] = (float)((double)tot[5] / pairs);
    st[6] = (float)(log2(1.0 + valid / heads) / 17.0);
    st[7] = tot[12] > 0 ? (float)((double)tot[13] / (double)tot[12]) : 0.f;
    st[8] = (float)((double)tot[6] / pairs);
    st[9] = (float)((double)tot[7] / pairs);
    st[10] = (float)(log2(1.0 + span) / 32.0);
    st[11] = kmin >= 0 ? 1.f : 0.f;
    st[12] = slog2((double)kmin) / 32.f;
    st[13] = slog2((double)kmax) / 32.f;
    st[14] = (float)((log2(1.0 + span) - log2(1.0 + valid)) / 32.0);
    st[15] = (float)(log2(1.0 + 256.0 * (double)tot[11] / pairs) / 40.0);
    st[16] = (float)((double)tot[8] / pairs);
    st[17] = (float)((double)tot[9] / pairs);
    st[18] = valid > 0 ? (float)((double)tot[2] / valid) : 0.f;
    st[19] = valid > 0 ? (float)((double)tot[3] / valid) : 0.f;
    st[20] = valid > 0 ? (float)((double)tot[1] / valid) : 0.f;
    st[21] = valid > 0 ? (float)fmin(est / valid, 4.0) : 0.f;
    st[22] = (float)(log2((1.0 + (double)n) / (1.0 + (double)m)) / 16.0);
    st[23] = (float)((double)tot[10] / pairs);
  }
  if (!mlp.w) return;
  // Every other CTA has read the pass-1 fields and added its counters (it
  // counted itself done after both): zero the scratch for the next sketch.
  __syncthreads();
  sk->reg[threadIdx.x] = 0u;
  if (threadIdx.x < 16) sk->c[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) {
    sk->kmax_o = 0u;
    sk->kmin_c = 0u;
    sk->first_c = 0u;
    sk->done = 0u;
  }
  __shared__ MlpSmem msm;
  mlp_forward_block256(feat, mlp, msm);
}

}  // namespace
}  // namespace nfc

using namespace nfc;

int nfc::sketch_launch(const int32_t* keys, const uint8_t* key_validity, int64_t n, float* features_out,
                       void* scratch, cudaStream_t s, const MlpRef* mlp) {
  SketchScratch* sk = static_cast<SketchScratch*>(scratch);
  // With the network attached the scratch is left zeroed by the previous
  // sketch (and by the planner at creation).
  if (!mlp) NFC_CUDA(cudaMemsetAsync(sk, 0, sizeof(SketchScratch), s));
  const int64_t m = n < kSketchRows ? n : kSketchRows;
  const unsigned g = (unsigned)std::max<int64_t>(1, (m + kSkCtaRows - 1) / kSkCtaRows);
  MlpRef none{};
  k_sketch_pass1<<<g, 256, 0, s>>>(keys, key_validity, m, sk);
  k_sketch_pass2<<<g, 256, 0, s>>>(keys, key_validity, n, m, sk, features_out, mlp ? *mlp : none);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

size_t nfc::sketch_scratch_bytes() { return sizeof(SketchScratch); }

extern "C" int32_t nfc_sketch(const int32_t* keys, const uint8_t* key_validity, int64_t n, float* features_out,
                              void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (!features_out || (n > 0 && !keys)) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  unsigned char* scratch = nullptr;
  NFC_CUDA(sc.alloc(&scratch, sketch_scratch_bytes()));
  return sketch_launch(keys, key_validity, n, features_out, scratch, s);
}
