// Counter-based Philox4x32-10 input generation on the device.
//
// Lane layout and key derivation follow the reference RNG so that a fill
// here is bit-identical to rng_fill_i32 / rng_fill_f64
// (src/Drivers/CPU/_lib/rng.py:44-141, numfast-native/src/rng.rs):
//   key      = SplitMix64(seed + golden + stream * C1) split into two u32
//   counter  = (lo32(offset+i), hi32(offset+i), lo32(stream)^0xC0FFEE00,
//               hi32(stream)^0x9E3779B9)
//   10 rounds of the published Philox4x32 round function (Salmon et al.,
//   SC'11) with the standard multipliers and Weyl key increments.
// Each thread produces a contiguous run of lanes so stores are coalesced.
#include <math.h>

#include "nfc_common.cuh"

namespace nfc {

struct PhiloxKey {
  uint32_t k0, k1;
};

NFC_HD uint64_t splitmix64_out(uint64_t state) {
  uint64_t z = state + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static PhiloxKey derive_key(uint64_t seed, uint64_t stream) {
  uint64_t st = seed + 0x9E3779B97F4A7C15ull + stream * 0xBF58476D1CE4E5B9ull;
  uint64_t k = splitmix64_out(st);
  return {static_cast<uint32_t>(k), static_cast<uint32_t>(k >> 32)};
}

struct Philox4 {
  uint32_t r0, r1, r2, r3;
};

NFC_DEV Philox4 philox10(uint64_t ctr, uint32_t c2, uint32_t c3, PhiloxKey key) {
  uint32_t a0 = static_cast<uint32_t>(ctr), a1 = static_cast<uint32_t>(ctr >> 32);
  uint32_t a2 = c2, a3 = c3;
  uint32_t k0 = key.k0, k1 = key.k1;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = a0 * 0xD2511F53u, hi0 = __umulhi(a0, 0xD2511F53u);
    const uint32_t lo1 = a2 * 0xCD9E8D57u, hi1 = __umulhi(a2, 0xCD9E8D57u);
    const uint32_t n0 = hi1 ^ a1 ^ k0, n2 = hi0 ^ a3 ^ k1;
    a0 = n0;
    a1 = lo1;
    a2 = n2;
    a3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return {a0, a1, a2, a3};
}

struct LaneCfg {
  uint64_t offset;
  uint32_t c2, c3;
  PhiloxKey key;
};

static LaneCfg lane_cfg(uint64_t seed, uint64_t stream, uint64_t offset) {
  LaneCfg c;
  c.offset = offset;
  c.c2 = static_cast<uint32_t>(stream) ^ 0xC0FFEE00u;
  c.c3 = static_cast<uint32_t>(stream >> 32) ^ 0x9E3779B9u;
  c.key = derive_key(seed, stream);
  return c;
}

NFC_DEV double u53(const Philox4& r) {
  const uint64_t u = (static_cast<uint64_t>(r.r0 >> 5) << 26) | static_cast<uint64_t>(r.r1 >> 6);
  return static_cast<double>(u) * (1.0 / 9007199254740992.0);
}

__global__ void k_fill_i32(int64_t n, LaneCfg c, uint64_t width, int64_t lo, int32_t* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const Philox4 r = philox10(c.offset + (uint64_t)i, c.c2, c.c3, c.key);
    const uint64_t v = (static_cast<uint64_t>(r.r0) * width) >> 32;
    out[i] = static_cast<int32_t>(static_cast<int64_t>(v) + lo);
  }
}

__global__ void k_fill_f64(int64_t n, LaneCfg c, double lo, double span, double* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const Philox4 r = philox10(c.offset + (uint64_t)i, c.c2, c.c3, c.key);
    // Separately rounded multiply and add (no FMA contraction), as the
    // reference evaluates lo + f * (hi - lo).
    out[i] = __dadd_rn(lo, __dmul_rn(u53(r), span));
  }
}

__global__ void k_lognormal(int64_t n, LaneCfg a, LaneCfg b, double mu, double sigma, double* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double u1 = 1.0 - u53(philox10(a.offset + (uint64_t)i, a.c2, a.c3, a.key));  // (0, 1]
    const double u2 = u53(philox10(b.offset + (uint64_t)i, b.c2, b.c3, b.key));
    const double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    out[i] = exp(mu + sigma * z);
  }
}

__global__ void k_zipf(int64_t n, LaneCfg c, double one_minus_s, double dom_pow, int64_t domain,
                       int32_t* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double u = u53(philox10(c.offset + (uint64_t)i, c.c2, c.c3, c.key));
    // Continuous power law on [1, domain+1): x = (1 + u*(D^(1-s) - 1))^(1/(1-s)).
    double x = pow(1.0 + u * (dom_pow - 1.0), 1.0 / one_minus_s);
    int64_t rank = static_cast<int64_t>(floor(x));
    rank = rank < 1 ? 1 : (rank > domain ? domain : rank);
    out[i] = static_cast<int32_t>(rank - 1);
  }
}

// One thread writes one bitmap byte (8 lanes).
__global__ void k_validity(int64_t n, LaneCfg c, double p_null, uint8_t* bm) {
  const int64_t nbytes = (n + 7) >> 3;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nbytes;
       j += (int64_t)gridDim.x * blockDim.x) {
    uint32_t byte = 0;
    for (int b = 0; b < 8; ++b) {
      const int64_t i = j * 8 + b;
      if (i < n) {
        const double u = u53(philox10(c.offset + (uint64_t)i, c.c2, c.c3, c.key));
        byte |= (u >= p_null ? 1u : 0u) << b;
      }
    }
    bm[j] = static_cast<uint8_t>(byte);
  }
}

static int grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  const int64_t cap = (int64_t)num_sms() * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return static_cast<int>(g);
}

}  // namespace nfc

using namespace nfc;

extern "C" int32_t nfc_rng_fill_i32(int64_t n, uint64_t seed, uint64_t stream_id, uint64_t offset,
                                    int64_t lo, int64_t hi, int32_t* out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (!(hi > lo)) return NFC_ERR_RANGE;
  if (n == 0) return NFC_OK;
  if (!out) return NFC_ERR_NULL;
  const uint64_t width = static_cast<uint64_t>(hi - lo);
  if (width > (1ull << 32)) return NFC_ERR_RANGE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_fill_i32<<<grid_for(n), 256, 0, s>>>(n, lane_cfg(seed, stream_id, offset), width, lo, out);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_rng_fill_f64(int64_t n, uint64_t seed, uint64_t stream_id, uint64_t offset,
                                    double lo, double hi, double* out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (!(isfinite(lo) && isfinite(hi) && lo < hi)) return NFC_ERR_RANGE;
  if (n == 0) return NFC_OK;
  if (!out) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_fill_f64<<<grid_for(n), 256, 0, s>>>(n, lane_cfg(seed, stream_id, offset), lo, hi - lo, out);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_gen_lognormal(int64_t n, uint64_t seed, uint64_t stream_a, uint64_t stream_b,
                                     double mu, double sigma, double* out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (n == 0) return NFC_OK;
  if (!out) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_lognormal<<<grid_for(n), 256, 0, s>>>(n, lane_cfg(seed, stream_a, 0), lane_cfg(seed, stream_b, 0),
                                          mu, sigma, out);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_gen_zipf(int64_t n, uint64_t seed, uint64_t stream_id, double s_exp,
                                int64_t domain, int32_t* out, void* stream) {
  if (n < 0 || domain < 1 || domain > INT32_MAX || !(s_exp > 0.0) || s_exp == 1.0)
    return NFC_ERR_MALFORMED;
  if (n == 0) return NFC_OK;
  if (!out) return NFC_ERR_NULL;
  const double oms = 1.0 - s_exp;
  const double dom_pow = pow(static_cast<double>(domain) + 1.0, oms);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_zipf<<<grid_for(n), 256, 0, s>>>(n, lane_cfg(seed, stream_id, 0), oms, dom_pow, domain, out);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int32_t nfc_gen_validity(int64_t n, uint64_t seed, uint64_t stream_id, double p_null,
                                    uint8_t* bitmap_out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (n == 0) return NFC_OK;
  if (!bitmap_out) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_validity<<<grid_for((n + 7) / 8), 256, 0, s>>>(n, lane_cfg(seed, stream_id, 0), p_null, bitmap_out);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}
