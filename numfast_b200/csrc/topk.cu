// Top-k of the stable argsort without sorting every row: the first k entries
// of nfc_sort_perm's permutation (the reference's sort -> slice -> gather,
// src/Drivers/CPU/_lib/cpu.py:3170-3200, over the order of _sort_perm,
// cpu.py:1154-1225), by radix selection.
//
//   1. selection   each row's key as an order-preserving unsigned image
//                  (descending = its complement); 11-bit digit histograms
//                  from the top, over the rows whose higher digits match the
//                  prefix chosen so far, find the k-th smallest image: rows
//                  below the prefix are all taken, `need` of the rows on it
//                  (ties) are taken in input order.  A pass stops early once
//                  every row on the prefix is taken.
//   2. compaction  per block of 4,096 rows: counts of taken-below, tie and
//                  NULL rows; one CTA scans them; each block then writes its
//                  taken rows' (image, row) pairs in input order, and the
//                  first k - valid NULL rows straight into the output tail.
//   3. sort        the k taken pairs by image, stable (radix sort; one CTA
//                  for k <= 2,048), which is the argsort's order of them.
//
// Descending float64: every NaN is its own group in the reference's
// _stable_desc_idx, so the NaN block comes first in REVERSE input order: the
// selection takes the last `need` NaN rows and the sorted NaN prefix is
// reversed.  For k above n / 8 the full argsort is cheaper and is used.
#include <algorithm>

#include "groupby_core.cuh"
#include "groupby_host.h"

namespace nfc {
namespace {

constexpr int kTkThreads = 256;
constexpr int kTkItems = 16;
constexpr int kTkBlockRows = kTkThreads * kTkItems;  // 4096
constexpr int kTkDigitBits = 11;
constexpr int kTkBins = 1 << kTkDigitBits;

// Order-preserving unsigned image of row i's key; descending complements it
// (32 bits for int32, 64 for int64 / float64).  float64: -0.0 ties +0.0 and
// every NaN maps past +inf, as in the full argsort.
template <int DT>
NFC_DEV uint64_t tk_image(const void* keys, int64_t i, bool desc) {
  uint64_t u;
  if (DT == NFC_I32) {
    u = (uint32_t)static_cast<const int32_t*>(keys)[i] ^ 0x80000000u;
    return desc ? (~u & 0xFFFFFFFFull) : u;
  }
  if (DT == NFC_I64) {
    u = (uint64_t)static_cast<const int64_t*>(keys)[i] ^ 0x8000000000000000ull;
  } else {
    uint64_t b = static_cast<const uint64_t*>(keys)[i];
    if (f64_bits_isnan(b)) {
      u = ~0ull;
    } else {
      if (b == 0x8000000000000000ull) b = 0ull;
      u = f64_ord(b);
    }
  }
  return desc ? ~u : u;
}

NFC_DEV bool tk_valid(const uint8_t* v, int64_t i) { return !v || ((v[i >> 3] >> (i & 7)) & 1u); }

// Digit histogram of the valid rows on the prefix ((image & mask) == prefix).
// A thread adds repeats of its last digit locally, so a column of one value
// costs one shared atomic per thread, not one per row.
template <int DT>
__global__ void __launch_bounds__(kTkThreads) k_tk_hist(const void* __restrict__ keys,
                                                       const uint8_t* __restrict__ validity, int64_t n, bool desc,
                                                       uint64_t mask, uint64_t prefix, int shift, uint32_t dmask,
                                                       uint32_t* __restrict__ ghist) {
  __shared__ uint32_t h[kTkBins];
  for (int i = threadIdx.x; i < kTkBins; i += blockDim.x) h[i] = 0u;
  __syncthreads();
  uint32_t last = 0xFFFFFFFFu, run = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!tk_valid(validity, i)) continue;
    const uint64_t u = tk_image<DT>(keys, i, desc);
    if ((u & mask) != prefix) continue;
    const uint32_t d = (uint32_t)(u >> shift) & dmask;
    if (d == last) {
      ++run;
    } else {
      if (run) atomicAdd(&h[last], run);
      last = d;
      run = 1;
    }
  }
  if (run) atomicAdd(&h[last], run);
  __syncthreads();
  for (int i = threadIdx.x; i <= (int)dmask; i += blockDim.x)
    if (h[i]) atomicAdd(&ghist[i], h[i]);
}

// Row class: 0 taken (below the prefix), 1 tie (on the prefix), 2 NULL,
// 3 neither.
template <int DT>
NFC_DEV int tk_class(const void* keys, const uint8_t* validity, int64_t i, bool desc, uint64_t mask,
                     uint64_t prefix) {
  if (!tk_valid(validity, i)) return 2;
  const uint64_t m = tk_image<DT>(keys, i, desc) & mask;
  return m < prefix ? 0 : m == prefix ? 1 : 3;
}

// Per block of kTkBlockRows rows: counts of classes 0, 1, 2 -> cnt[3 b + c].
template <int DT>
__global__ void __launch_bounds__(kTkThreads) k_tk_count(const void* __restrict__ keys,
                                                        const uint8_t* __restrict__ validity, int64_t n, bool desc,
                                                        uint64_t mask, uint64_t prefix, uint32_t* __restrict__ cnt) {
  __shared__ uint32_t s[3][kTkThreads / 32];
  uint32_t c[3] = {0u, 0u, 0u};
  const int64_t base = (int64_t)blockIdx.x * kTkBlockRows;
#pragma unroll 4
  for (int j = 0; j < kTkItems; ++j) {
    const int64_t i = base + j * kTkThreads + threadIdx.x;
    if (i >= n) break;
    const int k = tk_class<DT>(keys, validity, i, desc, mask, prefix);
    if (k < 3) ++c[k];
  }
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint32_t w = warp_sum(c[k]);
    if (lane_id() == 0) s[k][warp] = w;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    uint32_t t = 0;
    for (int w = 0; w < kTkThreads / 32; ++w) t += s[threadIdx.x][w];
    cnt[3 * (int64_t)blockIdx.x + threadIdx.x] = t;
  }
}

// Exclusive scan of the three count columns over nb blocks (one CTA).
__global__ void __launch_bounds__(1024) k_tk_scan(const uint32_t* __restrict__ cnt, int64_t nb,
                                                 uint32_t* __restrict__ pre) {
  __shared__ uint32_t sm[33];
  for (int k = 0; k < 3; ++k) {
    uint32_t carry = 0;
    for (int64_t b0 = 0; b0 < nb; b0 += blockDim.x) {
      const int64_t b = b0 + threadIdx.x;
      const uint32_t v = b < nb ? cnt[3 * b + k] : 0u;
      uint32_t total;
      const uint32_t e = block_excl_scan(v, sm, &total);
      if (b < nb) pre[3 * b + k] = carry + e;
      carry += total;
    }
  }
}

// Each block writes its taken rows, in input order, as (image, row) pairs at
// their place among all taken rows, and its NULL rows of rank < null_take at
// tail[rank].  A tie is taken when its rank among the ties is in
// [tie_lo, tie_lo + need); the number of taken ties before a row follows from
// the tie count before it, so every block knows its base from the scans.
template <int DT, class K>
__global__ void __launch_bounds__(kTkThreads) k_tk_compact(const void* __restrict__ keys,
                                                          const uint8_t* __restrict__ validity, int64_t n, bool desc,
                                                          uint64_t mask, uint64_t prefix,
                                                          const uint32_t* __restrict__ pre, uint32_t tie_lo,
                                                          uint32_t need, uint32_t ksel, uint32_t null_take,
                                                          K* __restrict__ img_out, uint32_t* __restrict__ row_out,
                                                          int32_t* __restrict__ tail, int32_t* err) {
  __shared__ uint32_t sm[33];
  const int64_t b = blockIdx.x;
  uint32_t b_lt = pre[3 * b], b_tie = pre[3 * b + 1], b_null = pre[3 * b + 2];
  const int64_t base = b * kTkBlockRows;
  for (int j = 0; j < kTkItems; ++j) {
    if (base + j * kTkThreads >= n) break;  // uniform across the block
    const int64_t i = base + j * kTkThreads + threadIdx.x;
    const int k = i < n ? tk_class<DT>(keys, validity, i, desc, mask, prefix) : 3;
    const uint32_t v = k == 0 ? 1u : k == 1 ? (1u << 10) : k == 2 ? (1u << 20) : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(v, sm, &tot);
    const uint32_t lt_before = b_lt + (ex & 1023u);
    const uint32_t tie_before = b_tie + ((ex >> 10) & 1023u);
    const uint32_t taken_ties = min(max(tie_before, tie_lo), tie_lo + need) - tie_lo;
    if (k == 0 || (k == 1 && tie_before >= tie_lo && tie_before < tie_lo + need)) {
      const uint32_t pos = lt_before + (k == 0 ? taken_ties : tie_before - tie_lo);
      if (pos < ksel) {
        img_out[pos] = (K)tk_image<DT>(keys, i, desc);
        row_out[pos] = (uint32_t)i;
      } else {
        atomicExch(err, NFC_ERR_RANGE);
      }
    } else if (k == 2) {
      const uint32_t q = b_null + (ex >> 20);
      if (q < null_take) tail[q] = (int32_t)i;
    }
    b_lt += tot & 1023u;
    b_tie += (tot >> 10) & 1023u;
    b_null += tot >> 20;
  }
}

// Valid float64 rows whose key is NaN (descending top-k reverses their block).
__global__ void __launch_bounds__(kTkThreads) k_tk_nan_count(const uint64_t* __restrict__ keys,
                                                            const uint8_t* __restrict__ validity, int64_t n,
                                                            unsigned long long* cnt) {
  uint32_t c = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    c += tk_valid(validity, i) && f64_bits_isnan(keys[i]);
  c = warp_sum(c);
  if (lane_id() == 0 && c) atomicAdd(cnt, (unsigned long long)c);
}

__global__ void k_tk_reverse(int32_t* p, int64_t m) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m / 2; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = p[i];
    p[i] = p[m - 1 - i];
    p[m - 1 - i] = t;
  }
}

unsigned tk_grid(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + kTkThreads - 1) / kTkThreads, (int64_t)num_sms() * 8));
}

}  // namespace
}  // namespace nfc

using namespace nfc;

namespace {

int tk_status(cudaStream_t s, const int32_t* d_err) {
  int32_t h = 0;
  NFC_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  return h;
}

template <int DT>
int topk_impl(const void* keys, const uint8_t* validity, int64_t n, bool desc, int64_t k, int32_t* perm_out,
              cudaStream_t s) {
  using K = typename std::conditional<DT == NFC_I32, uint32_t, uint64_t>::type;
  Scratch sc(s);
  int32_t* d_err = nullptr;
  uint32_t* hist = nullptr;
  NFC_CUDA(sc.alloc(&d_err, 4));
  NFC_CUDA(sc.alloc(&hist, kTkBins));
  NFC_CUDA(cudaMemsetAsync(d_err, 0, 4 * sizeof(int32_t), s));
  // ---- selection: prefix / mask of the k-th smallest image, ties to take.
  const int bits = DT == NFC_I32 ? 32 : 64;
  uint64_t mask = 0, prefix = 0;
  int shift = bits;
  int64_t nv = 0, ksel = 0, need = 0, on_prefix = 0;
  uint32_t hh[kTkBins];
  bool first = true;
  while (shift > 0) {
    const int dbits = std::min(kTkDigitBits, shift);
    shift -= dbits;
    const uint32_t dmask = (1u << dbits) - 1u;
    NFC_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (dmask + 1), s));
    k_tk_hist<DT><<<tk_grid(n), kTkThreads, 0, s>>>(keys, validity, n, desc, mask, prefix, shift, dmask, hist);
    NFC_CUDA(cudaGetLastError());
    NFC_CUDA(cudaMemcpyAsync(hh, hist, sizeof(uint32_t) * (dmask + 1), cudaMemcpyDeviceToHost, s));
    NFC_CUDA(cudaStreamSynchronize(s));
    if (first) {
      first = false;
      for (uint32_t d = 0; d <= dmask; ++d) nv += hh[d];
      ksel = std::min(k, nv);
      need = ksel;
      if (ksel == nv) {  // every valid row is taken: all of them sit on the empty prefix
        on_prefix = nv;
        break;
      }
    }
    int64_t cum = 0;
    uint32_t d = 0;
    while (d < dmask && cum + hh[d] < need) cum += hh[d++];
    need -= cum;
    prefix |= (uint64_t)d << shift;
    mask |= (uint64_t)dmask << shift;
    on_prefix = hh[d];
    if (on_prefix == need) break;  // the whole prefix group is taken
  }
  if (on_prefix < need) {
    set_last_error("topk: selection found %lld rows on the prefix for %lld", (long long)on_prefix, (long long)need);
    return NFC_ERR_RANGE;
  }
  // Descending float64 NaNs (image 0) are taken from the end of their block.
  const int64_t tie_lo = (DT == NFC_F64 && desc && prefix == 0) ? on_prefix - need : 0;
  // ---- compaction of the taken rows (and the first k - nv NULL rows).
  const int64_t nb = (n + kTkBlockRows - 1) / kTkBlockRows;
  uint32_t *cnt = nullptr, *pre = nullptr, *row = nullptr, *row_alt = nullptr;
  K *img = nullptr, *img_alt = nullptr;
  NFC_CUDA(sc.alloc(&cnt, (size_t)(3 * nb)));
  NFC_CUDA(sc.alloc(&pre, (size_t)(3 * nb)));
  NFC_CUDA(sc.alloc(&img, (size_t)std::max<int64_t>(1, ksel)));
  NFC_CUDA(sc.alloc(&img_alt, (size_t)std::max<int64_t>(1, ksel)));
  NFC_CUDA(sc.alloc(&row, (size_t)std::max<int64_t>(1, ksel)));
  NFC_CUDA(sc.alloc(&row_alt, (size_t)std::max<int64_t>(1, ksel)));
  k_tk_count<DT><<<(unsigned)nb, kTkThreads, 0, s>>>(keys, validity, n, desc, mask, prefix, cnt);
  NFC_CUDA(cudaGetLastError());
  k_tk_scan<<<1, 1024, 0, s>>>(cnt, nb, pre);
  NFC_CUDA(cudaGetLastError());
  const int64_t null_take = k - ksel;  // NULL rows follow every valid row
  k_tk_compact<DT, K><<<(unsigned)nb, kTkThreads, 0, s>>>(keys, validity, n, desc, mask, prefix, pre,
                                                         (uint32_t)tie_lo, (uint32_t)need, (uint32_t)ksel,
                                                         (uint32_t)null_take, img, row, perm_out + ksel, d_err);
  NFC_CUDA(cudaGetLastError());
  // ---- sort of the taken rows by image (stable: they are in input order).
  if (ksel > 0) {
    K* kr = nullptr;
    uint32_t* vr = nullptr;
    int rc;
    if constexpr (DT == NFC_I32)
      rc = radix_sort_u32(img, img_alt, row, row_alt, ksel, 32, false, s, sc, d_err, &kr, &vr);
    else
      rc = radix_sort_u64(img, img_alt, row, row_alt, ksel, 64, false, s, sc, d_err, &kr, &vr);
    if (rc) return rc;
    NFC_CUDA(cudaMemcpyAsync(perm_out, vr, sizeof(int32_t) * ksel, cudaMemcpyDeviceToDevice, s));
  }
  if (DT == NFC_F64 && desc && ksel > 0) {
    unsigned long long* d_nan = nullptr;
    NFC_CUDA(sc.alloc(&d_nan, 1));
    NFC_CUDA(cudaMemsetAsync(d_nan, 0, sizeof(unsigned long long), s));
    k_tk_nan_count<<<tk_grid(n), kTkThreads, 0, s>>>(static_cast<const uint64_t*>(keys), validity, n, d_nan);
    NFC_CUDA(cudaGetLastError());
    unsigned long long h_nan = 0;
    NFC_CUDA(cudaMemcpyAsync(&h_nan, d_nan, sizeof(h_nan), cudaMemcpyDeviceToHost, s));
    NFC_CUDA(cudaStreamSynchronize(s));
    const int64_t m = std::min<int64_t>(ksel, (int64_t)h_nan);
    if (m > 1) {
      k_tk_reverse<<<tk_grid(m / 2 + 1), kTkThreads, 0, s>>>(perm_out, m);
      NFC_CUDA(cudaGetLastError());
    }
  }
  return tk_status(s, d_err);
}

}  // namespace

extern "C" int32_t nfc_sort_topk(int32_t dtype, const void* keys, const uint8_t* validity, int64_t n,
                                 int32_t descending, int64_t k, int32_t* perm_out, void* stream) {
  if (n < 0 || k < 0 || k > n) return NFC_ERR_MALFORMED;
  if (k == 0) return NFC_OK;
  if (!keys || !perm_out) return NFC_ERR_NULL;
  if (dtype != NFC_I32 && dtype != NFC_I64 && dtype != NFC_F64) return NFC_ERR_MALFORMED;
  if (n >= (1ll << 30)) {
    set_last_error("topk: n=%lld >= 2^30", (long long)n);
    return NFC_ERR_UNSUPPORTED;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (k * 8 > n || n < 65536) {
    // Most rows are kept (or few exist): the full argsort, then its first k.
    Scratch sc(s);
    int32_t* full = nullptr;
    NFC_CUDA(sc.alloc(&full, (size_t)n));
    const int32_t rc = nfc_sort_perm(dtype, keys, validity, n, descending, full, stream);
    if (rc) return rc;
    NFC_CUDA(cudaMemcpyAsync(perm_out, full, sizeof(int32_t) * k, cudaMemcpyDeviceToDevice, s));
    return NFC_OK;
  }
  const bool desc = descending != 0;
  if (dtype == NFC_I32) return topk_impl<NFC_I32>(keys, validity, n, desc, k, perm_out, s);
  if (dtype == NFC_I64) return topk_impl<NFC_I64>(keys, validity, n, desc, k, perm_out, s);
  return topk_impl<NFC_F64>(keys, validity, n, desc, k, perm_out, s);
}
