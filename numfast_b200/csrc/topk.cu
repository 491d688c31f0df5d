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
//                  every row on the prefix is taken, and the passes over the
//                  column stop once the rows on the prefix fit the candidate
//                  buffer (kTkCandCap rows).
//   2. compaction  usual case -- the selection stopped with at most
//                  kTkCandCap rows on the prefix and k <= valid rows: ONE
//                  pass (k_tk_split, 16,384-row tiles, decoupled look-back)
//                  writes the taken rows and every row on the prefix (the
//                  candidates) in input order; the candidates are sorted by
//                  image (stable) and their first `need` join the taken
//                  rows, so the rest of the selection runs on the
//                  candidates, not on the column.  Otherwise (the prefix
//                  group is taken whole, more NULL rows are needed than
//                  exist, or every digit was resolved on the column): per
//                  block of 4,096 rows, counts of taken-below, tie and NULL
//                  rows, one CTA scans them, each block writes its taken
//                  rows' (image, row) pairs in input order and the first
//                  k - valid NULL rows straight into the output tail.
//   3. sort        the k taken pairs by image, stable (radix sort; one CTA
//                  for k <= 2,048), which is the argsort's order of them.
//
// Full passes over the column in the usual case: one histogram (more only
// while the prefix group exceeds the buffer) and the split.  100M float64
// keys, k = 1,000: 0.82 ms against 8.9 ms for the full argsort.
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
constexpr int64_t kTkCandCap = 1 << 20;  // rows on the prefix that end the full passes

// Order-preserving unsigned image of a key's bits; descending complements it
// (32 bits for int32, 64 for int64 / float64).  float64: -0.0 ties +0.0 and
// every NaN maps past +inf, as in the full argsort.
template <int DT>
NFC_DEV uint64_t tk_image_bits(uint64_t raw, bool desc) {
  uint64_t u;
  if (DT == NFC_I32) {
    u = (uint32_t)raw ^ 0x80000000u;
    return desc ? (~u & 0xFFFFFFFFull) : u;
  }
  if (DT == NFC_I64) {
    u = raw ^ 0x8000000000000000ull;
  } else {
    uint64_t b = raw;
    if (f64_bits_isnan(b)) {
      u = ~0ull;
    } else {
      if (b == 0x8000000000000000ull) b = 0ull;
      u = f64_ord(b);
    }
  }
  return desc ? ~u : u;
}

template <int DT>
NFC_DEV uint64_t tk_image(const void* keys, int64_t i, bool desc) {
  const uint64_t raw = DT == NFC_I32 ? (uint64_t)(uint32_t) static_cast<const int32_t*>(keys)[i]
                                     : static_cast<const uint64_t*>(keys)[i];
  return tk_image_bits<DT>(raw, desc);
}

// Images and validity of rows i0 .. i0+3 (i0 a multiple of 4): one 16-byte
// load of int32 keys or two of 8-byte keys when `vec` (16-byte aligned
// keys), and the rows' four bits of the LSB-first bitmap (one byte).  Rows
// at or past n are invalid.
template <int DT>
NFC_DEV uint32_t tk_load4(const void* __restrict__ keys, const uint8_t* __restrict__ validity, int64_t i0,
                          int64_t n, bool vec, bool desc, uint64_t img[4]) {
  uint32_t ok = i0 + 4 <= n ? 0xFu : (i0 < n ? (1u << (uint32_t)(n - i0)) - 1u : 0u);
  if (validity && ok) ok &= (uint32_t)(__ldg(validity + (i0 >> 3)) >> (i0 & 7)) & 0xFu;
  if (vec && i0 + 4 <= n) {
    if (DT == NFC_I32) {
      const uint4 q = __ldcs(reinterpret_cast<const uint4*>(static_cast<const int32_t*>(keys) + i0));
      img[0] = tk_image_bits<DT>(q.x, desc); img[1] = tk_image_bits<DT>(q.y, desc);
      img[2] = tk_image_bits<DT>(q.z, desc); img[3] = tk_image_bits<DT>(q.w, desc);
    } else {
      const ulonglong2* p = reinterpret_cast<const ulonglong2*>(static_cast<const uint64_t*>(keys) + i0);
      const ulonglong2 a = __ldcs(p), b = __ldcs(p + 1);
      img[0] = tk_image_bits<DT>(a.x, desc); img[1] = tk_image_bits<DT>(a.y, desc);
      img[2] = tk_image_bits<DT>(b.x, desc); img[3] = tk_image_bits<DT>(b.y, desc);
    }
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r) img[r] = i0 + r < n ? tk_image<DT>(keys, i0 + r, desc) : 0ull;
  }
  return ok;
}

NFC_DEV bool tk_valid(const uint8_t* v, int64_t i) { return !v || ((v[i >> 3] >> (i & 7)) & 1u); }

// Digit histogram of the valid rows on the prefix ((image & mask) == prefix).
// Each thread takes four consecutive rows per step (16-byte loads), two steps
// in flight.  Pairs of warps count into their own copy of the histogram (four
// per CTA), which spreads the atomics of a skewed digit (the sign and
// exponent bits of float64 keys put most rows in a few bins); measured on
// 100M lognormal keys: 255 us, against 315 us merging equal digits of a warp
// with match_any first and 630 us with one shared copy.
template <int DT>
__global__ void __launch_bounds__(kTkThreads) k_tk_hist(const void* __restrict__ keys,
                                                       const uint8_t* __restrict__ validity, int64_t n, bool vec,
                                                       bool desc, uint64_t mask, uint64_t prefix, int shift,
                                                       uint32_t dmask, uint32_t* __restrict__ ghist) {
  constexpr int kCopies = 4;
  __shared__ uint32_t h[kCopies][kTkBins];
  uint32_t* hs = h[(threadIdx.x >> 6) & (kCopies - 1)];
  for (int i = threadIdx.x; i < kCopies * kTkBins; i += blockDim.x) (&h[0][0])[i] = 0u;
  __syncthreads();
  const int64_t ngroups = (n + 3) >> 2;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  constexpr int U = 2;  // groups of four rows in flight per thread
  for (int64_t g0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g0 < ngroups; g0 += U * stride) {
    uint64_t img[U][4];
    uint32_t ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t g = g0 + u * stride;
      ok[u] = g < ngroups ? tk_load4<DT>(keys, validity, g * 4, n, vec, desc, img[u]) : 0u;
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (((ok[u] >> r) & 1u) && (img[u][r] & mask) == prefix)
          atomicAdd(&hs[(uint32_t)(img[u][r] >> shift) & dmask], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= (int)dmask; i += blockDim.x) {
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kCopies; ++k) c += h[k][i];
    if (c) atomicAdd(&ghist[i], c);
  }
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

// One pass, used when the selection stopped with a prefix group of at most
// kTkCandCap rows (and every NULL row is left out: k <= valid rows): taken
// rows (image under the prefix) go to t_img/t_row and every row on the
// prefix to c_img/c_row, both in input order.  Tiles of kTkSplitRows rows
// are claimed in order; warp w of a tile takes its 2,048 contiguous rows in
// 16 steps of four consecutive rows per lane, keeping only two class bits
// per row; the tile's place in both lists comes from one decoupled
// look-back over (taken << 32 | tie) counts, and the few selected rows
// reload their key to write it out.
constexpr int kTkSplitRows = 16384;

template <int DT, class K>
__global__ void __launch_bounds__(kTkThreads) k_tk_split(const void* __restrict__ keys,
                                                        const uint8_t* __restrict__ validity, int64_t n, bool vec,
                                                        bool desc, uint64_t mask, uint64_t prefix, uint32_t n_taken,
                                                        uint32_t n_cand, K* __restrict__ t_img,
                                                        uint32_t* __restrict__ t_row, K* __restrict__ c_img,
                                                        uint32_t* __restrict__ c_row, uint64_t* lb, uint32_t* ticket,
                                                        int32_t* err) {
  constexpr int kWarps = kTkThreads / 32;
  constexpr int kSteps = kTkSplitRows / (kTkThreads * 4);  // 16 steps of 128 rows per warp
  constexpr int U = 4;                                      // steps in flight
  __shared__ int64_t s_tile;
  __shared__ uint32_t s_wt[kWarps][2];
  __shared__ uint64_t s_base;
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t row0 = tile * kTkSplitRows + (int64_t)warp * (kSteps * 128);
  uint64_t tk_bits = 0, tie_bits = 0;  // bit 4 j + r: step j, row r
#pragma unroll
  for (int j0 = 0; j0 < kSteps; j0 += U) {
    uint64_t img[U][4];
    uint32_t ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) ok[u] = tk_load4<DT>(keys, validity, row0 + (j0 + u) * 128 + lane * 4, n, vec, desc, img[u]);
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (!((ok[u] >> r) & 1u)) continue;
        const uint64_t m = img[u][r] & mask;
        if (m < prefix) tk_bits |= 1ull << (4 * (j0 + u) + r);
        else if (m == prefix) tie_bits |= 1ull << (4 * (j0 + u) + r);
      }
  }
  const uint32_t w_tk = warp_sum((uint32_t)__popcll(tk_bits)), w_tie = warp_sum((uint32_t)__popcll(tie_bits));
  if (lane == 0) { s_wt[warp][0] = w_tk; s_wt[warp][1] = w_tie; }
  __syncthreads();
  if (warp == 0) {
    uint32_t a = 0, b = 0;
    for (int w = 0; w < kWarps; ++w) { a += s_wt[w][0]; b += s_wt[w][1]; }
    const uint64_t base = (uint64_t)lookback_exclusive(lb, tile, ((uint64_t)a << 32) | b, err);  // whole warp
    if (lane == 0) s_base = base;
  }
  __syncthreads();
  if ((w_tk | w_tie) == 0) return;
  uint32_t t_pos = (uint32_t)(s_base >> 32), c_pos = (uint32_t)s_base;
  for (int w = 0; w < warp; ++w) { t_pos += s_wt[w][0]; c_pos += s_wt[w][1]; }
  for (int j = 0; j < kSteps; ++j) {
    const uint32_t tj = (uint32_t)(tk_bits >> (4 * j)) & 0xFu, cj = (uint32_t)(tie_bits >> (4 * j)) & 0xFu;
    if (!__any_sync(0xffffffffu, (tj | cj) != 0u)) continue;
    // Exclusive scan over lanes of both counts at once (<= 128 each per step).
    const uint32_t x = (uint32_t)__popc(tj) | ((uint32_t)__popc(cj) << 16);
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t tp = t_pos + ((incl - x) & 0xFFFFu), cp = c_pos + ((incl - x) >> 16);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int64_t i = row0 + j * 128 + lane * 4 + r;
      if ((tj >> r) & 1u) {
        if (tp < n_taken) { t_img[tp] = (K)tk_image<DT>(keys, i, desc); t_row[tp] = (uint32_t)i; }
        else atomicExch(err, NFC_ERR_RANGE);
        ++tp;
      } else if ((cj >> r) & 1u) {
        if (cp < n_cand) { c_img[cp] = (K)tk_image<DT>(keys, i, desc); c_row[cp] = (uint32_t)i; }
        else atomicExch(err, NFC_ERR_RANGE);
        ++cp;
      }
    }
    t_pos += tot & 0xFFFFu;
    c_pos += tot >> 16;
  }
}

// Entries whose image is 0 (descending float64: the NaN rows).
template <class K>
__global__ void __launch_bounds__(kTkThreads) k_tk_zero_count(const K* __restrict__ img, int64_t m,
                                                             unsigned long long* cnt) {
  uint32_t c = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    c += img[i] == (K)0;
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
  NFC_CUDA(readback(&h, d_err, sizeof(int32_t), s));
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
  const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0;
  // ---- selection: prefix / mask of the k-th smallest image, ties to take.
  const int bits = DT == NFC_I32 ? 32 : 64;
  uint64_t mask = 0, prefix = 0;
  int shift = bits;
  int64_t nv = 0, ksel = 0, need = 0, on_prefix = 0;
  uint32_t hh[kTkBins];
  bool first = true;
  bool use_cand = false;
  while (shift > 0) {
    const int dbits = std::min(kTkDigitBits, shift);
    shift -= dbits;
    const uint32_t dmask = (1u << dbits) - 1u;
    NFC_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (dmask + 1), s));
    k_tk_hist<DT><<<tk_grid((n + 3) / 4), kTkThreads, 0, s>>>(keys, validity, n, vec, desc, mask, prefix, shift,
                                                              dmask, hist);
    NFC_CUDA(cudaGetLastError());
    NFC_CUDA(readback(hh, hist, sizeof(uint32_t) * (dmask + 1), s));
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
    if (on_prefix <= kTkCandCap && shift > 0) {
      use_cand = true;  // the rest of the selection runs on the prefix group
      break;
    }
  }
  if (on_prefix < need) {
    set_last_error("topk: selection found %lld rows on the prefix for %lld", (long long)on_prefix, (long long)need);
    return NFC_ERR_RANGE;
  }
  // Descending float64 NaNs (image 0) are taken from the end of their block.
  const int64_t tie_lo = (DT == NFC_F64 && desc && prefix == 0) ? on_prefix - need : 0;
  // ---- compaction of the taken rows (and the first k - nv NULL rows).
  const int64_t nb = (n + kTkBlockRows - 1) / kTkBlockRows;
  uint32_t *row = nullptr, *row_alt = nullptr;
  K *img = nullptr, *img_alt = nullptr;
  NFC_CUDA(sc.alloc(&img, (size_t)std::max<int64_t>(1, ksel)));
  NFC_CUDA(sc.alloc(&img_alt, (size_t)std::max<int64_t>(1, ksel)));
  NFC_CUDA(sc.alloc(&row, (size_t)std::max<int64_t>(1, ksel)));
  NFC_CUDA(sc.alloc(&row_alt, (size_t)std::max<int64_t>(1, ksel)));
  if (!use_cand) {
    uint32_t *cnt = nullptr, *pre = nullptr;
    NFC_CUDA(sc.alloc(&cnt, (size_t)(3 * nb)));
    NFC_CUDA(sc.alloc(&pre, (size_t)(3 * nb)));
    k_tk_count<DT><<<(unsigned)nb, kTkThreads, 0, s>>>(keys, validity, n, desc, mask, prefix, cnt);
    NFC_CUDA(cudaGetLastError());
    k_tk_scan<<<1, 1024, 0, s>>>(cnt, nb, pre);
    NFC_CUDA(cudaGetLastError());
    const int64_t null_take = k - ksel;  // NULL rows follow every valid row
    k_tk_compact<DT, K><<<(unsigned)nb, kTkThreads, 0, s>>>(keys, validity, n, desc, mask, prefix, pre,
                                                           (uint32_t)tie_lo, (uint32_t)need, (uint32_t)ksel,
                                                           (uint32_t)null_take, img, row, perm_out + ksel, d_err);
    NFC_CUDA(cudaGetLastError());
  } else {
    // Taken rows (ksel - need of them) straight to img/row; the prefix group
    // to the candidate buffer, sorted by image (stable: input order within
    // equal images); its first `need` entries are the rest of the selection.
    // Descending float64 with the NaN block on the prefix (prefix 0: NaN and
    // +inf rows): when the block is cut, its last `need` rows are taken.
    // ksel < nv here, so no NULL row is part of the output.
    const int64_t cum = ksel - need;
    K *c_img = nullptr, *c_img_alt = nullptr;
    uint32_t *c_row = nullptr, *c_row_alt = nullptr;
    uint64_t* lb = nullptr;
    NFC_CUDA(sc.alloc(&c_img, (size_t)on_prefix));
    NFC_CUDA(sc.alloc(&c_img_alt, (size_t)on_prefix));
    NFC_CUDA(sc.alloc(&c_row, (size_t)on_prefix));
    NFC_CUDA(sc.alloc(&c_row_alt, (size_t)on_prefix));
    const int64_t ns = (n + kTkSplitRows - 1) / kTkSplitRows;
    NFC_CUDA(sc.alloc(&lb, (size_t)ns + 1));
    uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ns);
    NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ns + 1), s));
    k_tk_split<DT, K><<<(unsigned)ns, kTkThreads, 0, s>>>(keys, validity, n, vec, desc, mask, prefix, (uint32_t)cum,
                                                         (uint32_t)on_prefix, img, row, c_img, c_row, lb, ticket,
                                                         d_err);
    NFC_CUDA(cudaGetLastError());
    K* ckr = nullptr;
    uint32_t* cvr = nullptr;
    int rc;
    if constexpr (DT == NFC_I32)
      rc = radix_sort_u32(c_img, c_img_alt, c_row, c_row_alt, on_prefix, 32, false, s, sc, d_err, &ckr, &cvr);
    else
      rc = radix_sort_u64(c_img, c_img_alt, c_row, c_row_alt, on_prefix, 64, false, s, sc, d_err, &ckr, &cvr);
    if (rc) return rc;
    int64_t off = 0;
    if (DT == NFC_F64 && desc && prefix == 0) {
      unsigned long long* d_z = nullptr;
      NFC_CUDA(sc.alloc(&d_z, 1));
      NFC_CUDA(cudaMemsetAsync(d_z, 0, sizeof(unsigned long long), s));
      k_tk_zero_count<K><<<tk_grid(on_prefix), kTkThreads, 0, s>>>(ckr, on_prefix, d_z);
      NFC_CUDA(cudaGetLastError());
      unsigned long long h_z = 0;
      NFC_CUDA(readback(&h_z, d_z, sizeof(h_z), s));
      if ((int64_t)h_z > need) off = (int64_t)h_z - need;
    }
    NFC_CUDA(cudaMemcpyAsync(img + cum, ckr + off, sizeof(K) * need, cudaMemcpyDeviceToDevice, s));
    NFC_CUDA(cudaMemcpyAsync(row + cum, cvr + off, sizeof(uint32_t) * need, cudaMemcpyDeviceToDevice, s));
  }
  // ---- sort of the taken rows by image (stable: they are in input order).
  K* kr = nullptr;
  if (ksel > 0) {
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
    // The taken NaN rows (image 0) lead the sorted selection; reverse them.
    unsigned long long* d_nan = nullptr;
    NFC_CUDA(sc.alloc(&d_nan, 1));
    NFC_CUDA(cudaMemsetAsync(d_nan, 0, sizeof(unsigned long long), s));
    k_tk_zero_count<K><<<tk_grid(ksel), kTkThreads, 0, s>>>(kr, ksel, d_nan);
    NFC_CUDA(cudaGetLastError());
    unsigned long long h_nan = 0;
    NFC_CUDA(readback(&h_nan, d_nan, sizeof(h_nan), s));
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
