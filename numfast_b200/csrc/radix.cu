// Onesweep LSD radix sort (8-bit digits) with decoupled look-back, and the
// entry points built on it: stable argsort (ir_sort), sorted unique with
// first-occurrence rows and counts (ir_unique_inverse), and gather.
//
// Semantics follow the reference:
//   * ascending argsort == np.argsort(kind="stable")  (sort.rs:55-118);
//   * descending == _stable_desc_idx: key groups reversed, input order kept
//     inside each group (cpu.py:1154-1171) -- done by sorting ~key;
//   * float64 keys: -0.0 and +0.0 tie, NaN sorts after +inf ascending; in
//     descending order every NaN forms its own group, so NaNs come first in
//     reverse input order (what _stable_desc_idx yields, since NaN != NaN);
//   * invalid rows go last in input order (_sort_perm, cpu.py:1174-1225);
//   * unique: uniq ascending, inverse with uniq[inv] == keys (unique.rs:30-91).
//
// Pass structure: one histogram kernel computes every pass's digit counts;
// passes whose digit is constant over all keys are skipped; each remaining
// pass is ONE kernel: tiles of 8192 keys rank locally (per-warp digit peers
// from eight ballots), publish per-digit tile counts, look back over predecessor tiles
// for their global offset, stage the tile in shared memory in digit order
// and write it out in runs.
#include <algorithm>

#include "groupby_host.h"

namespace nfc {

constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 8192
constexpr uint32_t kStAgg = 1u << 30;
constexpr uint32_t kStInc = 2u << 30;
constexpr uint32_t kStVal = (1u << 30) - 1u;

template <class K>
__global__ void __launch_bounds__(256) k_radix_hist(const K* __restrict__ keys, int64_t n, int npasses,
                                                    uint32_t* __restrict__ ghist, K xr) {
  __shared__ uint32_t h[8][256];
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0u;
  __syncthreads();
  // 16-byte vector loads, U of them in flight per thread, when the keys are
  // 16-byte aligned; the scalar loop takes the rest.
  constexpr int VEC = 16 / sizeof(K);
  constexpr int U = 4;
  int64_t done = 0;
  if ((reinterpret_cast<uintptr_t>(keys) & 15u) == 0) {
    const int64_t nvec = n / VEC;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v0 < nvec; v0 += stride * U) {
      K kk[U][VEC];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t v = v0 + u * stride;
        if (v < nvec) {
          if constexpr (sizeof(K) == 4) {
            const uint4 q = __ldcs(reinterpret_cast<const uint4*>(keys) + v);
            kk[u][0] = q.x ^ xr; kk[u][1] = q.y ^ xr; kk[u][2] = q.z ^ xr; kk[u][3] = q.w ^ xr;
          } else {
            const ulonglong2 q = __ldcs(reinterpret_cast<const ulonglong2*>(keys) + v);
            kk[u][0] = q.x ^ xr; kk[u][1] = q.y ^ xr;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (v0 + u * stride < nvec)
#pragma unroll
          for (int e = 0; e < VEC; ++e)
            for (int p = 0; p < npasses; ++p) atomicAdd(&h[p][(uint32_t)(kk[u][e] >> (8 * p)) & 255u], 1u);
    }
    done = nvec * VEC;
  }
  for (int64_t i = done + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const K k = keys[i] ^ xr;
    for (int p = 0; p < npasses; ++p) atomicAdd(&h[p][(uint32_t)(k >> (8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < npasses * 256; i += blockDim.x)
    if ((&h[0][0])[i]) atomicAdd(&ghist[i], (&h[0][0])[i]);
}

// Exclusive scan of each pass's 256 bins (one block of 256 per pass).
__global__ void k_radix_scan(const uint32_t* ghist, uint32_t* base) {
  __shared__ uint32_t s_scan[33];
  const int p = blockIdx.x;
  uint32_t total;
  const uint32_t v = ghist[p * 256 + threadIdx.x];
  base[p * 256 + threadIdx.x] = block_excl_scan(v, s_scan, &total);
}

// The per-warp digit counters are dead once every element knows its tile
// position, so the staging arrays overlay them: u64 keys with u32 values fit
// in ~98 KB and two CTAs stay resident per SM.
template <class K>
struct SortSmem {
  uint32_t dstart[256];
  uint32_t gofs[256];
  uint32_t scan[33];
  uint32_t tile;
  union {
    uint32_t wh[kSortWarps][256];
    struct {
      K keys[kSortTile];
      uint32_t vals[kSortTile];
    } st;
  } u;
};

// Lanes holding the same 8-bit digit as this lane (and the same validity):
// one ballot per digit bit.  __match_any_sync serialises over the distinct
// values in the warp, which for random digits is most of the 32 lanes; eight
// ballots cost the same for any distribution.
NFC_DEV unsigned match_digit8(uint32_t d, bool ok) {
  const unsigned v = __ballot_sync(0xffffffffu, ok);
  unsigned m = ok ? v : ~v;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const bool p = (d >> b) & 1u;
    const unsigned bb = __ballot_sync(0xffffffffu, p);
    m &= p ? bb : ~bb;
  }
  return m;
}

// Keys are read as kin[i] ^ xr (the first pass of a sort from a caller's
// column applies an order-preserving flip on the way in) and written flipped.
template <class K, bool HAS_VALS, bool IOTA>
__global__ void __launch_bounds__(kSortThreads, 2) k_onesweep(const K* __restrict__ kin, K* __restrict__ kout,
                                                           const uint32_t* __restrict__ vin,
                                                           uint32_t* __restrict__ vout, int64_t n, int shift,
                                                           const uint32_t* __restrict__ digit_base,
                                                           uint32_t* __restrict__ status, uint32_t* ticket,
                                                           int32_t* err, K xr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SortSmem<K>& S = *reinterpret_cast<SortSmem<K>*>(smem_raw);
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) S.tile = atomicAdd(ticket, 1u);
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&S.u.wh[0][0])[i] = 0u;
  __syncthreads();
  const int64_t tile = S.tile;
  const int64_t base = tile * kSortTile;
  // Digits are recomputed from the keys and IOTA values from the index
  // instead of being held, which keeps two CTAs resident per SM.
  K key[kSortItems];
  uint32_t val[(HAS_VALS && !IOTA) ? kSortItems : 1];
  uint32_t rank[kSortItems];
  const int64_t wbase = base + warp * (32 * kSortItems) + lane;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const int64_t idx = wbase + j * 32;
    const bool ok = idx < n;
    key[j] = ok ? kin[idx] ^ xr : (K)0;
    if (HAS_VALS && !IOTA) val[j] = ok ? vin[idx] : 0u;
  }
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const bool ok = wbase + j * 32 < n;
    const uint32_t d = (uint32_t)(key[j] >> shift) & 255u;
    const unsigned peers = match_digit8(d, ok);
    const int leader = __ffs(peers) - 1;
    uint32_t b = 0;
    if (lane == leader && ok) {
      b = S.u.wh[warp][d];
      S.u.wh[warp][d] = b + (uint32_t)__popc(peers);
    }
    b = __shfl_sync(0xffffffffu, b, leader);
    rank[j] = b + (uint32_t)__popc(peers & lanemask_lt());
    __syncwarp();
  }
  __syncthreads();
  uint32_t tile_cnt = 0;
  if (threadIdx.x < 256) {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = S.u.wh[w][threadIdx.x];
      S.u.wh[w][threadIdx.x] = run;
      run += c;
    }
    tile_cnt = run;
  }
  uint32_t total;
  const uint32_t dstart = block_excl_scan(threadIdx.x < 256 ? tile_cnt : 0u, S.scan, &total);
  if (threadIdx.x < 256) {
    const int d = threadIdx.x;
    S.dstart[d] = dstart;
    uint32_t excl = 0;
    uint32_t* st = status + (size_t)tile * 256 + d;
    if (tile == 0) {
      __threadfence();
      atomicExch(st, kStInc | tile_cnt);
    } else {
      __threadfence();
      atomicExch(st, kStAgg | tile_cnt);
      // Windowed walk: kLbWin independent loads per round (tiles j .. j-7),
      // consumed in order up to the first inclusive or unpublished status.
      constexpr int kLbWin = 8;
      int64_t j = tile - 1;
      uint32_t spins = 0;
      bool done = false;
      while (!done) {
        uint32_t w[kLbWin];
#pragma unroll
        for (int k = 0; k < kLbWin; ++k)
          w[k] = j - k >= 0 ? ld_volatile_u32(status + (size_t)(j - k) * 256 + d) : kStInc;  // past tile 0: end
        int take = 0;
#pragma unroll
        for (int k = 0; k < kLbWin; ++k) {
          if (done) break;
          const uint32_t flag = w[k] & ~kStVal;
          if (flag == 0) break;
          excl += w[k] & kStVal;
          ++take;
          if (flag == kStInc) done = true;
        }
        if (done) break;
        if (take == 0 && ++spins > kSpinLimit) {
          atomicExch(err, NFC_ERR_TIMEOUT);
          break;
        }
        j -= take;
      }
      __threadfence();
      atomicExch(st, kStInc | (excl + tile_cnt));
    }
    S.gofs[d] = digit_base[d] + excl - dstart;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint32_t d = (uint32_t)(key[j] >> shift) & 255u;
    rank[j] += S.dstart[d] + S.u.wh[warp][d];
  }
  __syncthreads();  // the counters are overwritten by the staged tile below
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const int64_t idx = wbase + j * 32;
    if (idx < n) {
      const uint32_t p = rank[j];
      S.u.st.keys[p] = key[j];
      if (HAS_VALS) S.u.st.vals[p] = IOTA ? (uint32_t)idx : val[(HAS_VALS && !IOTA) ? j : 0];
    }
  }
  __syncthreads();
  const int tile_n = (int)std::min<int64_t>(kSortTile, n - base);
  for (int i = threadIdx.x; i < tile_n; i += kSortThreads) {
    const K k = S.u.st.keys[i];
    const uint32_t d = (uint32_t)(k >> shift) & 255u;
    const uint32_t dst = S.gofs[d] + (uint32_t)i;
    kout[dst] = k;
    if (HAS_VALS) vout[dst] = S.u.st.vals[i];
  }
}

// Inputs of at most kSmallSort keys (the distinct keys of a low-cardinality
// hash group-by, small argsorts) are sorted by one CTA: a bitonic network in
// shared memory over (masked key, input index) pairs, which makes it stable,
// then a gather of the full keys and values.  One launch and no host round
// trip, where the multi-pass sort costs a histogram read-back and up to
// eight more launches.
constexpr int kSmallSort = 2048;

template <class K>
__global__ void __launch_bounds__(1024) k_sort_small(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                     bool iota, int n, K mask, K xr, K* __restrict__ kout,
                                                     uint32_t* __restrict__ vout) {
  __shared__ K sk[kSmallSort];
  __shared__ uint32_t si[kSmallSort];
  int m = 1;
  while (m < n) m <<= 1;
  // Padding (index >= n) holds the largest key and sorts after every real key.
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    sk[i] = i < n ? ((kin[i] ^ xr) & mask) : ~(K)0;
    si[i] = (uint32_t)i;
  }
  __syncthreads();
  for (int size = 2; size <= m; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < (m >> 1); t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1));  // pair (lo, lo + stride), bit 'stride' of lo clear
        const int hi = lo + stride;
        const K a = sk[lo], b = sk[hi];
        const uint32_t ia = si[lo], ib = si[hi];
        const bool gt = a > b || (a == b && ia > ib);
        if (gt == ((lo & size) == 0)) {  // ascending where bit 'size' of lo is clear
          sk[lo] = b;
          sk[hi] = a;
          si[lo] = ib;
          si[hi] = ia;
        }
      }
      __syncthreads();
    }
  }
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const uint32_t i = si[r];
    kout[r] = kin[i] ^ xr;
    if (vout) vout[r] = iota ? i : vin[i];
  }
}

template <class K>
__global__ void k_xor_copy(const K* __restrict__ in, K xr, int64_t n, K* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i] ^ xr;
}

__global__ void k_iota(uint32_t* v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

// src (when not null) is a read-only key column that the histogram and the
// first pass read as src[i] ^ in_xor; keys / keys_alt are then only the
// ping-pong buffers, and the result never aliases src.
template <class K>
static int radix_sort_impl(K* keys, K* keys_alt, uint32_t* vals, uint32_t* vals_alt, int64_t n, int key_bits,
                           bool iota_vals, cudaStream_t s, Scratch& sc, int32_t* d_err, K** keys_result,
                           uint32_t** vals_result, const K* src = nullptr, K in_xor = 0) {
  if (!src) {
    src = keys;
    in_xor = 0;
  }
  *keys_result = keys;
  *vals_result = vals;
  if (n <= 0) return NFC_OK;
  const bool has_vals = vals != nullptr;
  if (n <= kSmallSort) {
    const K mask = key_bits >= (int)(8 * sizeof(K)) ? ~(K)0 : (K)(((K)1 << key_bits) - 1);
    k_sort_small<K><<<1, 1024, 0, s>>>(src, vals, iota_vals, (int)n, mask, in_xor, keys_alt,
                                       has_vals ? vals_alt : nullptr);
    NFC_CUDA(cudaGetLastError());
    *keys_result = keys_alt;
    if (has_vals) *vals_result = vals_alt;
    return NFC_OK;
  }
  if (n >= (1ll << 30)) {
    set_last_error("radix sort: n=%lld >= 2^30", (long long)n);
    return NFC_ERR_UNSUPPORTED;
  }
  const int npasses = (key_bits + 7) / 8;
  uint32_t* hist = nullptr;
  uint32_t* dbase = nullptr;
  NFC_CUDA(sc.alloc(&hist, 2 * 8 * 256));
  dbase = hist + 8 * 256;
  NFC_CUDA(cudaMemsetAsync(hist, 0, 8 * 256 * sizeof(uint32_t), s));
  {
    int64_t g = std::min<int64_t>((n + 4095) / 4096, (int64_t)num_sms() * 4);
    k_radix_hist<K><<<(unsigned)std::max<int64_t>(g, 1), 256, 0, s>>>(src, n, npasses, hist, in_xor);
    NFC_CUDA(cudaGetLastError());
  }
  k_radix_scan<<<npasses, 256, 0, s>>>(hist, dbase);
  NFC_CUDA(cudaGetLastError());
  uint32_t hh[8 * 256];
  NFC_CUDA(readback(hh, hist, sizeof(uint32_t) * 256 * npasses, s));
  const int64_t ntiles = (n + kSortTile - 1) / kSortTile;
  uint32_t* status = nullptr;
  uint32_t* ticket = nullptr;
  NFC_CUDA(sc.alloc(&status, (size_t)ntiles * 256 + 64));
  ticket = status + (size_t)ntiles * 256;
  const size_t smem = sizeof(SortSmem<K>);
  if (has_vals) {
    NFC_CUDA(cudaFuncSetAttribute(k_onesweep<K, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    NFC_CUDA(cudaFuncSetAttribute(k_onesweep<K, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  } else {
    NFC_CUDA(cudaFuncSetAttribute(k_onesweep<K, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  const K* kin = src;
  K* kout = src == keys ? keys_alt : keys;
  K xr = in_xor;
  uint32_t* vin = vals;
  uint32_t* vout = vals_alt;
  bool need_iota = has_vals && iota_vals;
  for (int p = 0; p < npasses; ++p) {
    bool trivial = false;
    for (int d = 0; d < 256; ++d)
      if ((int64_t)hh[p * 256 + d] == n) trivial = true;
    if (trivial) continue;
    NFC_CUDA(cudaMemsetAsync(status, 0, ((size_t)ntiles * 256 + 64) * sizeof(uint32_t), s));
    if (has_vals && need_iota)
      k_onesweep<K, true, true><<<(unsigned)ntiles, kSortThreads, smem, s>>>(kin, kout, vin, vout, n, 8 * p,
                                                                             dbase + 256 * p, status, ticket, d_err,
                                                                             xr);
    else if (has_vals)
      k_onesweep<K, true, false><<<(unsigned)ntiles, kSortThreads, smem, s>>>(kin, kout, vin, vout, n, 8 * p,
                                                                              dbase + 256 * p, status, ticket, d_err,
                                                                              xr);
    else
      k_onesweep<K, false, false><<<(unsigned)ntiles, kSortThreads, smem, s>>>(kin, kout, vin, vout, n, 8 * p,
                                                                               dbase + 256 * p, status, ticket,
                                                                               d_err, xr);
    NFC_CUDA(cudaGetLastError());
    need_iota = false;
    xr = 0;
    K* written = kout;
    kout = written == keys ? keys_alt : keys;
    kin = written;
    std::swap(vin, vout);
  }
  const unsigned g1 = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8);
  if (kin == src && src != keys) {
    // Every pass was trivial (all keys equal in the sorted bits): the result
    // is the source itself, flipped into the first buffer.
    k_xor_copy<K><<<g1, 256, 0, s>>>(src, in_xor, n, keys);
    NFC_CUDA(cudaGetLastError());
    kin = keys;
  }
  if (need_iota) {
    // Every pass was trivial: the input order is already sorted.
    k_iota<<<g1, 256, 0, s>>>(vin, n);
    NFC_CUDA(cudaGetLastError());
  }
  *keys_result = const_cast<K*>(kin);
  *vals_result = vin;
  return NFC_OK;
}

int radix_sort_u32(uint32_t* keys, uint32_t* keys_alt, uint32_t* vals, uint32_t* vals_alt, int64_t n, int key_bits,
                   bool iota_vals, cudaStream_t s, Scratch& sc, int32_t* d_err, uint32_t** kr, uint32_t** vr) {
  return radix_sort_impl<uint32_t>(keys, keys_alt, vals, vals_alt, n, key_bits, iota_vals, s, sc, d_err, kr, vr);
}
int radix_sort_u32_from(const uint32_t* src, uint32_t in_xor, uint32_t* keys, uint32_t* keys_alt, uint32_t* vals,
                        uint32_t* vals_alt, int64_t n, int key_bits, bool iota_vals, cudaStream_t s, Scratch& sc,
                        int32_t* d_err, uint32_t** kr, uint32_t** vr) {
  return radix_sort_impl<uint32_t>(keys, keys_alt, vals, vals_alt, n, key_bits, iota_vals, s, sc, d_err, kr, vr, src,
                                   in_xor);
}
int radix_sort_u64(uint64_t* keys, uint64_t* keys_alt, uint32_t* vals, uint32_t* vals_alt, int64_t n, int key_bits,
                   bool iota_vals, cudaStream_t s, Scratch& sc, int32_t* d_err, uint64_t** kr, uint32_t** vr) {
  return radix_sort_impl<uint64_t>(keys, keys_alt, vals, vals_alt, n, key_bits, iota_vals, s, sc, d_err, kr, vr);
}

// ---------------------------------------------------------------------
// Key transforms (order-preserving maps to unsigned).
// ---------------------------------------------------------------------
__global__ void k_xform_i32(const int32_t* __restrict__ in, const uint32_t* __restrict__ pos, int64_t n, bool desc,
                            uint32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)in[pos ? pos[i] : i] ^ 0x80000000u;
    out[i] = desc ? ~u : u;
  }
}

__global__ void k_xform_i64(const int64_t* __restrict__ in, const uint32_t* __restrict__ pos, int64_t n, bool desc,
                            uint64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t u = (uint64_t)in[pos ? pos[i] : i] ^ 0x8000000000000000ull;
    out[i] = desc ? ~u : u;
  }
}

// float64: -0.0 -> +0.0 (they tie), every NaN -> all-ones (after +inf).
__global__ void k_xform_f64(const uint64_t* __restrict__ in, const uint32_t* __restrict__ pos, int64_t n, bool desc,
                            uint64_t* __restrict__ out, unsigned long long* nan_count) {
  uint32_t nans = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t b = in[pos ? pos[i] : i];
    uint64_t u;
    if (f64_bits_isnan(b)) { u = ~0ull; ++nans; }
    else {
      if (b == 0x8000000000000000ull) b = 0ull;
      u = f64_ord(b);
    }
    out[i] = desc ? ~u : u;
  }
  nans = warp_sum(nans);
  if (lane_id() == 0 && nans) atomicAdd(nan_count, (unsigned long long)nans);
}

// Reverse perm[0:k] (the NaN block of a descending float sort).
__global__ void k_reverse_prefix(uint32_t* perm, const unsigned long long* kptr) {
  const int64_t k = (int64_t)*kptr;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k / 2; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t t = perm[i];
    perm[i] = perm[k - 1 - i];
    perm[k - 1 - i] = t;
  }
}

// ---------------------------------------------------------------------
// Stable compaction of row positions by a validity bitmap: valid rows
// first, then (when ipos_tail is given) invalid rows, both in input order.
// Tiles of kSvTile rows are claimed in order; a warp takes 2,048 rows as 64
// steps of 32, and the bitmap word of a step is the warp's ballot of its
// rows: a lane's place is one popc, a step's stores are contiguous.  One
// decoupled look-back per tile gives its valid base; an invalid row's place
// is its row number minus the valid rows before it.
// ---------------------------------------------------------------------
constexpr int kSvTile = 16384;

// Validity bits of rows [32 g, 32 g + 32), zero past n.
NFC_DEV uint32_t sv_word(const uint8_t* __restrict__ bm, int64_t g, int64_t n, bool word_aligned) {
  const int64_t r0 = g * 32;
  if (r0 >= n) return 0u;
  const int64_t rem = n - r0;
  uint32_t w;
  if (word_aligned && rem >= 32) {
    w = __ldg(reinterpret_cast<const uint32_t*>(bm) + g);
  } else {
    w = 0u;
    const int nbytes = rem >= 32 ? 4 : (int)((rem + 7) >> 3);
    for (int i = 0; i < nbytes; ++i) w |= (uint32_t)__ldg(bm + 4 * g + i) << (8 * i);
  }
  return rem < 32 ? w & ((1u << rem) - 1u) : w;
}

__global__ void __launch_bounds__(256) k_split_valid(const uint8_t* __restrict__ bm, int64_t n, bool word_aligned,
                                                     uint32_t* __restrict__ vpos, uint32_t* __restrict__ ipos_tail,
                                                     uint64_t* lb, uint32_t* ticket, int64_t* nvalid_out,
                                                     int32_t* err) {
  __shared__ int64_t s_tile, s_base;
  __shared__ uint32_t s_wc[8];
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t ntiles = (n + kSvTile - 1) / kSvTile;
  if (tile >= ntiles) return;
  const int64_t w0 = tile * kSvTile + (int64_t)warp * 2048;  // first row of this warp
  uint32_t wv[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) wv[q] = sv_word(bm, (w0 >> 5) + q * 32 + lane, n, word_aligned);
  const uint32_t wc = warp_sum((uint32_t)(__popc(wv[0]) + __popc(wv[1])));
  if (lane == 0) s_wc[warp] = wc;
  __syncthreads();
  if (warp == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < 8; ++w) tot += s_wc[w];
    const int64_t base = lookback_exclusive(lb, tile, tot, err);  // whole warp
    if (lane == 0) {
      s_base = base;
      if (tile == ntiles - 1) *nvalid_out = base + tot;
    }
  }
  __syncthreads();
  int64_t v = s_base;
  for (int w = 0; w < warp; ++w) v += s_wc[w];
  const unsigned lt = lanemask_lt();
  for (int st = 0; st < 64; ++st) {
    const int64_t row0 = w0 + 32 * st;
    if (row0 >= n) break;  // uniform across the warp
    const uint32_t word = __shfl_sync(0xffffffffu, wv[st >> 5], st & 31);
    const int64_t r = row0 + lane;
    const int64_t before = v + __popc(word & lt);
    if ((word >> lane) & 1u) vpos[before] = (uint32_t)r;
    else if (ipos_tail && r < n) ipos_tail[r - before] = (uint32_t)r;
    v += __popc(word);
  }
}

template <class T>
__global__ void k_gather(const T* __restrict__ src, const int32_t* __restrict__ idx, int64_t n, int64_t nsrc,
                         T* __restrict__ dst, int32_t* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t j = idx[i];
    if (j < 0 || j >= nsrc) { atomicExch(err, NFC_ERR_RANGE); continue; }
    dst[i] = src[j];
  }
}

static unsigned grid1d(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8));
}

static int read_status(cudaStream_t s, const int32_t* d_err) {
  int32_t h = 0;
  NFC_CUDA(readback(&h, d_err, sizeof(int32_t), s));
  if (h) set_last_error("device status %d", h);
  return h;
}

// Argsort core: the stable argsort of n keys (keys[pos[i]] when pos holds
// the valid rows' positions, else keys[0..n-1]).  The payload
// that rides through the radix passes is the row number itself: the iota
// without pos, else pos (the caller's scratch, overwritten), so the result
// is the permutation of original rows with no gather afterwards.
static int argsort_core(int32_t dtype, const void* keys, uint32_t* pos, int64_t n, bool desc, uint32_t* perm_out,
                        cudaStream_t s, Scratch& sc, int32_t* d_err) {
  if (n == 0) return NFC_OK;
  uint32_t* vals_alt = nullptr;
  NFC_CUDA(sc.alloc(&vals_alt, (size_t)n));
  uint32_t* vals = pos ? pos : perm_out;
  const bool iota = pos == nullptr;
  uint32_t* vres = nullptr;
  unsigned long long* nan_cnt = nullptr;
  bool nan_fix = false;
  if (dtype == NFC_I32) {
    uint32_t *k0 = nullptr, *k1 = nullptr, *kres = nullptr;
    NFC_CUDA(sc.alloc(&k0, (size_t)n));
    NFC_CUDA(sc.alloc(&k1, (size_t)n));
    k_xform_i32<<<grid1d(n), 256, 0, s>>>(static_cast<const int32_t*>(keys), pos, n, desc, k0);
    NFC_CUDA(cudaGetLastError());
    int rc = radix_sort_u32(k0, k1, vals, vals_alt, n, 32, iota, s, sc, d_err, &kres, &vres);
    if (rc) return rc;
  } else {
    uint64_t *k0 = nullptr, *k1 = nullptr, *kres = nullptr;
    NFC_CUDA(sc.alloc(&k0, (size_t)n));
    NFC_CUDA(sc.alloc(&k1, (size_t)n));
    if (dtype == NFC_I64) {
      k_xform_i64<<<grid1d(n), 256, 0, s>>>(static_cast<const int64_t*>(keys), pos, n, desc, k0);
    } else {
      NFC_CUDA(sc.alloc(&nan_cnt, 1));
      NFC_CUDA(cudaMemsetAsync(nan_cnt, 0, sizeof(unsigned long long), s));
      k_xform_f64<<<grid1d(n), 256, 0, s>>>(static_cast<const uint64_t*>(keys), pos, n, desc, k0, nan_cnt);
      nan_fix = desc;
    }
    NFC_CUDA(cudaGetLastError());
    int rc = radix_sort_u64(k0, k1, vals, vals_alt, n, 64, iota, s, sc, d_err, &kres, &vres);
    if (rc) return rc;
  }
  if (vres != perm_out) NFC_CUDA(cudaMemcpyAsync(perm_out, vres, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
  if (nan_fix) {
    k_reverse_prefix<<<grid1d(n / 2 + 1), 256, 0, s>>>(perm_out, nan_cnt);
    NFC_CUDA(cudaGetLastError());
  }
  return NFC_OK;
}

// Run-encode over sorted keys: heads, run ids, outputs.  A tile is 4096
// sorted elements, 16 consecutive per thread (128-bit loads).
constexpr int kRunPer = 16;
constexpr int kRunTile = 256 * kRunPer;

// Runs of the sorted keys: uniq / first row / count per run.  Registers are
// capped for four CTAs per SM (three at the 79 the compiler picks unbounded;
// 200M unique keys 8.18 -> 8.06 ms; five CTAs at 48 registers, 8.11 ms).
// A run's count is written here when its end (the next head) lies in the
// same tile; the last run of each tile is left to k_run_fix, which reads the
// start of the next run (run_start is written for the first run of every
// tile only).
__global__ void __launch_bounds__(256, 4) k_runs(const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ perm,
                                              int64_t n, int32_t* uniq, int32_t* first, int64_t* counts,
                                              uint32_t* run_start, int64_t* tile_q, uint32_t* tile_start,
                                              int32_t* inv, uint64_t* lb, uint32_t* ticket, int64_t* ng_out,
                                              int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  // The tile's runs, staged so that their outputs leave as contiguous blocks
  // (each thread owns 16 consecutive sorted elements, so direct stores from
  // the threads would land 64 B apart across a warp).
  __shared__ int32_t s_uniq[kRunTile];
  __shared__ int32_t s_first[kRunTile];
  __shared__ uint16_t s_rs[kRunTile];
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t ntiles = (n + kRunTile - 1) / kRunTile;
  if (tile >= ntiles) return;
  const int64_t tile0 = tile * kRunTile;
  const int64_t i0 = tile0 + (int64_t)threadIdx.x * kRunPer;
  uint32_t k[kRunPer], pm[kRunPer];
  if (i0 + kRunPer <= n) {
#pragma unroll
    for (int q = 0; q < kRunPer / 4; ++q) {
      const uint4 v = *reinterpret_cast<const uint4*>(skeys + i0 + 4 * q);
      k[4 * q] = v.x; k[4 * q + 1] = v.y; k[4 * q + 2] = v.z; k[4 * q + 3] = v.w;
      const uint4 w = *reinterpret_cast<const uint4*>(perm + i0 + 4 * q);
      pm[4 * q] = w.x; pm[4 * q + 1] = w.y; pm[4 * q + 2] = w.z; pm[4 * q + 3] = w.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kRunPer; ++j) {
      k[j] = i0 + j < n ? skeys[i0 + j] : 0u;
      pm[j] = i0 + j < n ? perm[i0 + j] : 0u;
    }
  }
  const uint32_t prev = (i0 > 0 && i0 < n) ? skeys[i0 - 1] : 0u;
  uint32_t heads = 0, c = 0;
#pragma unroll
  for (int j = 0; j < kRunPer; ++j) {
    const int64_t i = i0 + j;
    if (i < n) {
      const bool h = (i == 0) || (j == 0 ? prev != k[0] : k[j - 1] != k[j]);
      if (h) { heads |= 1u << j; ++c; }
    }
  }
  uint32_t total;
  const uint32_t excl = block_excl_scan(c, s_scan, &total);
  if (threadIdx.x < 32) {
    const int64_t lbx = lookback_exclusive(lb, tile, total, err);  // whole warp
    if (threadIdx.x == 0) {
      s_base = lbx;
      if (tile == ntiles - 1) *ng_out = s_base + total;
    }
  }
  __syncthreads();
  const int64_t base = s_base;
  int32_t l = (int32_t)excl - 1;  // tile-local run of the element before i0's first head
#pragma unroll
  for (int j = 0; j < kRunPer; ++j) {
    const int64_t i = i0 + j;
    if (i >= n) break;
    if (heads & (1u << j)) {
      ++l;
      s_uniq[l] = (int32_t)(k[j] ^ 0x80000000u);
      s_first[l] = (int32_t)pm[j];
      s_rs[l] = (uint16_t)(i - tile0);
    }
    if (inv) inv[pm[j]] = (int32_t)(base + l);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < (int)total; t += blockDim.x) {
    uniq[base + t] = s_uniq[t];
    first[base + t] = s_first[t];
    if (t + 1 < (int)total) counts[base + t] = (int64_t)s_rs[t + 1] - (int64_t)s_rs[t];
    if (t == 0) run_start[base] = (uint32_t)(tile0 + s_rs[0]);
  }
  if (threadIdx.x == 0) {
    tile_q[tile] = total ? base + (int64_t)total - 1 : -1;
    tile_start[tile] = total ? (uint32_t)(tile0 + s_rs[total - 1]) : 0u;
  }
}

// Count of the last run of each tile: it ends where the next run starts (the
// first run of a later tile) or at n.
__global__ void k_run_fix(const int64_t* tile_q, const uint32_t* tile_start, const uint32_t* run_start,
                          const int64_t* ng_ptr, int64_t n, int64_t ntiles, int64_t* counts) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int64_t q = tile_q[t];
  if (q < 0) return;
  const int64_t end = q + 1 < *ng_ptr ? (int64_t)run_start[q + 1] : n;
  counts[q] = end - (int64_t)tile_start[t];
}


// ---------------------------------------------------------------------
// Low-cardinality unique: per-CTA shared-memory hash tables (warp-level
// run aggregation with match_any), merged into one small global table.
// A CTA whose table passes half full flags overflow and stops; the caller
// then takes the radix-sort path.  Slot word = 1<<32 | key, 0 = empty.
// ---------------------------------------------------------------------
constexpr int kLcSlots = 4096;       // per-CTA table
constexpr int kLcGlobalSlots = 8192; // merged table (at most kLcSlots/2 keys survive)
// Linear probing at load <= 0.5 needs a few probes; a key that finds neither
// itself nor a free slot within kLcMaxProbe counts as an overflow (the call
// then sorts), so a table that other warps filled past the threshold in the
// same round is never walked end to end.
constexpr int kLcMaxProbe = 128;

struct LowCard {
  unsigned long long* gkey;  // [kLcGlobalSlots]
  uint32_t* gfirst;          // [kLcGlobalSlots]
  unsigned long long* gcnt;  // [kLcGlobalSlots]
  int32_t* overflow;         // [1]
  uint32_t* gused;           // [1]
};

NFC_DEV uint32_t lc_hash(uint32_t k) { return (k * 0x9E3779B1u) ^ (k >> 15); }

__global__ void __launch_bounds__(512) k_unique_lowcard(const int32_t* __restrict__ keys, int64_t n, LowCard lc) {
  extern __shared__ __align__(16) unsigned char lc_smem[];  // kLcSlots * 16 bytes
  unsigned long long* s_key = reinterpret_cast<unsigned long long*>(lc_smem);
  uint32_t* s_first = reinterpret_cast<uint32_t*>(s_key + kLcSlots);
  uint32_t* s_cnt = s_first + kLcSlots;
  __shared__ uint32_t s_used;
  __shared__ int s_over;
  for (int i = threadIdx.x; i < kLcSlots; i += blockDim.x) { s_key[i] = 0ull; s_first[i] = 0xFFFFFFFFu; s_cnt[i] = 0u; }
  if (threadIdx.x == 0) { s_used = 0; s_over = 0; }
  __syncthreads();
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t nchunks = (n + 127) / 128;
  // The next chunk's four keys are loaded while this one is processed, and
  // the grid's overflow flag read here is used on the next iteration, so no
  // global round trip sits in front of a chunk's work.
  uint32_t key[4], nkey[4];
  auto load = [&](int64_t c, uint32_t* k) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t row = c * 128 + j * 32 + lane;
      k[j] = c < nchunks && row < n ? (uint32_t)__ldcs(keys + row) : 0u;
    }
  };
  load(gw, key);
  int gstop = 0;
  for (int64_t ch = gw; ch < nchunks; ch += nw) {
    // Stop at any CTA's overflow (the call then sorts): the first CTA to
    // overflow raises the global flag at once, so the rest of the grid stops
    // within a chunk or two instead of filling its own table first.  The
    // decision is taken by the whole warp at once: a lane that has just set
    // s_over must not leave while the others go on into the warp-wide
    // intrinsics below.
    if (__any_sync(0xffffffffu, *(volatile int*)&s_over || gstop)) break;
    gstop = *(volatile int32_t*)lc.overflow;
    load(ch + nw, nkey);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t row = ch * 128 + j * 32 + lane;
      const bool ok = row < n;
      const unsigned act = __ballot_sync(0xffffffffu, ok);
      const unsigned peers = __match_any_sync(0xffffffffu, key[j]) & act;
      if (ok && (__ffs(peers) - 1) == lane) {
        // Leader of a run of equal keys in this warp: its row is the smallest.
        const unsigned long long want = (1ull << 32) | key[j];
        uint32_t slot = lc_hash(key[j]) & (kLcSlots - 1);
        bool placed = false;
        for (int probe = 0; probe < kLcMaxProbe; ++probe) {
          unsigned long long cur = s_key[slot];
          if (cur == 0ull) {
            cur = atomicCAS(&s_key[slot], 0ull, want);
            if (cur == 0ull) {
              // Only the CTA's first overflow raises the grid's flag: every
              // insert after the threshold doing it made one global address
              // take hundreds of thousands of atomics.
              if (atomicAdd(&s_used, 1u) >= kLcSlots / 2 && atomicExch(&s_over, 1) == 0) atomicExch(lc.overflow, 1);
              cur = want;
            }
          }
          if (cur == want) {
            atomicMin(&s_first[slot], (uint32_t)row);
            atomicAdd(&s_cnt[slot], (uint32_t)__popc(peers));
            placed = true;
            break;
          }
          slot = (slot + 1) & (kLcSlots - 1);
        }
        if (!placed && atomicExch(&s_over, 1) == 0) atomicExch(lc.overflow, 1);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) key[j] = nkey[j];
  }
  __syncthreads();
  if (s_over) {
    if (threadIdx.x == 0) atomicExch(lc.overflow, 1);
    return;
  }
  if (*(volatile int32_t*)lc.overflow) return;  // another CTA overflowed: this table is not needed
  // Merge into the global table.
  for (int i = threadIdx.x; i < kLcSlots; i += blockDim.x) {
    const unsigned long long w = s_key[i];
    if (!w) continue;
    uint32_t slot = lc_hash((uint32_t)w) & (kLcGlobalSlots - 1);
    bool placed = false;
    for (int probe = 0; probe < kLcMaxProbe; ++probe) {
      unsigned long long cur = lc.gkey[slot];
      if (cur == 0ull) {
        cur = atomicCAS(&lc.gkey[slot], 0ull, w);
        if (cur == 0ull) {
          if (atomicAdd(lc.gused, 1u) == kLcGlobalSlots / 2) atomicExch(lc.overflow, 1);
          cur = w;
        }
      }
      if (cur == w) {
        atomicMin(&lc.gfirst[slot], s_first[i]);
        atomicAdd(&lc.gcnt[slot], (unsigned long long)s_cnt[i]);
        placed = true;
        break;
      }
      slot = (slot + 1) & (kLcGlobalSlots - 1);
    }
    if (!placed) atomicExch(lc.overflow, 1);
  }
}

// One CTA: compact the global table, bitonic-sort it by key (order-preserving
// u32 encoding), emit uniq/first/counts, keep each slot's rank for inverse.
__global__ void __launch_bounds__(1024) k_unique_lowcard_emit(LowCard lc, int32_t* uniq, int32_t* first,
                                                              int64_t* counts, uint32_t* slot_rank,
                                                              int64_t* ng_out) {
  constexpr int N = kLcGlobalSlots / 2;  // at most this many keys
  __shared__ unsigned long long s_sort[N];  // (ordered key << 32) | slot
  __shared__ uint32_t s_n;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < kLcGlobalSlots; i += blockDim.x) {
    const unsigned long long w = lc.gkey[i];
    if (w) {
      const uint32_t p = atomicAdd(&s_n, 1u);
      if (p < (uint32_t)N) s_sort[p] = ((unsigned long long)((uint32_t)w ^ 0x80000000u) << 32) | (uint32_t)i;
    }
  }
  __syncthreads();
  const int m = (int)min(s_n, (uint32_t)N);
  for (int i = m + threadIdx.x; i < N; i += blockDim.x) s_sort[i] = ~0ull;
  __syncthreads();
  for (int k = 2; k <= N; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = s_sort[i], b = s_sort[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) { s_sort[i] = b; s_sort[ixj] = a; }
        }
      }
      __syncthreads();
    }
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const unsigned long long e = s_sort[r];
    const uint32_t slot = (uint32_t)e;
    uniq[r] = (int32_t)((uint32_t)(e >> 32) ^ 0x80000000u);
    first[r] = (int32_t)lc.gfirst[slot];
    counts[r] = (int64_t)lc.gcnt[slot];
    if (slot_rank) slot_rank[slot] = (uint32_t)r;
  }
  if (threadIdx.x == 0) *ng_out = m;
}

__global__ void k_unique_lowcard_inverse(const int32_t* __restrict__ keys, int64_t n, LowCard lc,
                                         const uint32_t* __restrict__ slot_rank, int32_t* __restrict__ inv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t key = (uint32_t)keys[i];
    const unsigned long long want = (1ull << 32) | key;
    uint32_t slot = lc_hash(key) & (kLcGlobalSlots - 1);
    int32_t r = -1;
    for (int probe = 0; probe < kLcGlobalSlots; ++probe) {
      const unsigned long long cur = lc.gkey[slot];
      if (cur == want) { r = (int32_t)slot_rank[slot]; break; }
      if (cur == 0ull) break;
      slot = (slot + 1) & (kLcGlobalSlots - 1);
    }
    inv[i] = r;
  }
}

}  // namespace nfc

using namespace nfc;

int nfc::valid_positions(const uint8_t* bm, int64_t n, uint32_t* pos, int64_t* nv_out, cudaStream_t s, Scratch& sc,
                         int32_t* d_err) {
  *nv_out = 0;
  if (n <= 0) return NFC_OK;
  const int64_t ntiles = (n + kSvTile - 1) / kSvTile;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 2));
  int64_t* d_nv = reinterpret_cast<int64_t*>(lb + ntiles);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles + 1);
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 2), s));
  k_split_valid<<<(unsigned)ntiles, 256, 0, s>>>(bm, n, (reinterpret_cast<uintptr_t>(bm) & 3u) == 0, pos, nullptr, lb,
                                                 ticket, d_nv, d_err);
  NFC_CUDA(cudaGetLastError());
  NFC_CUDA(readback(nv_out, d_nv, sizeof(int64_t), s));
  return NFC_OK;
}

int nfc::sort_valid_rows_i32(const int32_t* keys, const uint32_t* vmask, int64_t n, int64_t n_valid, uint32_t* perm_out,
                        cudaStream_t s, Scratch& sc, int32_t* d_err) {
  if (n_valid <= 0) return NFC_OK;
  if (n_valid >= (1ll << 30)) {
    set_last_error("sort: %lld valid rows >= 2^30", (long long)n_valid);
    return NFC_ERR_UNSUPPORTED;
  }
  if (!vmask) return argsort_core(NFC_I32, keys, nullptr, n, false, perm_out, s, sc, d_err);
  const int64_t ntiles = (n + kSvTile - 1) / kSvTile;
  uint32_t* vpos = nullptr;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&vpos, (size_t)n_valid));
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 2));
  int64_t* d_nv = reinterpret_cast<int64_t*>(lb + ntiles);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles + 1);
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 2), s));
  k_split_valid<<<(unsigned)ntiles, 256, 0, s>>>(reinterpret_cast<const uint8_t*>(vmask), n, true, vpos, nullptr,
                                                 lb, ticket, d_nv, d_err);
  NFC_CUDA(cudaGetLastError());
  return argsort_core(NFC_I32, keys, vpos, n_valid, false, perm_out, s, sc, d_err);
}

extern "C" int32_t nfc_sort_perm(int32_t dtype, const void* keys, const uint8_t* validity, int64_t n,
                                 int32_t descending, int32_t* perm_out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (n == 0) return NFC_OK;
  if (!keys || !perm_out) return NFC_ERR_NULL;
  if (dtype != NFC_I32 && dtype != NFC_I64 && dtype != NFC_F64) return NFC_ERR_MALFORMED;
  if (n >= (1ll << 30)) {
    set_last_error("sort: n=%lld >= 2^30", (long long)n);
    return NFC_ERR_UNSUPPORTED;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  int32_t* d_err = nullptr;
  NFC_CUDA(sc.alloc(&d_err, 4));
  NFC_CUDA(cudaMemsetAsync(d_err, 0, 4 * sizeof(int32_t), s));
  uint32_t* perm = reinterpret_cast<uint32_t*>(perm_out);
  if (!validity) {
    int rc = argsort_core(dtype, keys, nullptr, n, descending != 0, perm, s, sc, d_err);
    if (rc) return rc;
    return read_status(s, d_err);
  }
  // Valid rows first (compacted positions), invalid rows appended.
  const int64_t ntiles = (n + kSvTile - 1) / kSvTile;
  uint32_t* vpos = nullptr;
  uint64_t* lb = nullptr;
  int64_t* d_nv = nullptr;
  NFC_CUDA(sc.alloc(&vpos, (size_t)n));
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 2));
  d_nv = reinterpret_cast<int64_t*>(lb + ntiles);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles + 1);
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 2), s));
  // ipos is written straight into the tail of perm_out: invalid row number
  // q (in input order) lands at perm_out[n_valid + q]; we do not know
  // n_valid yet, so stage it at the front of a scratch copy.
  uint32_t* ipos = nullptr;
  NFC_CUDA(sc.alloc(&ipos, (size_t)n));
  k_split_valid<<<(unsigned)ntiles, 256, 0, s>>>(validity, n, (reinterpret_cast<uintptr_t>(validity) & 3u) == 0, vpos,
                                                 ipos, lb, ticket, d_nv, d_err);
  NFC_CUDA(cudaGetLastError());
  int64_t nv = 0;
  NFC_CUDA(readback(&nv, d_nv, sizeof(int64_t), s));
  int rc = argsort_core(dtype, keys, vpos, nv, descending != 0, perm, s, sc, d_err);
  if (rc) return rc;
  if (n - nv > 0)
    NFC_CUDA(cudaMemcpyAsync(perm + nv, ipos, sizeof(uint32_t) * (n - nv), cudaMemcpyDeviceToDevice, s));
  return read_status(s, d_err);
}

extern "C" int32_t nfc_gather(int32_t elem_bytes, const void* values, int64_t nvalues, const int32_t* idx, int64_t n,
                              void* out, void* stream) {
  if (n < 0 || nvalues < 0) return NFC_ERR_MALFORMED;
  if (n == 0) return NFC_OK;
  if (!values || !idx || !out) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  int32_t* d_err = nullptr;
  NFC_CUDA(sc.alloc(&d_err, 1));
  NFC_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int32_t), s));
  if (elem_bytes == 4)
    k_gather<uint32_t><<<grid1d(n), 256, 0, s>>>(static_cast<const uint32_t*>(values), idx, n, nvalues,
                                                 static_cast<uint32_t*>(out), d_err);
  else if (elem_bytes == 8)
    k_gather<uint64_t><<<grid1d(n), 256, 0, s>>>(static_cast<const uint64_t*>(values), idx, n, nvalues,
                                                 static_cast<uint64_t*>(out), d_err);
  else
    return NFC_ERR_MALFORMED;
  NFC_CUDA(cudaGetLastError());
  return read_status(s, d_err);
}

extern "C" int64_t nfc_unique(const int32_t* keys, int64_t n, int32_t* uniq_out, int32_t* first_out,
                              int64_t* counts_out, int32_t* inv_out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (n == 0) return 0;
  if (!keys || !uniq_out || !first_out || !counts_out) return NFC_ERR_NULL;
  if (n >= (1ll << 30)) {
    set_last_error("unique: n=%lld >= 2^30", (long long)n);
    return NFC_ERR_UNSUPPORTED;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  int32_t* d_err = nullptr;
  NFC_CUDA(sc.alloc(&d_err, 4));
  NFC_CUDA(cudaMemsetAsync(d_err, 0, 4 * sizeof(int32_t), s));
  {
    // Few distinct keys: shared-memory hash tables, no sort of the rows.
    unsigned char* lcb = nullptr;
    const size_t lc_bytes = (size_t)kLcGlobalSlots * (8 + 4 + 8 + 4) + 64;
    NFC_CUDA(sc.alloc(&lcb, lc_bytes));
    LowCard lc;
    lc.gkey = reinterpret_cast<unsigned long long*>(lcb);
    lc.gcnt = lc.gkey + kLcGlobalSlots;
    lc.gfirst = reinterpret_cast<uint32_t*>(lc.gcnt + kLcGlobalSlots);
    uint32_t* slot_rank = lc.gfirst + kLcGlobalSlots;
    lc.overflow = reinterpret_cast<int32_t*>(slot_rank + kLcGlobalSlots);
    lc.gused = reinterpret_cast<uint32_t*>(lc.overflow + 1);
    int64_t* d_ng = reinterpret_cast<int64_t*>(lc.overflow + 2);
    NFC_CUDA(cudaMemsetAsync(lcb, 0, lc_bytes, s));
    NFC_CUDA(cudaMemsetAsync(lc.gfirst, 0xFF, kLcGlobalSlots * sizeof(uint32_t), s));
    const int64_t nchunks = (n + 127) / 128;
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nchunks + 15) / 16, (int64_t)num_sms() * 3));
    const int lc_smem = kLcSlots * 16;
    NFC_CUDA(cudaFuncSetAttribute(k_unique_lowcard, cudaFuncAttributeMaxDynamicSharedMemorySize, lc_smem));
    k_unique_lowcard<<<g, 512, lc_smem, s>>>(keys, n, lc);
    NFC_CUDA(cudaGetLastError());
    int32_t over = 0;
    NFC_CUDA(cudaMemcpyAsync(&over, lc.overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    NFC_CUDA(cudaStreamSynchronize(s));
    if (!over) {
      k_unique_lowcard_emit<<<1, 1024, 0, s>>>(lc, uniq_out, first_out, counts_out, slot_rank, d_ng);
      NFC_CUDA(cudaGetLastError());
      if (inv_out) {
        k_unique_lowcard_inverse<<<grid1d(n), 256, 0, s>>>(keys, n, lc, slot_rank, inv_out);
        NFC_CUDA(cudaGetLastError());
      }
      int64_t ng = 0;
      NFC_CUDA(cudaMemcpyAsync(&ng, d_ng, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      const int st = read_status(s, d_err);
      if (st) return st;
      return ng;
    }
  }
  uint32_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr, *kres = nullptr, *vres = nullptr;
  NFC_CUDA(sc.alloc(&k0, (size_t)n));
  NFC_CUDA(sc.alloc(&k1, (size_t)n));
  NFC_CUDA(sc.alloc(&v0, (size_t)n));
  NFC_CUDA(sc.alloc(&v1, (size_t)n));
  // int32 keys sort as unsigned after a sign flip, applied as the keys are read.
  int rc = radix_sort_u32_from(reinterpret_cast<const uint32_t*>(keys), 0x80000000u, k0, k1, v0, v1, n, 32, true, s,
                               sc, d_err, &kres, &vres);
  if (rc) return rc;
  const int64_t ntiles = (n + kRunTile - 1) / kRunTile;
  uint64_t* lb = nullptr;
  uint32_t* run_start = nullptr;
  int64_t* tile_q = nullptr;
  uint32_t* tile_start = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 2));
  NFC_CUDA(sc.alloc(&run_start, (size_t)n));
  NFC_CUDA(sc.alloc(&tile_q, (size_t)ntiles));
  NFC_CUDA(sc.alloc(&tile_start, (size_t)ntiles));
  int64_t* d_ng = reinterpret_cast<int64_t*>(lb + ntiles);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles + 1);
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 2), s));
  k_runs<<<(unsigned)ntiles, 256, 0, s>>>(kres, vres, n, uniq_out, first_out, counts_out, run_start, tile_q,
                                          tile_start, inv_out, lb, ticket, d_ng, d_err);
  NFC_CUDA(cudaGetLastError());
  k_run_fix<<<(unsigned)((ntiles + 255) / 256), 256, 0, s>>>(tile_q, tile_start, run_start, d_ng, n, ntiles,
                                                              counts_out);
  NFC_CUDA(cudaGetLastError());
  int64_t ng = 0;
  NFC_CUDA(cudaMemcpyAsync(&ng, d_ng, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  const int st = read_status(s, d_err);
  if (st) return st;
  return ng;
}
