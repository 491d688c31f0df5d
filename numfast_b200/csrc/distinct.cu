// Grouped COUNT DISTINCT: per int32 key, the number of distinct int32 values
// among the rows whose key and value are both valid.
//
// Reference: the executor's group_count_distinct (src/Drivers/CPU/_lib/
// cpu.py:3705-3768): valid-mask, compact, sort by (key, value), one scan of
// group bounds and value transitions (_count_distinct_sorted_dedup,
// cpu.py:2647-2700); output ukeys ascending and nunique, both int64.
//
// Here:
//   1. k_cd_range: count of valid rows and the range of tk = key ^ 2^31 and
//      tv = value ^ 2^31 over them; k_cd_pack: pair = (tk - tk_min) << wv |
//      (tv - tv_min), wv the bit width of tv's range, an unsigned order equal
//      to (key, value) order in wk + wv bits; invalid rows get the all-ones
//      word of that width, so after the sort the first n_valid entries are
//      exactly the valid pairs (an all-ones valid pair is identical to the
//      filler and indistinguishable from it, so dropping n - n_valid of them
//      keeps the right multiset);
//   2. onesweep radix sort of the pairs over wk + wv bits (radix.cu; passes
//      whose digit is the same for every pair are skipped);
//   3. k_cd_runs: 4096 sorted pairs per tile; a key head is a change of the
//      high half, a pair head any change; one decoupled look-back carries
//      both counts (key heads << 31 | pair heads), so key run r learns its
//      output slot and the number of pair heads before it;
//   4. k_cd_counts: nunique[r] = pair heads before run r+1 - before run r.
#include <algorithm>

#include "groupby_host.h"

namespace nfc {
namespace {

constexpr int kCdThreads = 256;
constexpr int kCdPer = 16;
constexpr int kCdTile = kCdThreads * kCdPer;
constexpr uint64_t kCdPairBits = 31;

NFC_DEV bool cd_valid(const uint8_t* bm, int64_t i) { return !bm || ((bm[i >> 3] >> (i & 7)) & 1u); }

// Range of the flipped halves over the valid rows and their number:
// mm[0] = max(~tk), mm[1] = max(tk), mm[2] = max(~tv), mm[3] = max(tv)
// (zero-initialised; ~mm[0] and ~mm[2] are the minima).
__global__ void __launch_bounds__(256) k_cd_range(const int32_t* __restrict__ keys, const uint8_t* __restrict__ kv,
                                                  const int32_t* __restrict__ vals, const uint8_t* __restrict__ vv,
                                                  int64_t n, uint32_t* __restrict__ mm,
                                                  unsigned long long* __restrict__ nvalid) {
  uint32_t x0 = 0, x1 = 0, x2 = 0, x3 = 0, c = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t done = 0;
  if (((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals)) & 15u) == 0) {
    // Four rows per 16-byte load, U loads of each column in flight; rows
    // 4q .. 4q+3 take the nibble (q & 1) of bitmap byte q >> 1.
    constexpr int U = 4;
    const int64_t nq = n / 4;
    for (int64_t q0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q0 < nq; q0 += stride * U) {
      int4 kk[U], vq[U];
      uint32_t ok[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t q = q0 + u * stride;
        ok[u] = 0u;
        if (q < nq) {
          kk[u] = __ldcs(reinterpret_cast<const int4*>(keys) + q);
          vq[u] = __ldcs(reinterpret_cast<const int4*>(vals) + q);
          const uint32_t sh = (uint32_t)(q & 1) * 4u;
          ok[u] = (kv ? (uint32_t)(kv[q >> 1] >> sh) : 0xFu) & (vv ? (uint32_t)(vv[q >> 1] >> sh) : 0xFu) & 0xFu;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t ks[4] = {kk[u].x, kk[u].y, kk[u].z, kk[u].w};
        const int32_t vs[4] = {vq[u].x, vq[u].y, vq[u].z, vq[u].w};
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if ((ok[u] >> r) & 1u) {
            const uint32_t tk = (uint32_t)ks[r] ^ 0x80000000u, tv = (uint32_t)vs[r] ^ 0x80000000u;
            x0 = max(x0, ~tk);
            x1 = max(x1, tk);
            x2 = max(x2, ~tv);
            x3 = max(x3, tv);
            ++c;
          }
      }
    }
    done = nq * 4;
  }
  for (int64_t i = done + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    if (!(cd_valid(kv, i) && cd_valid(vv, i))) continue;
    const uint32_t tk = (uint32_t)keys[i] ^ 0x80000000u, tv = (uint32_t)vals[i] ^ 0x80000000u;
    x0 = max(x0, ~tk);
    x1 = max(x1, tk);
    x2 = max(x2, ~tv);
    x3 = max(x3, tv);
    ++c;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x0 = max(x0, __shfl_xor_sync(0xffffffffu, x0, o));
    x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, o));
    x2 = max(x2, __shfl_xor_sync(0xffffffffu, x2, o));
    x3 = max(x3, __shfl_xor_sync(0xffffffffu, x3, o));
  }
  c = warp_sum(c);
  if (lane_id() == 0) {
    atomicMax(&mm[0], x0);
    atomicMax(&mm[1], x1);
    atomicMax(&mm[2], x2);
    atomicMax(&mm[3], x3);
    if (c) atomicAdd(nvalid, (unsigned long long)c);
  }
}

// pair = (tk - tk_min) << wv | (tv - tv_min) in wk + wv bits; invalid rows get
// the largest word of that width (the filler).
__global__ void __launch_bounds__(256) k_cd_pack(const int32_t* __restrict__ keys, const uint8_t* __restrict__ kv,
                                                 const int32_t* __restrict__ vals, const uint8_t* __restrict__ vv,
                                                 int64_t n, uint32_t kmin, uint32_t vmin, int wv, uint64_t filler,
                                                 uint64_t* __restrict__ pairs) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool ok = cd_valid(kv, i) && cd_valid(vv, i);
    pairs[i] = ok ? (((uint64_t)(((uint32_t)keys[i] ^ 0x80000000u) - kmin) << wv) |
                     (uint64_t)(((uint32_t)vals[i] ^ 0x80000000u) - vmin))
                  : filler;
  }
}

__global__ void __launch_bounds__(kCdThreads) k_cd_runs(const uint64_t* __restrict__ sp, int64_t nv, int wv,
                                                        uint32_t kmin,
                                                        int64_t* __restrict__ ukeys, int64_t* __restrict__ pstart,
                                                        uint64_t* lb, uint32_t* ticket, int64_t* ng_out,
                                                        int64_t* pairs_out, int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_kbase, s_pbase;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t ntiles = (nv + kCdTile - 1) / kCdTile;
  if (tile >= ntiles) return;
  const int64_t i0 = tile * kCdTile + (int64_t)threadIdx.x * kCdPer;
  uint64_t w[kCdPer];
  if (i0 + kCdPer <= nv) {
#pragma unroll
    for (int q = 0; q < kCdPer / 2; ++q) {
      const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(sp + i0 + 2 * q);
      w[2 * q] = v.x;
      w[2 * q + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kCdPer; ++j) w[j] = i0 + j < nv ? sp[i0 + j] : 0ull;
  }
  const uint64_t prev = (i0 > 0 && i0 < nv) ? sp[i0 - 1] : 0ull;
  uint32_t kh = 0, ph = 0, kc = 0, pc = 0;
#pragma unroll
  for (int j = 0; j < kCdPer; ++j) {
    const int64_t i = i0 + j;
    if (i >= nv) break;
    const uint64_t p = j == 0 ? prev : w[j - 1];
    const bool first = i == 0;
    if (first || (p >> wv) != (w[j] >> wv)) { kh |= 1u << j; ++kc; }
    if (first || p != w[j]) { ph |= 1u << j; ++pc; }
  }
  // Exclusive scans of both counts in one u32 each (a tile holds < 2^16 of each).
  uint32_t tot;
  const uint32_t ex = block_excl_scan((kc << 16) | pc, s_scan, &tot);
  const uint32_t tk = tot >> 16, tp = tot & 0xFFFFu;
  if (threadIdx.x < 32) {
    const uint64_t agg = ((uint64_t)tk << kCdPairBits) | tp;
    const int64_t lbx = lookback_exclusive(lb, tile, agg, err);  // whole warp
    if (threadIdx.x == 0) {
      const uint64_t e = (uint64_t)lbx;
      s_kbase = (int64_t)(e >> kCdPairBits);
      s_pbase = (int64_t)(e & ((1ull << kCdPairBits) - 1));
      if (tile == ntiles - 1) {
        *ng_out = s_kbase + tk;
        *pairs_out = s_pbase + tp;
      }
    }
  }
  __syncthreads();
  int64_t r = s_kbase + (ex >> 16) - 1;  // run of the element before this thread's first head
  int64_t q = s_pbase + (ex & 0xFFFFu);   // pair heads before this thread's first element
#pragma unroll
  for (int j = 0; j < kCdPer; ++j) {
    const int64_t i = i0 + j;
    if (i >= nv) break;
    if (kh & (1u << j)) {
      ++r;
      ukeys[r] = (int64_t)(int32_t)(((uint32_t)(w[j] >> wv) + kmin) ^ 0x80000000u);
      pstart[r] = q;
    }
    if (ph & (1u << j)) ++q;
  }
}

__global__ void k_cd_counts(const int64_t* __restrict__ pstart, const int64_t* ng_ptr, const int64_t* pairs_ptr,
                            int64_t* __restrict__ nunique) {
  const int64_t ng = *ng_ptr, total = *pairs_ptr;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < ng; r += (int64_t)gridDim.x * blockDim.x)
    nunique[r] = (r + 1 < ng ? pstart[r + 1] : total) - pstart[r];
}

unsigned cd_grid(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8));
}

}  // namespace
}  // namespace nfc

using namespace nfc;

extern "C" int64_t nfc_group_count_distinct(const int32_t* keys, const uint8_t* key_validity, const int32_t* values,
                                            const uint8_t* value_validity, int64_t n, int64_t out_cap,
                                            int64_t* ukeys_out, int64_t* nunique_out, void* stream) {
  if (n < 0 || out_cap < 0) return NFC_ERR_MALFORMED;
  if (n == 0) return 0;
  if (!keys || !values || !ukeys_out || !nunique_out) return NFC_ERR_NULL;
  if (n >= (1ll << 30)) {
    set_last_error("group_count_distinct: n=%lld >= 2^30", (long long)n);
    return NFC_ERR_UNSUPPORTED;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  uint64_t *p0 = nullptr, *p1 = nullptr;
  int64_t* small = nullptr;  // nvalid | ng | pairs | err
  NFC_CUDA(sc.alloc(&p0, (size_t)n));
  NFC_CUDA(sc.alloc(&p1, (size_t)n));
  NFC_CUDA(sc.alloc(&small, 4));
  NFC_CUDA(cudaMemsetAsync(small, 0, 4 * sizeof(int64_t), s));
  int32_t* d_err = reinterpret_cast<int32_t*>(small + 3);
  uint32_t* mm = nullptr;
  NFC_CUDA(sc.alloc(&mm, 4));
  NFC_CUDA(cudaMemsetAsync(mm, 0, 4 * sizeof(uint32_t), s));
  k_cd_range<<<cd_grid(n), 256, 0, s>>>(keys, key_validity, values, value_validity, n, mm,
                                       reinterpret_cast<unsigned long long*>(small));
  NFC_CUDA(cudaGetLastError());
  struct {
    uint32_t mm[4];
    int64_t nv;
  } hr;
  NFC_CUDA(cudaMemcpyAsync(hr.mm, mm, sizeof(hr.mm), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaMemcpyAsync(&hr.nv, small, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  const int64_t nv = hr.nv;
  if (nv == 0) return 0;
  auto bitlen = [](uint32_t x) { int b = 0; while (x) { ++b; x >>= 1; } return b; };
  const uint32_t kmin = ~hr.mm[0], vmin = ~hr.mm[2];
  const int wk = bitlen(hr.mm[1] - kmin), wv = bitlen(hr.mm[3] - vmin);
  const int bits = std::max(1, wk + wv);
  const uint64_t filler = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
  k_cd_pack<<<cd_grid(n), 256, 0, s>>>(keys, key_validity, values, value_validity, n, kmin, vmin, wv, filler, p0);
  NFC_CUDA(cudaGetLastError());
  uint64_t* sorted = nullptr;
  uint32_t* unused = nullptr;
  int rc = radix_sort_u64(p0, p1, nullptr, nullptr, n, bits, false, s, sc, d_err, &sorted, &unused);
  if (rc) return rc;
  const int64_t ntiles = (nv + kCdTile - 1) / kCdTile;
  uint64_t* lb = nullptr;
  int64_t* pstart = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 1));
  NFC_CUDA(sc.alloc(&pstart, (size_t)nv));
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 1), s));
  // ukeys_out needs room for every distinct key: at most nv; the caller's
  // out_cap is checked against the exact count below before anything is
  // written there, so the run kernel first writes into scratch.
  int64_t* ukeys_tmp = nullptr;
  NFC_CUDA(sc.alloc(&ukeys_tmp, (size_t)nv));
  k_cd_runs<<<(unsigned)ntiles, kCdThreads, 0, s>>>(sorted, nv, wv, kmin, ukeys_tmp, pstart, lb,
                                                   reinterpret_cast<uint32_t*>(lb + ntiles), small + 1, small + 2,
                                                   d_err);
  NFC_CUDA(cudaGetLastError());
  int64_t h[4] = {0, 0, 0, 0};
  NFC_CUDA(cudaMemcpyAsync(h, small, sizeof(h), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if ((int32_t)h[3]) {
    set_last_error("group_count_distinct: device status %d", (int)(int32_t)h[3]);
    return (int32_t)h[3];
  }
  const int64_t ng = h[1];
  if (ng > out_cap) {
    set_last_error("group_count_distinct: %lld groups > out_cap %lld", (long long)ng, (long long)out_cap);
    return NFC_ERR_RANGE;
  }
  NFC_CUDA(cudaMemcpyAsync(ukeys_out, ukeys_tmp, sizeof(int64_t) * ng, cudaMemcpyDeviceToDevice, s));
  k_cd_counts<<<cd_grid(ng), 256, 0, s>>>(pstart, small + 1, small + 2, nunique_out);
  NFC_CUDA(cudaGetLastError());
  NFC_CUDA(cudaStreamSynchronize(s));
  return ng;
}
