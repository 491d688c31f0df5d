// Composite group keys: dense int32 codes for pairs of int32 key columns.
//
// The reference groups tuple keys with composite_tuple_index
// (src/Drivers/CPU/_lib/groupindex.py:520-639): two int32 columns are packed
// as (a << 32) | (b & 0xFFFFFFFF) and sorted as int64, i.e. by a (signed)
// then b (unsigned); three columns sort by the third, then that pair; four
// by the packed first pair, then the packed second pair.  One pairwise fold
// reproduces each of these orders: codes of (a, b) are the ranks of the
// distinct pairs in that order, and a code (non-negative) is itself a
// column for the next fold.
//
// nfc_composite_codes(a, a_flip, b, b_flip, ...): the order of a column is
// its bits XOR the flip word (0x80000000 = signed order, 0 = unsigned).
//   1. positions of the rows valid in the bitmap (all rows without one);
//   2. word = ((a ^ a_flip) << 32) | (b ^ b_flip) per valid row;
//   3. onesweep radix sort of (word, position index);
//   4. k_cc_runs: run heads of equal words, run ids by a block scan and a
//      decoupled look-back; codes[row] = run id, and each head writes its
//      pair (ua, ub) at the run id.  Rows not valid keep code -1.
#include <algorithm>

#include "groupby_host.h"

namespace nfc {
namespace {

constexpr int kCcThreads = 256;
constexpr int kCcPer = 16;
constexpr int kCcTile = kCcThreads * kCcPer;

__global__ void k_cc_pack(const int32_t* __restrict__ a, uint32_t a_flip, const int32_t* __restrict__ b,
                          uint32_t b_flip, const uint32_t* __restrict__ pos, int64_t nv, uint64_t* __restrict__ words) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = pos ? (int64_t)pos[i] : i;
    words[i] = ((uint64_t)((uint32_t)a[r] ^ a_flip) << 32) | ((uint32_t)b[r] ^ b_flip);
  }
}

__global__ void __launch_bounds__(kCcThreads) k_cc_runs(const uint64_t* __restrict__ sw, const uint32_t* __restrict__ idx,
                                                        const uint32_t* __restrict__ pos, int64_t nv, uint32_t a_flip,
                                                        uint32_t b_flip, int32_t* __restrict__ codes,
                                                        int32_t* __restrict__ ua, int32_t* __restrict__ ub,
                                                        uint64_t* lb, uint32_t* ticket, int64_t* ng_out, int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t ntiles = (nv + kCcTile - 1) / kCcTile;
  if (tile >= ntiles) return;
  const int64_t i0 = tile * kCcTile + (int64_t)threadIdx.x * kCcPer;
  uint64_t w[kCcPer];
#pragma unroll
  for (int j = 0; j < kCcPer; ++j) w[j] = i0 + j < nv ? sw[i0 + j] : 0ull;
  const uint64_t prev = (i0 > 0 && i0 < nv) ? sw[i0 - 1] : 0ull;
  uint32_t heads = 0, c = 0;
#pragma unroll
  for (int j = 0; j < kCcPer; ++j) {
    const int64_t i = i0 + j;
    if (i >= nv) break;
    if (i == 0 || (j == 0 ? prev : w[j - 1]) != w[j]) {
      heads |= 1u << j;
      ++c;
    }
  }
  uint32_t total;
  const uint32_t ex = block_excl_scan(c, s_scan, &total);
  if (threadIdx.x == 0) {
    s_base = lookback_exclusive(lb, tile, total, err);
    if (tile == ntiles - 1) *ng_out = s_base + total;
  }
  __syncthreads();
  int64_t r = s_base + ex - 1;
#pragma unroll
  for (int j = 0; j < kCcPer; ++j) {
    const int64_t i = i0 + j;
    if (i >= nv) break;
    if (heads & (1u << j)) {
      ++r;
      ua[r] = (int32_t)((uint32_t)(w[j] >> 32) ^ a_flip);
      ub[r] = (int32_t)((uint32_t)w[j] ^ b_flip);
    }
    const uint32_t k = idx[i];
    codes[pos ? pos[k] : k] = (int32_t)r;
  }
}

unsigned cc_grid(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8));
}

}  // namespace
}  // namespace nfc

using namespace nfc;

extern "C" int64_t nfc_composite_codes(const int32_t* a, uint32_t a_flip, const int32_t* b, uint32_t b_flip,
                                       const uint8_t* validity, int64_t n, int32_t* codes_out, int32_t* ua_out,
                                       int32_t* ub_out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if ((a_flip != 0u && a_flip != 0x80000000u) || (b_flip != 0u && b_flip != 0x80000000u)) return NFC_ERR_MALFORMED;
  if (n == 0) return 0;
  if (!a || !b || !codes_out || !ua_out || !ub_out) return NFC_ERR_NULL;
  if (n >= (1ll << 30)) {
    set_last_error("composite_codes: n=%lld >= 2^30", (long long)n);
    return NFC_ERR_UNSUPPORTED;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  int64_t* small = nullptr;  // nv | ng | err
  NFC_CUDA(sc.alloc(&small, 3));
  NFC_CUDA(cudaMemsetAsync(small, 0, 3 * sizeof(int64_t), s));
  int32_t* d_err = reinterpret_cast<int32_t*>(small + 2);
  NFC_CUDA(cudaMemsetAsync(codes_out, 0xFF, sizeof(int32_t) * n, s));
  uint32_t* pos = nullptr;
  int64_t nv = n;
  if (validity) {
    NFC_CUDA(sc.alloc(&pos, (size_t)n));
    int rc = valid_positions(validity, n, pos, &nv, s, sc, d_err);
    if (rc) return rc;
    if (nv == 0) return 0;
  }
  uint64_t *w0 = nullptr, *w1 = nullptr;
  uint32_t *i0 = nullptr, *i1 = nullptr;
  NFC_CUDA(sc.alloc(&w0, (size_t)nv));
  NFC_CUDA(sc.alloc(&w1, (size_t)nv));
  NFC_CUDA(sc.alloc(&i0, (size_t)nv));
  NFC_CUDA(sc.alloc(&i1, (size_t)nv));
  k_cc_pack<<<cc_grid(nv), 256, 0, s>>>(a, a_flip, b, b_flip, pos, nv, w0);
  NFC_CUDA(cudaGetLastError());
  uint64_t* ws = nullptr;
  uint32_t* is = nullptr;
  int rc = radix_sort_u64(w0, w1, i0, i1, nv, 64, true, s, sc, d_err, &ws, &is);
  if (rc) return rc;
  const int64_t ntiles = (nv + kCcTile - 1) / kCcTile;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 1));
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 1), s));
  k_cc_runs<<<(unsigned)ntiles, kCcThreads, 0, s>>>(ws, is, pos, nv, a_flip, b_flip, codes_out, ua_out, ub_out, lb,
                                                   reinterpret_cast<uint32_t*>(lb + ntiles), small + 1, d_err);
  NFC_CUDA(cudaGetLastError());
  int64_t h[3] = {0, 0, 0};
  NFC_CUDA(cudaMemcpyAsync(h, small, sizeof(h), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if ((int32_t)h[2]) {
    set_last_error("composite_codes: device status %d", (int)(int32_t)h[2]);
    return (int32_t)h[2];
  }
  return h[1];
}
