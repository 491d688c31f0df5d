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
//   2. range of the flipped halves, then word = (ta - ta_min) << wb |
//      (tb - tb_min) with ta = a ^ a_flip, tb = b ^ b_flip and wb the bit
//      width of tb's range: the pair's order in just the bits it needs;
//   3. onesweep radix sort of (word, position index) over those bits;
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

// Range of the flipped halves over the rows to pack: mm[0] = max(~ta) (so
// ~mm[0] is the minimum), mm[1] = max(ta), mm[2] = max(~tb), mm[3] = max(tb);
// zero-initialised.
__global__ void k_cc_range(const int32_t* __restrict__ a, uint32_t a_flip, const int32_t* __restrict__ b,
                           uint32_t b_flip, const uint32_t* __restrict__ pos, int64_t nv, uint32_t* mm) {
  uint32_t x0 = 0, x1 = 0, x2 = 0, x3 = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = pos ? (int64_t)pos[i] : i;
    const uint32_t ta = (uint32_t)a[r] ^ a_flip, tb = (uint32_t)b[r] ^ b_flip;
    x0 = max(x0, ~ta);
    x1 = max(x1, ta);
    x2 = max(x2, ~tb);
    x3 = max(x3, tb);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x0 = max(x0, __shfl_xor_sync(0xffffffffu, x0, o));
    x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, o));
    x2 = max(x2, __shfl_xor_sync(0xffffffffu, x2, o));
    x3 = max(x3, __shfl_xor_sync(0xffffffffu, x3, o));
  }
  if (lane_id() == 0) {
    atomicMax(&mm[0], x0);
    atomicMax(&mm[1], x1);
    atomicMax(&mm[2], x2);
    atomicMax(&mm[3], x3);
  }
}

// word = (ta - ta_min) << wb | (tb - tb_min): the same order as the flipped
// pair, in wa + wb bits, so the radix sort runs only the passes it needs.
__global__ void k_cc_pack(const int32_t* __restrict__ a, uint32_t a_flip, uint32_t a_min, const int32_t* __restrict__ b,
                          uint32_t b_flip, uint32_t b_min, int wb, const uint32_t* __restrict__ pos, int64_t nv,
                          uint64_t* __restrict__ words) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = pos ? (int64_t)pos[i] : i;
    words[i] = ((uint64_t)(((uint32_t)a[r] ^ a_flip) - a_min) << wb) | (uint64_t)(((uint32_t)b[r] ^ b_flip) - b_min);
  }
}

__global__ void __launch_bounds__(kCcThreads) k_cc_runs(const uint64_t* __restrict__ sw, const uint32_t* __restrict__ idx,
                                                        const uint32_t* __restrict__ pos, int64_t nv, uint32_t a_flip,
                                                        uint32_t a_min, uint32_t b_flip, uint32_t b_min, int wb,
                                                        int32_t* __restrict__ codes,
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
  if (i0 + kCcPer <= nv) {
#pragma unroll
    for (int q = 0; q < kCcPer / 2; ++q) {
      const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(sw + i0 + 2 * q);
      w[2 * q] = v.x;
      w[2 * q + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kCcPer; ++j) w[j] = i0 + j < nv ? sw[i0 + j] : 0ull;
  }
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
  if (threadIdx.x < 32) {
    const int64_t lbx = lookback_exclusive(lb, tile, total, err);  // whole warp
    if (threadIdx.x == 0) {
      s_base = lbx;
      if (tile == ntiles - 1) *ng_out = s_base + total;
    }
  }
  __syncthreads();
  int64_t r = s_base + ex - 1;
#pragma unroll
  for (int j = 0; j < kCcPer; ++j) {
    const int64_t i = i0 + j;
    if (i >= nv) break;
    if (heads & (1u << j)) {
      ++r;
      const uint64_t bmask = wb >= 64 ? ~0ull : ((1ull << wb) - 1ull);
      ua[r] = (int32_t)(((uint32_t)(w[j] >> wb) + a_min) ^ a_flip);
      ub[r] = (int32_t)(((uint32_t)(w[j] & bmask) + b_min) ^ b_flip);
    }
    const uint32_t k = idx[i];
    codes[pos ? pos[k] : k] = (int32_t)r;
  }
}

unsigned cc_grid(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8));
}

// ---- bit-packed tuple keys -------------------------------------------------
// A tuple key whose columns' flipped ranges fit in 31 bits together becomes
// one non-negative int32: the columns' (t - t_min) side by side, the most
// significant first.  Its integer order is the tuple's order, so the dense
// and partition group-bys take it directly -- no sort, no per-row codes.

struct KeyBits {
  const int32_t* col[NFC_MAX_KEY_COLS];
  uint32_t flip[NFC_MAX_KEY_COLS];
  uint32_t kmin[NFC_MAX_KEY_COLS];
  uint32_t shift[NFC_MAX_KEY_COLS];
  uint32_t mask[NFC_MAX_KEY_COLS];
  int ncols;
  bool vec;  // every column 16-byte aligned: four rows per 16-byte load
};

NFC_DEV int4 kb_load4(const KeyBits& kb, int c, int64_t q) {
  return __ldcs(reinterpret_cast<const int4*>(kb.col[c]) + q);
}

// mm[2c] = max(~t_c), mm[2c + 1] = max(t_c) over valid rows (zero-initialised);
// mm[2 * NFC_MAX_KEY_COLS] counts the valid rows.
__global__ void __launch_bounds__(256) k_kb_range(KeyBits kb, const uint8_t* __restrict__ validity, int64_t n,
                                                  uint32_t* __restrict__ mm) {
  uint32_t lo[NFC_MAX_KEY_COLS], hi[NFC_MAX_KEY_COLS];
#pragma unroll
  for (int c = 0; c < NFC_MAX_KEY_COLS; ++c) lo[c] = hi[c] = 0u;
  uint32_t cnt = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t done = 0;
  if (kb.vec) {
    // Rows 4q .. 4q+3: one 16-byte load per column, the nibble (q & 1) of
    // validity byte q >> 1.
    const int64_t nq = n / 4;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq; q += stride) {
      const uint32_t ok = validity ? (uint32_t)(validity[q >> 1] >> ((q & 1) * 4)) & 0xFu : 0xFu;
      cnt += __popc(ok);
#pragma unroll
      for (int c = 0; c < NFC_MAX_KEY_COLS; ++c) {
        if (c < kb.ncols) {
          const int4 v = kb_load4(kb, c, q);
          const int32_t e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int r = 0; r < 4; ++r)
            if ((ok >> r) & 1u) {
              const uint32_t t = (uint32_t)e[r] ^ kb.flip[c];
              lo[c] = max(lo[c], ~t);
              hi[c] = max(hi[c], t);
            }
        }
      }
    }
    done = nq * 4;
  }
  for (int64_t i = done + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    if (validity && !((validity[i >> 3] >> (i & 7)) & 1u)) continue;
    ++cnt;
#pragma unroll
    for (int c = 0; c < NFC_MAX_KEY_COLS; ++c) {
      if (c >= kb.ncols) break;
      const uint32_t t = (uint32_t)kb.col[c][i] ^ kb.flip[c];
      lo[c] = max(lo[c], ~t);
      hi[c] = max(hi[c], t);
    }
  }
  cnt = warp_sum(cnt);
#pragma unroll
  for (int c = 0; c < NFC_MAX_KEY_COLS; ++c) {
    if (c >= kb.ncols) break;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[c] = max(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = max(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
  }
  if (lane_id() == 0) {
#pragma unroll
    for (int c = 0; c < NFC_MAX_KEY_COLS; ++c)
      if (c < kb.ncols) {
        atomicMax(&mm[2 * c], lo[c]);
        atomicMax(&mm[2 * c + 1], hi[c]);
      }
    if (cnt) atomicAdd(&mm[2 * NFC_MAX_KEY_COLS], cnt);
  }
}

__global__ void __launch_bounds__(256) k_kb_pack(KeyBits kb, int64_t n, int32_t* __restrict__ codes) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t done = 0;
  if (kb.vec && (reinterpret_cast<uintptr_t>(codes) & 15u) == 0) {
    const int64_t nq = n / 4;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq; q += stride) {
      uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int c = 0; c < NFC_MAX_KEY_COLS; ++c) {
        if (c >= kb.ncols) break;
        const int4 v = kb_load4(kb, c, q);
        const int32_t e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int r = 0; r < 4; ++r) w[r] |= ((((uint32_t)e[r] ^ kb.flip[c]) - kb.kmin[c]) & kb.mask[c]) << kb.shift[c];
      }
      reinterpret_cast<int4*>(codes)[q] = make_int4((int32_t)w[0], (int32_t)w[1], (int32_t)w[2], (int32_t)w[3]);
    }
    done = nq * 4;
  }
  for (int64_t i = done + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t w = 0;
#pragma unroll
    for (int c = 0; c < NFC_MAX_KEY_COLS; ++c) {
      if (c >= kb.ncols) break;
      w |= ((((uint32_t)kb.col[c][i] ^ kb.flip[c]) - kb.kmin[c]) & kb.mask[c]) << kb.shift[c];
    }
    codes[i] = (int32_t)w;
  }
}

struct KeyOut {
  int32_t* col[NFC_MAX_KEY_COLS];
};

__global__ void __launch_bounds__(256) k_kb_unpack(KeyBits kb, const int64_t* __restrict__ codes, int64_t ng,
                                                   KeyOut out) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = (uint32_t)codes[g];
#pragma unroll
    for (int c = 0; c < NFC_MAX_KEY_COLS; ++c) {
      if (c >= kb.ncols) break;
      out.col[c][g] = (int32_t)((((w >> kb.shift[c]) & kb.mask[c]) + kb.kmin[c]) ^ kb.flip[c]);
    }
  }
}

int fill_keybits(const int32_t* const* cols, const uint32_t* flips, const uint32_t* mins, const int32_t* widths,
                 int ncols, KeyBits* kb) {
  if (ncols < 1 || ncols > NFC_MAX_KEY_COLS || !flips) return NFC_ERR_MALFORMED;
  *kb = KeyBits{};
  kb->ncols = ncols;
  int total = 0;
  for (int c = ncols - 1; c >= 0; --c) {
    if (flips[c] != 0u && flips[c] != 0x80000000u) return NFC_ERR_MALFORMED;
    kb->col[c] = cols ? cols[c] : nullptr;
    kb->flip[c] = flips[c];
    if (widths) {
      if (widths[c] < 0 || widths[c] > 31) return NFC_ERR_MALFORMED;
      kb->kmin[c] = mins ? mins[c] : 0u;
      kb->shift[c] = (uint32_t)total;
      kb->mask[c] = widths[c] ? ((1u << widths[c]) - 1u) : 0u;
      total += widths[c];
    }
  }
  if (total > 31) return NFC_ERR_RANGE;
  kb->vec = true;
  for (int c = 0; c < ncols; ++c)
    if (reinterpret_cast<uintptr_t>(kb->col[c]) & 15u) kb->vec = false;
  return NFC_OK;
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
  uint32_t* mm = nullptr;
  NFC_CUDA(sc.alloc(&mm, 4));
  NFC_CUDA(cudaMemsetAsync(mm, 0, 4 * sizeof(uint32_t), s));
  k_cc_range<<<cc_grid(nv), 256, 0, s>>>(a, a_flip, b, b_flip, pos, nv, mm);
  NFC_CUDA(cudaGetLastError());
  uint32_t hm[4];
  NFC_CUDA(cudaMemcpyAsync(hm, mm, sizeof(hm), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  const uint32_t a_min = ~hm[0], b_min = ~hm[2];
  auto bitlen = [](uint32_t x) { int b = 0; while (x) { ++b; x >>= 1; } return b; };
  const int wa = bitlen(hm[1] - a_min), wb = bitlen(hm[3] - b_min);
  k_cc_pack<<<cc_grid(nv), 256, 0, s>>>(a, a_flip, a_min, b, b_flip, b_min, wb, pos, nv, w0);
  NFC_CUDA(cudaGetLastError());
  uint64_t* ws = nullptr;
  uint32_t* is = nullptr;
  int rc = radix_sort_u64(w0, w1, i0, i1, nv, std::max(1, wa + wb), true, s, sc, d_err, &ws, &is);
  if (rc) return rc;
  const int64_t ntiles = (nv + kCcTile - 1) / kCcTile;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 1));
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 1), s));
  k_cc_runs<<<(unsigned)ntiles, kCcThreads, 0, s>>>(ws, is, pos, nv, a_flip, a_min, b_flip, b_min, wb, codes_out,
                                                   ua_out, ub_out, lb,
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

extern "C" int64_t nfc_key_ranges(const int32_t* const* cols, const uint32_t* flips, int ncols,
                                  const uint8_t* validity, int64_t n, uint32_t* min_out, uint32_t* max_out,
                                  void* stream) {
  if (n < 0 || !cols || !min_out || !max_out) return n < 0 ? NFC_ERR_MALFORMED : NFC_ERR_NULL;
  KeyBits kb;
  int rc = fill_keybits(cols, flips, nullptr, nullptr, ncols, &kb);
  if (rc) return rc;
  for (int c = 0; c < ncols; ++c) {
    min_out[c] = 0xFFFFFFFFu;
    max_out[c] = 0u;
    if (n && !cols[c]) return NFC_ERR_NULL;
  }
  if (n == 0) return 0;
  if (n >= (1ll << 32)) return NFC_ERR_UNSUPPORTED;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  uint32_t* mm = nullptr;
  const int nw = 2 * NFC_MAX_KEY_COLS + 1;
  NFC_CUDA(sc.alloc(&mm, nw));
  NFC_CUDA(cudaMemsetAsync(mm, 0, nw * sizeof(uint32_t), s));
  k_kb_range<<<cc_grid(n), 256, 0, s>>>(kb, validity, n, mm);
  NFC_CUDA(cudaGetLastError());
  uint32_t h[2 * NFC_MAX_KEY_COLS + 1];
  NFC_CUDA(cudaMemcpyAsync(h, mm, sizeof(h), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  const uint32_t nvalid = h[2 * NFC_MAX_KEY_COLS];
  if (nvalid == 0) return 0;
  for (int c = 0; c < ncols; ++c) {
    min_out[c] = ~h[2 * c];
    max_out[c] = h[2 * c + 1];
  }
  return (int64_t)nvalid;
}

extern "C" int nfc_pack_key_bits(const int32_t* const* cols, const uint32_t* flips, const uint32_t* mins,
                                 const int32_t* widths, int ncols, int64_t n, int32_t* codes_out, void* stream) {
  if (n < 0) return NFC_ERR_MALFORMED;
  if (!cols || !mins || !widths) return NFC_ERR_NULL;
  KeyBits kb;
  int rc = fill_keybits(cols, flips, mins, widths, ncols, &kb);
  if (rc) return rc;
  if (n == 0) return NFC_OK;
  if (!codes_out) return NFC_ERR_NULL;
  for (int c = 0; c < ncols; ++c)
    if (!cols[c]) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_kb_pack<<<cc_grid(n), 256, 0, s>>>(kb, n, codes_out);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

extern "C" int nfc_unpack_key_bits(const int64_t* codes, int64_t ng, const uint32_t* flips, const uint32_t* mins,
                                   const int32_t* widths, int ncols, int32_t* const* cols_out, void* stream) {
  if (ng < 0) return NFC_ERR_MALFORMED;
  if (!mins || !widths || !cols_out) return NFC_ERR_NULL;
  KeyBits kb;
  int rc = fill_keybits(nullptr, flips, mins, widths, ncols, &kb);
  if (rc) return rc;
  if (ng == 0) return NFC_OK;
  if (!codes) return NFC_ERR_NULL;
  KeyOut ko{};
  for (int c = 0; c < ncols; ++c) {
    if (!cols_out[c]) return NFC_ERR_NULL;
    ko.col[c] = cols_out[c];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_kb_unpack<<<cc_grid(ng), 256, 0, s>>>(kb, codes, ng, ko);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}
