// Group-by with validity on the device: probe -> plan -> aggregate -> compact.
//
// Replaces the executor's groupby_multi branch (src/Drivers/CPU/_lib/cpu.py:
// 3435-3704) for data resident in HBM:
//   * a row takes part only if its key AND every value column are valid
//     (_valid_mask, cpu.py:1374-1382; test_ops_groupby_quality.py:233-251);
//   * output groups are the distinct valid keys in ascending order with
//     int64 counts, int64 sums for integer columns, float64 sums for float
//     columns, and min/max in the value dtype (ColumnCarry, carry.py:21-115);
//   * a key whose every row is invalid is absent (no NULL group).
//
// Strategies (all give the same integers; float sums within 1e-12 rel):
//   DENSE_SMEM   span M fits one CTA's shared memory: each CTA folds a
//                65,536-row chunk into the whole state on chip and merges it
//                into a global table.
//   DENSE_GLOBAL span fits L2 and the input is small: rows update one global
//                table with atomics.
//   PARTITION    large span (or many rows): rows are scattered into
//                key-range buckets of W keys (one histogram pass, two
//                coalesced scatter passes); one CTA per bucket aggregates on
//                chip and writes its groups straight to their final place
//                (decoupled look-back over buckets).  See partition.cu.
//   HASH         sparse keys: see hash.cu.
//   SORTED       nondecreasing valid keys: runs reduced in one pass, see
//                sorted.cu.
#include <algorithm>
#include <cstring>
#include <vector>

#include "agg_smem.cuh"
#include "groupby_core.cuh"
#include "groupby_host.h"

namespace nfc {

// =====================================================================
// Probe: n_valid, kmin/kmax over valid rows, sortedness of valid keys,
// and the combined validity bitmap (AND of every input bitmap).
// =====================================================================
// A warp span is kProbeChunks chunks of 1024 rows.  In a chunk the warp
// reads the keys with eight coalesced 128-bit loads (group j = rows
// [128j, 128j+128), lane l holding rows 128j + 4l .. 128j + 4l + 3) and the
// bitmaps one 32-bit word per lane (lane l = rows [32l, 32l+32), which is
// also the combined validity word it writes); each group takes its 4-bit
// validity from the word's owner lane by a shuffle.

struct BitmapSet {
  int32_t nbm;
  uint32_t word_aligned;  // bit b: bitmap b is 4-byte aligned
  const uint8_t* bm[NFC_MAX_COLS + 2];  // key, columns, row filter
};

// Validity bits of rows [row0, row0+32) (row0 multiple of 32); only the
// bitmap bytes that cover rows < n are read.
NFC_DEV uint32_t bitmap_word(const uint8_t* bm, bool aligned4, int64_t row0, int64_t rem) {
  const uint8_t* p = bm + (row0 >> 3);
  if (rem >= 32) {
    if (aligned4) return __ldg(reinterpret_cast<const uint32_t*>(p));
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
  }
  uint32_t w = 0;
  for (int i = 0; i < (int)((rem + 7) >> 3); ++i) w |= (uint32_t)p[i] << (8 * i);
  return w;
}

// In-order merge of two span records (row order a then b).
NFC_DEV ProbeRec probe_rec_merge(const ProbeRec& a, const ProbeRec& b) {
  const bool ah = a.flags & 1u, bh = b.flags & 1u;
  const bool sorted = (a.flags & 2u) && (b.flags & 2u) && !(ah && bh && b.first < a.last);
  ProbeRec r;
  r.first = ah ? a.first : b.first;
  r.last = bh ? b.last : a.last;
  r.kmin = min(a.kmin, b.kmin);
  r.kmax = max(a.kmax, b.kmax);
  r.nvalid = a.nvalid + b.nvalid;
  r.flags = ((ah || bh) ? 1u : 0u) | (sorted ? 2u : 0u);
  return r;
}

// 256 threads: the block's 8 warps take 8 consecutive spans and the block
// writes ONE record for them (so the finalize reads nspans / 8 records).
__global__ void __launch_bounds__(256, 4) k_probe(const int32_t* __restrict__ keys, int64_t n, BitmapSet bms,
                                               uint32_t* vmask, ProbeRec* recs, int64_t nspans, bool aligned) {
  __shared__ ProbeRec s_rec[8];
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  const int64_t nbs = (nspans + 7) / 8;
  for (int64_t bs = blockIdx.x; bs < nbs; bs += gridDim.x) {
    const int64_t sp = bs * 8 + warp;
    if (sp >= nspans) {
      if (lane == 0) s_rec[warp] = ProbeRec{0, 0, INT_MAX, INT_MIN, 0u, 2u};
    } else {
    bool c_has = false;
    int32_t c_last = 0;
    bool span_has = false;
    int32_t span_first = 0;
    bool sorted = true;
    bool wsorted = true;  // warp-uniform: no descent found in this span yet
    int32_t kmn = INT_MAX, kmx = INT_MIN;
    uint32_t cnt = 0;
    for (int ch = 0; ch < kProbeChunks; ++ch) {
      const int64_t c0 = sp * kProbeSpan + (int64_t)ch * 1024;  // first row of the chunk
      if (c0 >= n) break;
      // Keys first (the largest loads in flight), then the bitmap words.
      int32_t k[8][4];
      if (aligned && c0 + 1024 <= n) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int4 kv = __ldg(reinterpret_cast<const int4*>(keys + c0 + 128 * j + 4 * lane));
          k[j][0] = kv.x; k[j][1] = kv.y; k[j][2] = kv.z; k[j][3] = kv.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int64_t i = c0 + 128 * j + 4 * lane + r;
            k[j][r] = i < n ? keys[i] : 0;
          }
      }
      // Combined validity of rows [c0 + 32 lane, +32).
      uint32_t vw = 0;
      {
        const int64_t row0 = c0 + 32 * lane;
        if (row0 < n) {
          const int64_t rem = n - row0;
          vw = rem >= 32 ? 0xFFFFFFFFu : ((1u << rem) - 1u);
#pragma unroll
          for (int b = 0; b < NFC_MAX_COLS + 2; ++b)
            if (b < bms.nbm) vw &= bitmap_word(bms.bm[b], (bms.word_aligned >> b) & 1u, row0, rem);
          if (vmask) vmask[row0 >> 5] = vw;
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t valid = (__shfl_sync(0xffffffffu, vw, 4 * j + (lane >> 3)) >> (4 * (lane & 7))) & 0xFu;
        if (!wsorted) {
          // The span is already known unsorted: its first / last keys can no
          // longer matter, so only the count and the range are kept.
#pragma unroll
          for (int r = 0; r < 4; ++r)
            if (valid & (1u << r)) {
              kmn = min(kmn, k[j][r]);
              kmx = max(kmx, k[j][r]);
            }
          cnt += __popc(valid);
          continue;
        }
        bool has = false;
        int32_t first = 0, last = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          if (valid & (1u << r)) {
            const int32_t x = k[j][r];
            if (!has) { first = x; has = true; }
            else if (x < last) sorted = false;
            last = x;
            kmn = min(kmn, x);
            kmx = max(kmx, x);
          }
        }
        cnt += __popc(valid);
        // Previous valid key in row order for this lane's first valid row.
        int eh;
        int32_t ev;
        int h31;
        int32_t v31;
        if (__all_sync(0xffffffffu, has)) {
          eh = 1;
          ev = __shfl_up_sync(0xffffffffu, last, 1);
          if (lane == 0) { eh = c_has ? 1 : 0; ev = c_last; }
          h31 = 1;
          v31 = __shfl_sync(0xffffffffu, last, 31);
        } else {
          int h = has ? 1 : 0;
          int32_t v = last;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int h2 = __shfl_up_sync(0xffffffffu, h, o);
            const int32_t v2 = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o && !h) { h = h2; v = v2; }
          }
          eh = __shfl_up_sync(0xffffffffu, h, 1);
          ev = __shfl_up_sync(0xffffffffu, v, 1);
          if (lane == 0) { eh = c_has ? 1 : 0; ev = c_last; }
          else if (!eh && c_has) { eh = 1; ev = c_last; }
          h31 = __shfl_sync(0xffffffffu, h, 31);
          v31 = __shfl_sync(0xffffffffu, v, 31);
        }
        if (has && eh && first < ev) sorted = false;
        if (h31) { c_has = true; c_last = v31; }
        const unsigned bal = __ballot_sync(0xffffffffu, has);
        if (!span_has && bal) {
          span_has = true;
          span_first = __shfl_sync(0xffffffffu, first, __ffs(bal) - 1);
        }
        wsorted = __all_sync(0xffffffffu, sorted);
      }
    }
    const bool all_sorted = __all_sync(0xffffffffu, sorted);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      kmn = min(kmn, __shfl_xor_sync(0xffffffffu, kmn, o));
      kmx = max(kmx, __shfl_xor_sync(0xffffffffu, kmx, o));
      cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    if (lane == 0) {
      ProbeRec r;
      r.first = span_first;
      r.last = c_last;
      r.kmin = kmn;
      r.kmax = kmx;
      r.nvalid = cnt;
      r.flags = (span_has ? 1u : 0u) | (all_sorted ? 2u : 0u);
      s_rec[warp] = r;
    }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      ProbeRec r = s_rec[0];
#pragma unroll
      for (int w = 1; w < 8; ++w) r = probe_rec_merge(r, s_rec[w]);
      recs[bs] = r;
    }
    __syncthreads();
  }
}

struct ProbeAcc {
  bool has, sorted;
  int32_t first, last, kmin, kmax;
  int64_t n;
};

NFC_DEV ProbeAcc probe_combine(const ProbeAcc& a, const ProbeAcc& b) {
  ProbeAcc r;
  r.has = a.has || b.has;
  r.sorted = a.sorted && b.sorted && !(a.has && b.has && b.first < a.last);
  r.first = a.has ? a.first : b.first;
  r.last = b.has ? b.last : a.last;
  r.kmin = min(a.kmin, b.kmin);
  r.kmax = max(a.kmax, b.kmax);
  r.n = a.n + b.n;
  return r;
}

NFC_DEV ProbeAcc probe_shfl_down(const ProbeAcc& a, int off) {
  ProbeAcc r;
  r.has = __shfl_down_sync(0xffffffffu, (int)a.has, off) != 0;
  r.sorted = __shfl_down_sync(0xffffffffu, (int)a.sorted, off) != 0;
  r.first = __shfl_down_sync(0xffffffffu, a.first, off);
  r.last = __shfl_down_sync(0xffffffffu, a.last, off);
  r.kmin = __shfl_down_sync(0xffffffffu, a.kmin, off);
  r.kmax = __shfl_down_sync(0xffffffffu, a.kmax, off);
  r.n = __shfl_down_sync(0xffffffffu, a.n, off);
  return r;
}

// In-order reduction of a warp's accumulators (lane order = row order).
NFC_DEV ProbeAcc probe_warp_reduce(ProbeAcc acc) {
  const int lane = lane_id();
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const ProbeAcc other = probe_shfl_down(acc, off);
    if ((lane & (2 * off - 1)) == 0) acc = probe_combine(acc, other);
  }
  return acc;
}

// One block of 1024 threads reduces the span records in row order: warp w
// owns a contiguous range and walks it in coalesced windows of 32 records.
__global__ void __launch_bounds__(1024) k_probe_finalize(const ProbeRec* recs, int64_t nspans, nfc_probe* out) {
  __shared__ ProbeAcc part[32];
  const int lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const ProbeAcc none{false, true, 0, 0, INT_MAX, INT_MIN, 0};
  const int64_t per_w = (nspans + nwarps - 1) / nwarps;
  const int64_t w0 = warp * per_w, w1 = min(nspans, w0 + per_w);
  ProbeAcc acc = none;  // meaningful in lane 0
  for (int64_t i0 = w0; i0 < w1; i0 += 32) {
    ProbeAcc x = none;
    if (i0 + lane < w1) {
      const ProbeRec r = recs[i0 + lane];
      x = ProbeAcc{(r.flags & 1u) != 0, (r.flags & 2u) != 0, r.first, r.last, r.kmin, r.kmax, (int64_t)r.nvalid};
    }
    x = probe_warp_reduce(x);
    if (lane == 0) acc = probe_combine(acc, x);
  }
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  if (warp == 0) {
    ProbeAcc w = lane < nwarps ? part[lane] : none;
    w = probe_warp_reduce(w);
    if (lane == 0) {
      nfc_probe p;
      p.n_valid = w.n;
      p.kmin = w.has ? w.kmin : 0;
      p.kmax = w.has ? w.kmax : 0;
      p.sorted = w.sorted ? 1 : 0;
      p.pad = 0;
      *out = p;
    }
  }
}

// =====================================================================
// Dense strategies.
// =====================================================================
__global__ void k_state_init(ColSet cs, StateRef st, int64_t slots) {
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < slots;
       d += (int64_t)gridDim.x * blockDim.x)
    state_init_slot(cs, st, d);
}

// Iterate the 128-row warp tiles of [0, n) owned by this warp (grid-stride)
// and call f(tile) for each.
template <bool LOAD_VALUES, class F>
NFC_DEV void for_each_tile(const int32_t* keys, const uint32_t* vmask, const ColSet& cs, int64_t n,
                           bool aligned, F&& f) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (n + 127) >> 7;
  for (int64_t tile = gw; tile < ntiles; tile += nw) {
    const int64_t row0 = tile * 128 + 4 * lane;
    Tile4 t;
    if (aligned && row0 + 4 <= n) load_tile4_full<LOAD_VALUES>(keys, vmask, cs, row0, t);
    else load_tile4_tail<LOAD_VALUES>(keys, vmask, cs, row0, n, t);
    f(t);
  }
}

__global__ void __launch_bounds__(256) k_dense_global(const int32_t* __restrict__ keys,
                                                      const uint32_t* __restrict__ vmask, ColSet cs,
                                                      int64_t n, bool aligned, int32_t kmin,
                                                      StateRef st) {
  // Row r of every lane in one warp-aggregated step: equal keys of a warp
  // (hot keys, runs) are combined before their atomics.
  for_each_tile<true>(keys, vmask, cs, n, aligned, [&](const Tile4& t) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      uint64_t raw[NFC_MAX_COLS];
#pragma unroll
      for (int c = 0; c < NFC_MAX_COLS; ++c) raw[c] = t.raw[c][r];
      warp_agg_apply(cs, st, (t.valid >> r) & 1u, t.key[r], raw,
                     [&](int32_t key) { return (int64_t)key - kmin; });
    }
  });
}

// DENSE_SMEM, typed: one CTA per chunk of kDsChunk rows folds its rows into
// a shared-memory state of the whole span with the split-sum / ordered
// min-max state of the partition aggregate (native 32- and 64-bit shared
// atomics only; a chunk of at most 65,536 rows keeps the 16-bit-half int32
// sums exact), then merges its present slots into the global state.
constexpr int64_t kDsChunk = 65536;

template <int NC>
__global__ void __launch_bounds__(512, 2) k_dense_smem_t(const int32_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ vmask, ColSet cs, int64_t n,
                                                        bool aligned, int32_t kmin, int32_t m, StateRef gst) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const AggState<NC> st = carve_agg<NC, 0>(cs, smem_raw, m);
  for (int g = threadIdx.x; g < m; g += blockDim.x) agg_init<NC, 0>(cs, st, g);
  __syncthreads();
  const int64_t r0 = blockIdx.x * kDsChunk;
  const int64_t r1 = min(n, r0 + kDsChunk);
  const int lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  constexpr int U = NC >= 2 ? 1 : 2;  // 128-row tiles in flight per warp (registers)
  for (int64_t t0 = r0 + (int64_t)warp * 128 * U; t0 < r1; t0 += (int64_t)nwarps * 128 * U) {
    TileT<NC> t[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t row0 = t0 + u * 128 + 4 * lane;
      if (aligned && row0 + 4 <= r1) load_tile4_full<true, NC, 0>(keys, vmask, cs, row0, t[u]);
      else load_tile4_tail<true, NC, 0>(keys, vmask, cs, row0, r1, t[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (t[u].valid & (1u << r)) {
          uint64_t raw[NC > 0 ? NC : 1];
#pragma unroll
          for (int c = 0; c < NC; ++c) raw[c] = t[u].raw[c][r];
          agg_apply<NC, 0>(cs, st, (uint32_t)(t[u].key[r] - kmin), raw);
        }
  }
  __syncthreads();
  for (int g = threadIdx.x; g < m; g += blockDim.x) agg_merge<NC, 0>(cs, gst, g, st, g);
}

template <int NC>
static int launch_dense_smem_t(const int32_t* keys, const uint32_t* vmask, const ColSet& cs, int64_t n, bool al,
                               int32_t kmin, int32_t m, const StateRef& gst, cudaStream_t s) {
  const size_t smem = (size_t)m * state_bytes_per_slot(cs) + 64;
  NFC_CUDA(cudaFuncSetAttribute(k_dense_smem_t<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t grid = std::max<int64_t>(1, (n + kDsChunk - 1) / kDsChunk);
  k_dense_smem_t<NC><<<(unsigned)grid, 512, smem, s>>>(keys, vmask, cs, n, al, kmin, m, gst);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

// Compact a dense global state (slots [0, m)) into ascending groups.
// Tile = blockDim * 4 consecutive slots; tiles claimed in order by ticket.
__global__ void __launch_bounds__(256) k_compact_dense(ColSet cs, StateRef st, int64_t m, int64_t kmin,
                                                       OutSet o, uint64_t* lb, uint32_t* ticket,
                                                       int64_t* ng_out, int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t per_tile = (int64_t)blockDim.x * 4;
  const int64_t ntiles = (m + per_tile - 1) / per_tile;
  if (tile >= ntiles) return;
  const int64_t s0 = tile * per_tile + threadIdx.x * 4;
  uint32_t pres = 0, c = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (s0 + j < m && st.cnt[s0 + j] != 0u) { pres |= 1u << j; ++c; }
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
  int64_t pos = s_base + excl;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (pres & (1u << j)) state_emit(cs, st, s0 + j, o, pos++, kmin + s0 + j);
}

// =====================================================================
// Host orchestration.
// =====================================================================
static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

static int grid_stream(int64_t work_tiles, int per_sm) {
  int64_t g = std::min<int64_t>(work_tiles, (int64_t)num_sms() * per_sm);
  return (int)std::max<int64_t>(g, 1);
}

int build_colset(const nfc_groupby_args* a, ColSet* cs, OutSet* o) {
  if (a->ncols < 0 || a->ncols > NFC_MAX_COLS) {
    set_last_error("ncols %d outside [0, %d]", a->ncols, NFC_MAX_COLS);
    return NFC_ERR_MALFORMED;
  }
  cs->ncols = a->ncols;
  o->ukeys = a->ukeys_out;
  o->counts = a->counts_out;
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    cs->dtype[c] = NFC_I32;
    cs->aggs[c] = 0;
    cs->data[c] = nullptr;
    o->sum[c] = o->mn[c] = o->mx[c] = nullptr;
  }
  for (int c = 0; c < a->ncols; ++c) {
    const nfc_value_col& v = a->cols[c];
    if (v.dtype != NFC_I32 && v.dtype != NFC_I64 && v.dtype != NFC_F64) {
      set_last_error("column %d: unknown dtype %d", c, v.dtype);
      return NFC_ERR_MALFORMED;
    }
    if (!v.data && a->n > 0) return NFC_ERR_NULL;
    if (((v.aggs & NFC_AGG_SUM) && !v.sum_out) || ((v.aggs & NFC_AGG_MIN) && !v.min_out) ||
        ((v.aggs & NFC_AGG_MAX) && !v.max_out))
      return NFC_ERR_NULL;
    cs->dtype[c] = v.dtype;
    cs->aggs[c] = v.aggs & (NFC_AGG_SUM | NFC_AGG_MIN | NFC_AGG_MAX);
    cs->data[c] = v.data;
    o->sum[c] = v.sum_out;
    o->mn[c] = v.min_out;
    o->mx[c] = v.max_out;
  }
  return NFC_OK;
}

bool inputs_aligned(const nfc_groupby_args* a) {
  if (!aligned16(a->keys)) return false;
  for (int c = 0; c < a->ncols; ++c)
    if (!aligned16(a->cols[c].data)) return false;
  return true;
}

int run_probe(const nfc_groupby_args* a, cudaStream_t s, Scratch& sc, uint32_t** vmask_out,
              nfc_probe* host_probe, StageTimer* tm, const ProbeRec** recs_out) {
  const int64_t n = a->n;
  BitmapSet bms{};
  bms.nbm = 0;
  bms.word_aligned = 0;
  if (a->key_validity) bms.bm[bms.nbm++] = a->key_validity;
  for (int c = 0; c < a->ncols; ++c)
    if (a->cols[c].validity) bms.bm[bms.nbm++] = a->cols[c].validity;
  if (a->row_filter) bms.bm[bms.nbm++] = a->row_filter;
  for (int b = 0; b < bms.nbm; ++b)
    if ((reinterpret_cast<uintptr_t>(bms.bm[b]) & 3u) == 0) bms.word_aligned |= 1u << b;
  uint32_t* vmask = nullptr;
  if (bms.nbm > 0) NFC_CUDA(sc.alloc(&vmask, (size_t)((n + 31) / 32 + 1)));
  const int64_t nspans = (n + kProbeSpan - 1) / kProbeSpan;
  ProbeRec* recs = nullptr;
  nfc_probe* dprobe = nullptr;
  NFC_CUDA(sc.alloc(&recs, (size_t)std::max<int64_t>((nspans + 7) / 8, 1)));
  NFC_CUDA(sc.alloc(&dprobe, 1));
  tm->mark(s);
  if (nspans > 0) {
    const int grid = grid_stream((nspans + 7) / 8, 8);
    k_probe<<<grid, 256, 0, s>>>(a->keys, n, bms, vmask, recs, nspans, aligned16(a->keys));
    NFC_CUDA(cudaGetLastError());
    tm->launched();
  }
  k_probe_finalize<<<1, 1024, 0, s>>>(recs, (nspans + 7) / 8, dprobe);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);
  NFC_CUDA(readback(host_probe, dprobe, sizeof(nfc_probe), s));
  *vmask_out = vmask;
  if (recs_out) *recs_out = recs;
  return NFC_OK;
}

// Shared-memory budget for one CTA's dense state.
constexpr size_t kSmemStateBudget = 200 * 1024;
// Valid rows from which PARTITION is preferred to DENSE_GLOBAL.
constexpr int64_t kDenseGlobalMaxRows = 4 << 20;
int plan_strategy(const ColSet& cs, const nfc_probe& p) {
  if (p.n_valid == 0) return NFC_STRAT_DENSE_GLOBAL;
  // Nondecreasing valid keys: one pass over runs, no atomics (the reference's
  // planner takes its sorted plan whenever the keys are sorted).
  if (p.sorted) return NFC_STRAT_SORTED;
  const int64_t m = p.kmax - p.kmin + 1;
  const size_t slot = state_bytes_per_slot(cs);
  // Span that one CTA's shared memory holds (two CTAs per SM).
  if ((size_t)m * slot <= 96 * 1024 && p.n_valid >= 4 * m) return NFC_STRAT_DENSE_SMEM;
  int wb;
  const bool part = m <= 4 * p.n_valid + 65536 && pick_partition_width(slot, m, &wb) == 0;
  // Span whose global state stays L2-resident: one global atomic per row
  // update.  From a few million rows the partition path (two coalesced
  // scatter passes, shared-memory aggregation) is faster on B200 (100M rows
  // over 50K..200K keys: 1.7 against 3.3 ms; 10M rows: 0.41 against 0.47 ms).
  if ((size_t)m * slot <= (size_t)24 << 20 && m <= 4 * p.n_valid + 4096 &&
      (!part || p.n_valid < kDenseGlobalMaxRows))
    return NFC_STRAT_DENSE_GLOBAL;
  if (part) return NFC_STRAT_PARTITION;
  return NFC_STRAT_HASH;
}

static int finish_ng(cudaStream_t s, const int64_t* d_ng, const int32_t* d_err, int64_t* ng, int32_t* status) {
  int64_t local[2] = {0, 0};
  unsigned char* pin = pinned_readback();
  int64_t* h = pin ? reinterpret_cast<int64_t*>(pin) : local;
  h[1] = 0;
  NFC_CUDA(cudaMemcpyAsync(&h[0], d_ng, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaMemcpyAsync(&h[1], d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  *ng = h[0];
  *status = (int32_t)h[1];
  return NFC_OK;
}

static int compact_dense(const ColSet& cs, const StateRef& st, int64_t m, int64_t kmin, const OutSet& o,
                         cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err, StageTimer* tm) {
  const int64_t per_tile = 256 * 4;
  const int64_t ntiles = (m + per_tile - 1) / per_tile;
  uint64_t* lb = nullptr;
  uint32_t* ticket = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)std::max<int64_t>(ntiles, 1)));
  NFC_CUDA(sc.alloc(&ticket, 1));
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * std::max<int64_t>(ntiles, 1), s));
  NFC_CUDA(cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s));
  if (ntiles > 0) {
    k_compact_dense<<<(unsigned)ntiles, 256, 0, s>>>(cs, st, m, kmin, o, lb, ticket, d_ng, d_err);
    NFC_CUDA(cudaGetLastError());
    tm->launched();
  }
  tm->mark(s);
  return NFC_OK;
}

int run_dense(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
              const uint32_t* vmask, bool smem_variant, cudaStream_t s, Scratch& sc, int64_t* d_ng,
              int32_t* d_err, StageTimer* tm) {
  const int64_t m = p.kmax - p.kmin + 1;
  const size_t slot = state_bytes_per_slot(cs);
  void* gbase = nullptr;
  unsigned char* gb = nullptr;
  NFC_CUDA(sc.alloc(&gb, (size_t)m * slot + 64));
  gbase = gb;
  const StateRef gst = carve_state(cs, gbase, m);
  k_state_init<<<grid_stream((m + 255) / 256, 8), 256, 0, s>>>(cs, gst, m);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);
  const bool al = inputs_aligned(a);
  const int64_t ntiles128 = (a->n + 127) / 128;
  if (smem_variant) {
    int rc;
    switch (cs.ncols) {
      case 0: rc = launch_dense_smem_t<0>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, (int32_t)m, gst, s); break;
      case 1: rc = launch_dense_smem_t<1>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, (int32_t)m, gst, s); break;
      case 2: rc = launch_dense_smem_t<2>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, (int32_t)m, gst, s); break;
      case 3: rc = launch_dense_smem_t<3>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, (int32_t)m, gst, s); break;
      default: rc = launch_dense_smem_t<4>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, (int32_t)m, gst, s); break;
    }
    if (rc) return rc;
  } else {
    const int grid = grid_stream((ntiles128 + 7) / 8, 8);
    k_dense_global<<<grid, 256, 0, s>>>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, gst);
  }
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);
  return compact_dense(cs, gst, m, p.kmin, o, s, sc, d_ng, d_err, tm);
}

}  // namespace nfc

using namespace nfc;

extern "C" int32_t nfc_plan_strategy(const nfc_groupby_args* args, const nfc_probe* probe) {
  if (!args || !probe) return NFC_ERR_NULL;
  ColSet cs;
  OutSet o;
  const int rc = build_colset(args, &cs, &o);
  if (rc) return rc;
  return plan_strategy(cs, *probe);
}

extern "C" int64_t nfc_groupby(const nfc_groupby_args* a, int32_t strategy, void* stream,
                               nfc_groupby_stats* stats) {
  return nfc::groupby_run(a, strategy, nullptr, stream, stats);
}

// Group-by body shared by nfc_groupby and nfc_groupby_planned: probe, pick
// the strategy (explicit, AUTO, or the planning hook), run it, read back ng.
int64_t nfc::groupby_run(const nfc_groupby_args* a, int32_t strategy, PlanHook* hook, void* stream,
                         nfc_groupby_stats* stats) {
  if (!a) return NFC_ERR_NULL;
  if (a->n < 0 || a->n > INT32_MAX) {
    set_last_error("n=%lld outside [0, 2^31)", (long long)a->n);
    return NFC_ERR_MALFORMED;
  }
  if (a->n > 0 && !a->keys) return NFC_ERR_NULL;
  if (!a->ukeys_out || !a->counts_out || (a->ncols > 0 && !a->cols)) return NFC_ERR_NULL;
  ColSet cs;
  OutSet o;
  int rc = build_colset(a, &cs, &o);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  StageTimer tm;
  tm.on = stats && stats->timing;
  uint32_t* vmask = nullptr;
  nfc_probe p;
  const ProbeRec* recs = nullptr;
  rc = run_probe(a, s, sc, &vmask, &p, &tm, &recs);
  if (rc) return rc;
  int strat = strategy == NFC_STRAT_AUTO ? plan_strategy(cs, p) : strategy;
  int64_t hint = stats ? stats->distinct_hint : 0;
  if (hook) {
    rc = hook->choose(cs, p, &strat, &hint);
    if (rc) return rc;
  }
  if (stats) {
    stats->probe = p;
    stats->strategy = strat;
    stats->status = 0;
    stats->ng = 0;
    stats->buckets = 0;
    stats->launches = tm.launches;
    stats->nstages = 0;
  }
  if (p.n_valid == 0) return 0;
  const int64_t m = p.kmax - p.kmin + 1;
  const int64_t ng_bound = std::min<int64_t>(m, p.n_valid);
  if (a->out_cap < ng_bound && a->out_cap < p.n_valid) {
    // Only the true ng matters, but it is unknown before the run; demand
    // the bound that is always sufficient.
    set_last_error("out_cap %lld < min(span, n_valid) = %lld", (long long)a->out_cap, (long long)ng_bound);
    return NFC_ERR_RANGE;
  }
  int64_t* d_ng = nullptr;
  int32_t* d_err = nullptr;
  NFC_CUDA(sc.alloc(&d_ng, 2));
  d_err = reinterpret_cast<int32_t*>(d_ng + 1);
  NFC_CUDA(cudaMemsetAsync(d_ng, 0, 2 * sizeof(int64_t), s));
  int64_t buckets = 0;
  int32_t overflowed = 0;
  const size_t slot = state_bytes_per_slot(cs);
  // The radix sort keeps 30-bit positions.
  if (strat == NFC_STRAT_SORT && p.n_valid >= (1ll << 30)) strat = NFC_STRAT_HASH;
  // SORTED needs nondecreasing valid keys; on other input it is only a hint.
  if (strat == NFC_STRAT_SORTED && !p.sorted) strat = plan_strategy(cs, p);
  if (strat == NFC_STRAT_DENSE_SMEM && (size_t)m * slot + 64 > kSmemStateBudget) strat = NFC_STRAT_DENSE_GLOBAL;
  switch (strat) {
    case NFC_STRAT_SORTED:
      rc = run_sorted(a, cs, o, p, vmask, recs, s, sc, d_ng, d_err, &tm);
      break;
    case NFC_STRAT_DENSE_SMEM:
      rc = run_dense(a, cs, o, p, vmask, true, s, sc, d_ng, d_err, &tm);
      break;
    case NFC_STRAT_DENSE_GLOBAL:
      if ((double)m * slot > 64.0e9) { rc = NFC_ERR_UNSUPPORTED; set_last_error("dense span too large"); break; }
      rc = run_dense(a, cs, o, p, vmask, false, s, sc, d_ng, d_err, &tm);
      break;
    case NFC_STRAT_PARTITION:
      rc = run_partition(a, cs, o, p, vmask, s, sc, d_ng, d_err, &buckets, &tm);
      break;
    case NFC_STRAT_HASH:
      rc = run_hash(a, cs, o, p, vmask, s, sc, d_ng, d_err, &buckets, &tm);
      break;
    case NFC_STRAT_SHARED_HASH: {
      int level = 0;
      rc = run_shared_hash(a, cs, o, p, vmask, hint, s, sc, d_ng, d_err, &buckets, &level, &tm);
      overflowed = level;
      if (rc == NFC_OK && level == 2) {
        // Even the full-size shared pass overflowed its probe bound: HASH.
        NFC_CUDA(cudaMemsetAsync(d_ng, 0, 2 * sizeof(int64_t), s));
        rc = run_hash(a, cs, o, p, vmask, s, sc, d_ng, d_err, &buckets, &tm);
      }
      break;
    }
    case NFC_STRAT_SORT:
      rc = run_sort_groupby(a, cs, o, p, vmask, s, sc, d_ng, d_err, &tm);
      break;
    default:
      set_last_error("unknown strategy %d", strat);
      return NFC_ERR_MALFORMED;
  }
  if (rc) return rc;
  int64_t ng = 0;
  int32_t status = 0;
  rc = finish_ng(s, d_ng, d_err, &ng, &status);
  if (rc) return rc;
  if (stats) {
    stats->strategy = strat;
    stats->status = status;
    stats->ng = ng;
    stats->buckets = buckets;
    stats->overflowed = overflowed;
    stats->launches = tm.launches;
    stats->nstages = tm.finish(stats->stage_ms);
  }
  if (status) {
    set_last_error("device status %d", status);
    return status;
  }
  return ng;
}

// =====================================================================
// Group-by without allocation (nfc_groupby_dense_noalloc).
//
// For callers that cannot allocate device memory: scratch is the static
// array below (NFC_NOALLOC_SCRATCH_BYTES, held by every GPU that loads the
// library until exit).  Host code never dereferences the array's name: it
// is a host-side stand-in, so the device address is looked up once per
// device with cudaGetSymbolAddress and passed to the kernels.
// =====================================================================
#include <mutex>

static __device__ __align__(256) unsigned char g_noalloc_scratch[NFC_NOALLOC_SCRATCH_BYTES];

namespace nfc {
namespace {

// Layout of the static scratch (byte offsets).
constexpr size_t kNaHdr = 0;                                              // ng i64, err i32, ticket u32, probe
constexpr size_t kNaRecs = 256;                                           // probe span records
constexpr size_t kNaRecsBytes = ((NFC_NOALLOC_MAX_ROWS + kProbeSpan - 1) / kProbeSpan) * sizeof(ProbeRec);
constexpr size_t kNaVmask = (kNaRecs + kNaRecsBytes + 255) & ~(size_t)255;
constexpr size_t kNaVmaskBytes = ((NFC_NOALLOC_MAX_ROWS + 31) / 32 + 1) * 4;
constexpr size_t kNaLb = (kNaVmask + kNaVmaskBytes + 255) & ~(size_t)255;
constexpr size_t kNaLbBytes = ((NFC_NOALLOC_STATE_BYTES / 4 + 1023) / 1024 + 1) * 8;  // tiles of 1024 slots
constexpr size_t kNaState = (kNaLb + kNaLbBytes + 255) & ~(size_t)255;
static_assert(kNaState + NFC_NOALLOC_STATE_BYTES <= NFC_NOALLOC_SCRATCH_BYTES, "no-alloc scratch budget");

std::mutex g_na_mu;
unsigned char* g_na_ptr[64] = {};

// Device address of the scratch array for the current device (looked up
// once per device, with that device current).  The address belongs to the
// device's primary context: after cudaDeviceReset it is stale, which is why
// the entry point's contract rules out calls after a reset.
int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  NFC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_last_error("device ordinal %d unsupported", dev);
    return NFC_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_na_mu);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    NFC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_na_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_na_ptr[dev];
  return NFC_OK;
}

}  // namespace
}  // namespace nfc

extern "C" int64_t nfc_groupby_dense_noalloc(const nfc_groupby_args* a, void* stream) {
  if (!a) return NFC_ERR_NULL;
  if (a->n < 0) return NFC_ERR_MALFORMED;
  if (a->n > NFC_NOALLOC_MAX_ROWS) {
    set_last_error("nfc_groupby_dense_noalloc: n=%lld exceeds NFC_NOALLOC_MAX_ROWS=%lld", (long long)a->n,
                   (long long)NFC_NOALLOC_MAX_ROWS);
    return NFC_ERR_RANGE;
  }
  if (a->n > 0 && !a->keys) return NFC_ERR_NULL;
  if (!a->ukeys_out || !a->counts_out || (a->ncols > 0 && !a->cols)) return NFC_ERR_NULL;
  ColSet cs;
  OutSet o;
  int rc = build_colset(a, &cs, &o);
  if (rc) return rc;
  unsigned char* base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int64_t* d_ng = reinterpret_cast<int64_t*>(base + kNaHdr);
  int32_t* d_err = reinterpret_cast<int32_t*>(base + kNaHdr + 8);
  uint32_t* d_ticket = reinterpret_cast<uint32_t*>(base + kNaHdr + 12);
  nfc_probe* d_probe = reinterpret_cast<nfc_probe*>(base + kNaHdr + 64);
  ProbeRec* recs = reinterpret_cast<ProbeRec*>(base + kNaRecs);
  uint32_t* vmask_buf = reinterpret_cast<uint32_t*>(base + kNaVmask);
  uint64_t* lb = reinterpret_cast<uint64_t*>(base + kNaLb);
  unsigned char* state = base + kNaState;

  // Probe: n_valid, kmin/kmax and the combined validity bitmap.
  BitmapSet bms{};
  bms.nbm = 0;
  bms.word_aligned = 0;
  if (a->key_validity) bms.bm[bms.nbm++] = a->key_validity;
  for (int c = 0; c < a->ncols; ++c)
    if (a->cols[c].validity) bms.bm[bms.nbm++] = a->cols[c].validity;
  if (a->row_filter) bms.bm[bms.nbm++] = a->row_filter;
  for (int b = 0; b < bms.nbm; ++b)
    if ((reinterpret_cast<uintptr_t>(bms.bm[b]) & 3u) == 0) bms.word_aligned |= 1u << b;
  uint32_t* vmask = bms.nbm > 0 ? vmask_buf : nullptr;
  NFC_CUDA(cudaMemsetAsync(base + kNaHdr, 0, 256, s));
  const int64_t nspans = (a->n + kProbeSpan - 1) / kProbeSpan;
  if (nspans > 0) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nspans + 7) / 8, (int64_t)num_sms() * 8));
    k_probe<<<grid, 256, 0, s>>>(a->keys, a->n, bms, vmask, recs, nspans,
                                 (reinterpret_cast<uintptr_t>(a->keys) & 15u) == 0);
    NFC_CUDA(cudaGetLastError());
  }
  k_probe_finalize<<<1, 1024, 0, s>>>(recs, (nspans + 7) / 8, d_probe);
  NFC_CUDA(cudaGetLastError());
  nfc_probe p;
  NFC_CUDA(cudaMemcpyAsync(&p, d_probe, sizeof(p), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if (p.n_valid == 0) return 0;
  const int64_t m = p.kmax - p.kmin + 1;
  const size_t slot = state_bytes_per_slot(cs);
  if ((double)m * (double)slot > (double)NFC_NOALLOC_STATE_BYTES) {
    set_last_error("nfc_groupby_dense_noalloc: key span %lld x %zu B/group exceeds NFC_NOALLOC_STATE_BYTES=%lld",
                   (long long)m, slot, (long long)NFC_NOALLOC_STATE_BYTES);
    return NFC_ERR_RANGE;
  }
  if (a->out_cap < std::min<int64_t>(m, p.n_valid)) {
    set_last_error("out_cap %lld < min(span, n_valid)", (long long)a->out_cap);
    return NFC_ERR_RANGE;
  }
  // Dense state (initialised every call), one atomic pass, compaction.
  const StateRef st = carve_state(cs, state, m);
  k_state_init<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, (int64_t)num_sms() * 8)), 256, 0,
                 s>>>(cs, st, m);
  NFC_CUDA(cudaGetLastError());
  const int64_t ntiles128 = (a->n + 127) / 128;
  const bool al = inputs_aligned(a);
  k_dense_global<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((ntiles128 + 7) / 8, (int64_t)num_sms() * 8)), 256,
                   0, s>>>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, st);
  NFC_CUDA(cudaGetLastError());
  const int64_t ctiles = (m + 1023) / 1024;
  NFC_CUDA(cudaMemsetAsync(lb, 0, (size_t)ctiles * sizeof(uint64_t), s));
  k_compact_dense<<<(unsigned)ctiles, 256, 0, s>>>(cs, st, m, p.kmin, o, lb, d_ticket, d_ng, d_err);
  NFC_CUDA(cudaGetLastError());
  int64_t h[2] = {0, 0};
  NFC_CUDA(cudaMemcpyAsync(h, d_ng, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  const int32_t status = (int32_t)(h[1] & 0xFFFFFFFF);
  if (status) {
    set_last_error("device status %d", status);
    return status;
  }
  return h[0];
}
