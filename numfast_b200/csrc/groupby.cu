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
//   DENSE_SMEM   span M fits one CTA's shared memory: every CTA keeps the
//                whole state on chip, merges it once into a global table.
//   DENSE_GLOBAL span fits L2: rows update one global table with atomics.
//   PARTITION    large span: rows are scattered into key-range buckets of W
//                keys (one histogram pass + one scatter pass); one CTA per
//                bucket aggregates on chip and writes its groups straight to
//                their final place (decoupled look-back over buckets).
//   HASH         sparse keys: see hash.cu.
#include <algorithm>
#include <vector>

#include "groupby_core.cuh"
#include "groupby_host.h"

namespace nfc {

// =====================================================================
// Probe: n_valid, kmin/kmax over valid rows, sortedness of valid keys,
// and the combined validity bitmap (AND of every input bitmap).
// =====================================================================
constexpr int kProbeIters = 16;  // 128-row iterations per warp span
constexpr int64_t kProbeSpan = 128 * kProbeIters;

struct ProbeRec {
  int32_t first, last, kmin, kmax;
  uint32_t nvalid, flags;  // flags: bit0 has-valid, bit1 sorted
};

struct BitmapSet {
  int32_t nbm;
  const uint8_t* bm[NFC_MAX_COLS + 1];
};

NFC_DEV uint32_t nibble_at(const uint8_t* bm, int64_t row0, int64_t n) {
  // row0 is a multiple of 4: the 4 bits live in one byte.
  uint32_t v = (bm[row0 >> 3] >> (row0 & 7)) & 0xFu;
  const int64_t rem = n - row0;
  if (rem < 4) v &= (1u << (rem > 0 ? rem : 0)) - 1u;
  return v;
}

__global__ void k_probe(const int32_t* __restrict__ keys, int64_t n, BitmapSet bms, uint32_t* vmask,
                        ProbeRec* recs, int64_t nspans, bool aligned) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sp = gw; sp < nspans; sp += nw) {
    bool c_has = false;
    int32_t c_last = 0;
    bool span_has = false;
    int32_t span_first = 0;
    bool sorted = true;
    int32_t kmn = INT_MAX, kmx = INT_MIN;
    uint32_t cnt = 0;
    for (int it = 0; it < kProbeIters; ++it) {
      const int64_t row0 = sp * kProbeSpan + it * 128 + 4 * lane;
      int32_t k[4] = {0, 0, 0, 0};
      uint32_t valid = 0;
      if (row0 + 4 <= n && aligned) {
        const int4 kv = __ldcs(reinterpret_cast<const int4*>(keys + row0));
        k[0] = kv.x; k[1] = kv.y; k[2] = kv.z; k[3] = kv.w;
        valid = 0xFu;
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (row0 + r < n) { k[r] = keys[row0 + r]; valid |= 1u << r; }
      }
      if (row0 >= n) valid = 0;
      for (int b = 0; b < bms.nbm; ++b)
        if (row0 < n) valid &= nibble_at(bms.bm[b], row0, n);
      if (vmask) {
        uint32_t word = valid << (4 * (lane & 7));
        word |= __shfl_xor_sync(0xffffffffu, word, 1);
        word |= __shfl_xor_sync(0xffffffffu, word, 2);
        word |= __shfl_xor_sync(0xffffffffu, word, 4);
        if ((lane & 7) == 0 && row0 < n) vmask[row0 >> 5] = word;
      }
      // Lane-local run over its 4 rows.
      bool has = false;
      int32_t first = 0, last = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (valid & (1u << r)) {
          if (!has) { first = k[r]; has = true; }
          else if (k[r] < last) sorted = false;
          last = k[r];
          kmn = min(kmn, k[r]);
          kmx = max(kmx, k[r]);
          ++cnt;
        }
      }
      // Inclusive "latest valid key" scan across lanes.
      int h = has ? 1 : 0;
      int32_t v = last;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int h2 = __shfl_up_sync(0xffffffffu, h, o);
        const int32_t v2 = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o && !h) { h = h2; v = v2; }
      }
      int eh = __shfl_up_sync(0xffffffffu, h, 1);
      int32_t ev = __shfl_up_sync(0xffffffffu, v, 1);
      if (lane == 0) { eh = c_has ? 1 : 0; ev = c_last; }
      else if (!eh && c_has) { eh = 1; ev = c_last; }
      if (has && eh && first < ev) sorted = false;
      const int h31 = __shfl_sync(0xffffffffu, h, 31);
      const int32_t v31 = __shfl_sync(0xffffffffu, v, 31);
      if (h31) { c_has = true; c_last = v31; }
      const unsigned bal = __ballot_sync(0xffffffffu, has);
      if (!span_has && bal) {
        span_has = true;
        span_first = __shfl_sync(0xffffffffu, first, __ffs(bal) - 1);
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
      recs[sp] = r;
    }
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

__global__ void k_probe_finalize(const ProbeRec* recs, int64_t nspans, nfc_probe* out) {
  __shared__ ProbeAcc part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int64_t per = (nspans + nt - 1) / nt;
  ProbeAcc acc{false, true, 0, 0, INT_MAX, INT_MIN, 0};
  for (int64_t i = t * per; i < min(nspans, (t + 1) * per); ++i) {
    const ProbeRec r = recs[i];
    ProbeAcc b{(r.flags & 1u) != 0, (r.flags & 2u) != 0, r.first, r.last, r.kmin, r.kmax, (int64_t)r.nvalid};
    acc = probe_combine(acc, b);
  }
  part[t] = acc;
  __syncthreads();
  if (t == 0) {
    ProbeAcc a = part[0];
    for (int i = 1; i < nt; ++i) a = probe_combine(a, part[i]);
    nfc_probe p;
    p.n_valid = a.n;
    p.kmin = a.has ? a.kmin : 0;
    p.kmax = a.has ? a.kmax : 0;
    p.sorted = a.sorted ? 1 : 0;
    p.pad = 0;
    *out = p;
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
  for_each_tile<true>(keys, vmask, cs, n, aligned, [&](const Tile4& t) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (t.valid & (1u << r)) {
        uint64_t raw[NFC_MAX_COLS];
#pragma unroll
        for (int c = 0; c < NFC_MAX_COLS; ++c) raw[c] = t.raw[c][r];
        state_apply(cs, st, (int64_t)t.key[r] - kmin, raw);
      }
    }
  });
}

__global__ void __launch_bounds__(512) k_dense_smem(const int32_t* __restrict__ keys,
                                                    const uint32_t* __restrict__ vmask, ColSet cs,
                                                    int64_t n, bool aligned, int32_t kmin, int32_t m,
                                                    StateRef gst) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const StateRef sst = carve_state(cs, smem_raw, m);
  for (int d = threadIdx.x; d < m; d += blockDim.x) state_init_slot(cs, sst, d);
  __syncthreads();
  for_each_tile<true>(keys, vmask, cs, n, aligned, [&](const Tile4& t) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (t.valid & (1u << r)) {
        uint64_t raw[NFC_MAX_COLS];
#pragma unroll
        for (int c = 0; c < NFC_MAX_COLS; ++c) raw[c] = t.raw[c][r];
        state_apply(cs, sst, t.key[r] - kmin, raw);
      }
    }
  });
  __syncthreads();
  for (int d = threadIdx.x; d < m; d += blockDim.x) state_merge(cs, gst, d, sst, d);
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
  if (threadIdx.x == 0) {
    s_base = lookback_exclusive(lb, tile, total, err);
    if (tile == ntiles - 1) *ng_out = s_base + total;
  }
  __syncthreads();
  int64_t pos = s_base + excl;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (pres & (1u << j)) state_emit(cs, st, s0 + j, o, pos++, kmin + s0 + j);
}

// =====================================================================
// PARTITION strategy.
// =====================================================================
__global__ void __launch_bounds__(256) k_part_hist(const int32_t* __restrict__ keys,
                                                   const uint32_t* __restrict__ vmask, int64_t n,
                                                   bool aligned, int32_t kmin, int wb, int32_t nb,
                                                   uint32_t* __restrict__ ghist) {
  extern __shared__ uint32_t s_hist[];
  for (int j = threadIdx.x; j < nb; j += blockDim.x) s_hist[j] = 0u;
  __syncthreads();
  ColSet none{};
  for_each_tile<false>(keys, vmask, none, n, aligned, [&](const Tile4& t) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const bool v = (t.valid >> r) & 1u;
      const uint32_t b = v ? (uint32_t)(((int64_t)t.key[r] - kmin) >> wb) : 0xFFFFFFFFu;
      const unsigned peers = __match_any_sync(0xffffffffu, b);
      if (v && (__ffs(peers) - 1) == lane_id()) atomicAdd(&s_hist[b], (uint32_t)__popc(peers));
    }
  });
  __syncthreads();
  for (int j = threadIdx.x; j < nb; j += blockDim.x)
    if (s_hist[j]) atomicAdd(&ghist[j], s_hist[j]);
}

struct PartPlan {
  int64_t* offs;        // [nb+1] record offsets
  uint32_t* cursor;     // [nb]   scatter cursors
  int32_t* item_base;   // [nb+1] work-item offsets (slices)
  int32_t* merge_slot;  // [nb]   -1 or merge-state slot
  int32_t* n_merge;     // [1]
};

// One CTA of 1024 threads scans the bucket histogram into record offsets,
// work items (buckets of more than `slice` records are split) and merge
// slots for the split buckets.
__global__ void __launch_bounds__(1024) k_part_plan(const uint32_t* ghist, int32_t nb, int64_t slice,
                                                    PartPlan pl) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_carry_off;
  __shared__ int32_t s_carry_item, s_carry_merge;
  if (threadIdx.x == 0) { s_carry_off = 0; s_carry_item = 0; s_carry_merge = 0; }
  __syncthreads();
  for (int64_t base = 0; base < nb; base += blockDim.x) {
    const int64_t b = base + threadIdx.x;
    const uint32_t h = b < nb ? ghist[b] : 0u;
    const uint32_t items = b < nb ? (uint32_t)(h > slice ? (h + slice - 1) / slice : 1) : 0u;
    const uint32_t multi = (b < nb && items > 1) ? 1u : 0u;
    uint32_t t_off, t_items, t_multi;
    const uint32_t e_off = block_excl_scan(h, s_scan, &t_off);
    const uint32_t e_items = block_excl_scan(items, s_scan, &t_items);
    const uint32_t e_multi = block_excl_scan(multi, s_scan, &t_multi);
    if (b < nb) {
      const int64_t off = s_carry_off + e_off;
      pl.offs[b] = off;
      pl.cursor[b] = (uint32_t)off;
      pl.item_base[b] = s_carry_item + (int32_t)e_items;
      pl.merge_slot[b] = multi ? s_carry_merge + (int32_t)e_multi : -1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_carry_off += t_off;
      s_carry_item += (int32_t)t_items;
      s_carry_merge += (int32_t)t_multi;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pl.offs[nb] = s_carry_off;
    pl.item_base[nb] = s_carry_item;
    *pl.n_merge = s_carry_merge;
  }
}

struct Records {
  uint16_t* klow;
  void* v[NFC_MAX_COLS];
};

constexpr int kScatterIters = 2;  // 128-row iterations per warp per tile
constexpr int kScatterThreads = 512;

template <int NC>
__global__ void __launch_bounds__(kScatterThreads, 1) k_part_scatter(const int32_t* __restrict__ keys,
                                                                    const uint32_t* __restrict__ vmask, ColSet cs,
                                                                    int64_t n, bool aligned, int32_t kmin, int wb,
                                                                    int32_t nb, uint32_t* __restrict__ cursor,
                                                                    Records rec) {
  extern __shared__ uint32_t s_part[];
  uint32_t* s_cnt = s_part;
  uint32_t* s_base = s_part + nb;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) s_cnt[j] = 0u;
  __syncthreads();
  const int lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int64_t tile_rows = (int64_t)nwarps * kScatterIters * 128;
  const int64_t ntiles = (n + tile_rows - 1) / tile_rows;
  const uint32_t wmask = (1u << wb) - 1u;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    TileT<NC> t[kScatterIters];
    uint32_t rank[kScatterIters][4];
#pragma unroll
    for (int it = 0; it < kScatterIters; ++it) {
      const int64_t row0 = tile * tile_rows + ((int64_t)warp * kScatterIters + it) * 128 + 4 * lane;
      if (aligned && row0 + 4 <= n) load_tile4_full<true, NC>(keys, vmask, cs, row0, t[it]);
      else load_tile4_tail<true, NC>(keys, vmask, cs, row0, n, t[it]);
    }
#pragma unroll
    for (int it = 0; it < kScatterIters; ++it)
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (t[it].valid & (1u << r)) {
          const uint32_t d = (uint32_t)((int64_t)t[it].key[r] - kmin);
          rank[it][r] = atomicAdd(&s_cnt[d >> wb], 1u);
        }
    __syncthreads();
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
      const uint32_t c = s_cnt[j];
      if (c) {
        s_base[j] = atomicAdd(&cursor[j], c);
        s_cnt[j] = 0u;
      }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kScatterIters; ++it)
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (t[it].valid & (1u << r)) {
          const uint32_t d = (uint32_t)((int64_t)t[it].key[r] - kmin);
          const int64_t pos = (int64_t)s_base[d >> wb] + rank[it][r];
          rec.klow[pos] = (uint16_t)(d & wmask);
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            if (c >= cs.ncols) break;
            if (cs.dtype[c] == NFC_I32) static_cast<int32_t*>(rec.v[c])[pos] = (int32_t)t[it].raw[c][r];
            else static_cast<uint64_t*>(rec.v[c])[pos] = t[it].raw[c][r];
          }
        }
  }
}

template <int NC>
static int launch_scatter(const int32_t* keys, const uint32_t* vmask, const ColSet& cs, int64_t n, bool al,
                          int32_t kmin, int wb, int32_t nb, uint32_t* cursor, const Records& rec, cudaStream_t s) {
  const size_t smem = (size_t)nb * 8;
  NFC_CUDA(cudaFuncSetAttribute(k_part_scatter<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t tile_rows = (kScatterThreads / 32) * kScatterIters * 128;
  int64_t g = std::min<int64_t>((n + tile_rows - 1) / tile_rows, (int64_t)num_sms());
  k_part_scatter<NC><<<(unsigned)std::max<int64_t>(g, 1), kScatterThreads, smem, s>>>(keys, vmask, cs, n, al, kmin,
                                                                                     wb, nb, cursor, rec);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

__global__ void k_merge_init(ColSet cs, StateRef gm, const int32_t* n_merge, int64_t w) {
  const int64_t slots = (int64_t)(*n_merge) * w;
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < slots;
       d += (int64_t)gridDim.x * blockDim.x)
    state_init_slot(cs, gm, d);
}

struct PartAggArgs {
  ColSet cs;
  Records rec;
  const int64_t* offs;
  const int32_t* item_base;
  const int32_t* merge_slot;
  uint32_t* slice_done;
  StateRef gm;  // merge state, n_merge * W slots
  uint64_t* lb;
  uint32_t* ticket;
  OutSet o;
  int64_t kmin, m, slice;
  int32_t nb, wb;
  int64_t* ng_out;
  int32_t* err;
};

NFC_DEV void part_finalize(const PartAggArgs& a, const StateRef& st, int64_t s0, int32_t b, int32_t wbk,
                           uint32_t* s_scan, int64_t* s_base) {
  const int per = (wbk + blockDim.x - 1) / blockDim.x;
  const int g0 = threadIdx.x * per;
  uint32_t c = 0;
  for (int j = 0; j < per; ++j)
    if (g0 + j < wbk && st.cnt[s0 + g0 + j] != 0u) ++c;
  uint32_t total;
  const uint32_t excl = block_excl_scan(c, s_scan, &total);
  if (threadIdx.x == 0) {
    *s_base = lookback_exclusive(a.lb, b, total, a.err);
    if (b == a.nb - 1) *a.ng_out = *s_base + total;
  }
  __syncthreads();
  int64_t pos = *s_base + excl;
  const int64_t key0 = a.kmin + ((int64_t)b << a.wb);
  for (int j = 0; j < per; ++j) {
    const int g = g0 + j;
    if (g < wbk && st.cnt[s0 + g] != 0u) state_emit(a.cs, st, s0 + g, a.o, pos++, key0 + g);
  }
}

__global__ void __launch_bounds__(512) k_part_agg(PartAggArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_base;
  __shared__ int32_t s_item, s_bucket, s_last;
  if (threadIdx.x == 0) {
    s_item = (int32_t)atomicAdd(a.ticket, 1u);
    // Bucket = last b with item_base[b] <= item.
    int lo = 0, hi = a.nb - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.item_base[mid] <= s_item) lo = mid; else hi = mid - 1;
    }
    s_bucket = lo;
  }
  __syncthreads();
  const int32_t item = s_item;
  if (item >= a.item_base[a.nb]) return;
  const int32_t b = s_bucket;
  const int32_t W = 1 << a.wb;
  const int64_t key_off = (int64_t)b << a.wb;
  const int32_t wbk = (int32_t)min((int64_t)W, a.m - key_off);
  const int32_t nslices = a.item_base[b + 1] - a.item_base[b];
  const int32_t sl = item - a.item_base[b];
  const int64_t r_lo = a.offs[b] + (int64_t)sl * a.slice;
  const int64_t r_hi = min(a.offs[b + 1], r_lo + a.slice);

  const StateRef sst = carve_state(a.cs, smem_raw, W);
  for (int g = threadIdx.x; g < wbk; g += blockDim.x) state_init_slot(a.cs, sst, g);
  __syncthreads();
  for (int64_t i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
    const int32_t g = a.rec.klow[i];
    uint64_t raw[NFC_MAX_COLS];
#pragma unroll
    for (int c = 0; c < NFC_MAX_COLS; ++c) {
      raw[c] = 0;
      if (c < a.cs.ncols)
        raw[c] = a.cs.dtype[c] == NFC_I32 ? (uint64_t)(int64_t) static_cast<const int32_t*>(a.rec.v[c])[i]
                                          : static_cast<const uint64_t*>(a.rec.v[c])[i];
    }
    state_apply(a.cs, sst, g, raw);
  }
  __syncthreads();
  if (nslices == 1) {
    part_finalize(a, sst, 0, b, wbk, s_scan, &s_base);
    return;
  }
  const int64_t mslot0 = (int64_t)a.merge_slot[b] * W;
  for (int g = threadIdx.x; g < wbk; g += blockDim.x) state_merge(a.cs, a.gm, mslot0 + g, sst, g);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&a.slice_done[b], 1u) == (uint32_t)(nslices - 1)) ? 1 : 0;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  part_finalize(a, a.gm, mslot0, b, wbk, s_scan, &s_base);
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
              nfc_probe* host_probe, StageTimer* tm) {
  const int64_t n = a->n;
  BitmapSet bms{};
  bms.nbm = 0;
  if (a->key_validity) bms.bm[bms.nbm++] = a->key_validity;
  for (int c = 0; c < a->ncols; ++c)
    if (a->cols[c].validity) bms.bm[bms.nbm++] = a->cols[c].validity;
  uint32_t* vmask = nullptr;
  if (bms.nbm > 0) NFC_CUDA(sc.alloc(&vmask, (size_t)((n + 31) / 32 + 1)));
  const int64_t nspans = (n + kProbeSpan - 1) / kProbeSpan;
  ProbeRec* recs = nullptr;
  nfc_probe* dprobe = nullptr;
  NFC_CUDA(sc.alloc(&recs, (size_t)std::max<int64_t>(nspans, 1)));
  NFC_CUDA(sc.alloc(&dprobe, 1));
  tm->mark(s);
  if (nspans > 0) {
    const int grid = grid_stream((nspans + 7) / 8, 8);
    k_probe<<<grid, 256, 0, s>>>(a->keys, n, bms, vmask, recs, nspans, aligned16(a->keys));
    NFC_CUDA(cudaGetLastError());
    tm->launched();
  }
  k_probe_finalize<<<1, 1024, 0, s>>>(recs, nspans, dprobe);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);
  NFC_CUDA(cudaMemcpyAsync(host_probe, dprobe, sizeof(nfc_probe), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  *vmask_out = vmask;
  return NFC_OK;
}

// Shared-memory budget for one CTA's dense state.
constexpr size_t kSmemStateBudget = 200 * 1024;
constexpr int64_t kMaxBuckets = 16384;
constexpr int64_t kSlice = 65536;

int pick_partition_width(size_t slot_bytes, int64_t m, int* wb_out) {
  int wb = 16;
  while (wb > 8 && ((size_t)1 << wb) * slot_bytes > kSmemStateBudget) --wb;
  if (((size_t)1 << wb) * slot_bytes > kSmemStateBudget) return -1;
  *wb_out = wb;
  const int64_t nb = (m + (1ll << wb) - 1) >> wb;
  return nb <= kMaxBuckets ? 0 : -1;
}

int plan_strategy(const ColSet& cs, const nfc_probe& p) {
  if (p.n_valid == 0) return NFC_STRAT_DENSE_GLOBAL;
  const int64_t m = p.kmax - p.kmin + 1;
  const size_t slot = state_bytes_per_slot(cs);
  // Span that one CTA's shared memory holds (two CTAs per SM).
  if ((size_t)m * slot <= 96 * 1024 && p.n_valid >= 4 * m) return NFC_STRAT_DENSE_SMEM;
  // Span whose global state stays L2-resident.
  if ((size_t)m * slot <= (size_t)24 << 20 && m <= 4 * p.n_valid + 4096) return NFC_STRAT_DENSE_GLOBAL;
  int wb;
  if (m <= 4 * p.n_valid + 65536 && pick_partition_width(slot, m, &wb) == 0) return NFC_STRAT_PARTITION;
  return NFC_STRAT_HASH;
}

static int finish_ng(cudaStream_t s, const int64_t* d_ng, const int32_t* d_err, int64_t* ng, int32_t* status) {
  int64_t h[2] = {0, 0};
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
    const size_t smem = (size_t)m * slot + 64;
    NFC_CUDA(cudaFuncSetAttribute(k_dense_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = grid_stream((ntiles128 + 15) / 16, 2);
    k_dense_smem<<<grid, 512, smem, s>>>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, (int32_t)m, gst);
  } else {
    const int grid = grid_stream((ntiles128 + 7) / 8, 8);
    k_dense_global<<<grid, 256, 0, s>>>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, gst);
  }
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);
  return compact_dense(cs, gst, m, p.kmin, o, s, sc, d_ng, d_err, tm);
}

int run_partition(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
                  const uint32_t* vmask, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err,
                  int64_t* buckets_out, StageTimer* tm) {
  const int64_t m = p.kmax - p.kmin + 1;
  const size_t slot = state_bytes_per_slot(cs);
  int wb = 0;
  if (pick_partition_width(slot, m, &wb) != 0) {
    set_last_error("partition: span %lld too wide", (long long)m);
    return NFC_ERR_UNSUPPORTED;
  }
  const int32_t nb = (int32_t)((m + (1ll << wb) - 1) >> wb);
  *buckets_out = nb;
  const int64_t nv = p.n_valid;
  const bool al = inputs_aligned(a);

  // One scratch block for all the small per-bucket arrays.
  struct {
    uint32_t* ghist; int64_t* offs; uint32_t* cursor; int32_t* item_base; int32_t* merge_slot;
    int32_t* n_merge; uint32_t* slice_done; uint64_t* lb; uint32_t* ticket;
  } w;
  unsigned char* small = nullptr;
  const size_t nbp = (size_t)nb + 1;
  const size_t small_bytes = nbp * (4 + 8 + 4 + 4 + 4 + 4 + 8) + 64;
  NFC_CUDA(sc.alloc(&small, small_bytes));
  NFC_CUDA(cudaMemsetAsync(small, 0, small_bytes, s));
  unsigned char* q = small;
  w.offs = reinterpret_cast<int64_t*>(q); q += 8 * nbp;
  w.lb = reinterpret_cast<uint64_t*>(q); q += 8 * nbp;
  w.ghist = reinterpret_cast<uint32_t*>(q); q += 4 * nbp;
  w.cursor = reinterpret_cast<uint32_t*>(q); q += 4 * nbp;
  w.item_base = reinterpret_cast<int32_t*>(q); q += 4 * nbp;
  w.merge_slot = reinterpret_cast<int32_t*>(q); q += 4 * nbp;
  w.slice_done = reinterpret_cast<uint32_t*>(q); q += 4 * nbp;
  w.n_merge = reinterpret_cast<int32_t*>(q); q += 8;
  w.ticket = reinterpret_cast<uint32_t*>(q); q += 8;

  const int64_t ntiles128 = (a->n + 127) / 128;
  {
    const size_t smem = (size_t)nb * 4;
    NFC_CUDA(cudaFuncSetAttribute(k_part_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_part_hist<<<grid_stream((ntiles128 + 15) / 16, 4), 256, smem, s>>>(a->keys, vmask, a->n, al,
                                                                         (int32_t)p.kmin, wb, nb, w.ghist);
    NFC_CUDA(cudaGetLastError());
  }
  PartPlan pl{w.offs, w.cursor, w.item_base, w.merge_slot, w.n_merge};
  k_part_plan<<<1, 1024, 0, s>>>(w.ghist, nb, kSlice, pl);
  NFC_CUDA(cudaGetLastError());
  tm->launched(2);
  tm->mark(s);

  Records rec{};
  NFC_CUDA(sc.alloc(&rec.klow, (size_t)std::max<int64_t>(nv, 1)));
  for (int c = 0; c < cs.ncols; ++c) {
    unsigned char* vp = nullptr;
    NFC_CUDA(sc.alloc(&vp, (size_t)std::max<int64_t>(nv, 1) * dtype_bytes(cs.dtype[c])));
    rec.v[c] = vp;
  }
  {
    int rc2;
    switch (cs.ncols) {
      case 0: rc2 = launch_scatter<0>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, wb, nb, w.cursor, rec, s); break;
      case 1: rc2 = launch_scatter<1>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, wb, nb, w.cursor, rec, s); break;
      case 2: rc2 = launch_scatter<2>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, wb, nb, w.cursor, rec, s); break;
      case 3: rc2 = launch_scatter<3>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, wb, nb, w.cursor, rec, s); break;
      default: rc2 = launch_scatter<4>(a->keys, vmask, cs, a->n, al, (int32_t)p.kmin, wb, nb, w.cursor, rec, s); break;
    }
    if (rc2) return rc2;
    tm->launched();
    tm->mark(s);
  }
  const int64_t W = 1ll << wb;
  const int64_t max_merge = nv / (kSlice + 1) + 1;
  unsigned char* gmb = nullptr;
  NFC_CUDA(sc.alloc(&gmb, (size_t)max_merge * W * slot + 64));
  const StateRef gm = carve_state(cs, gmb, max_merge * W);
  k_merge_init<<<grid_stream((max_merge * W + 255) / 256, 4), 256, 0, s>>>(cs, gm, w.n_merge, W);
  NFC_CUDA(cudaGetLastError());

  PartAggArgs pa;
  pa.cs = cs;
  pa.rec = rec;
  pa.offs = w.offs;
  pa.item_base = w.item_base;
  pa.merge_slot = w.merge_slot;
  pa.slice_done = w.slice_done;
  pa.gm = gm;
  pa.lb = w.lb;
  pa.ticket = w.ticket;
  pa.o = o;
  pa.kmin = p.kmin;
  pa.m = m;
  pa.slice = kSlice;
  pa.nb = nb;
  pa.wb = wb;
  pa.ng_out = d_ng;
  pa.err = d_err;
  const size_t smem = (size_t)W * slot + 64;
  NFC_CUDA(cudaFuncSetAttribute(k_part_agg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t max_items = nb + nv / kSlice + 1;
  k_part_agg<<<(unsigned)max_items, 512, smem, s>>>(pa);
  NFC_CUDA(cudaGetLastError());
  tm->launched(2);
  tm->mark(s);
  return NFC_OK;
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
  rc = run_probe(a, s, sc, &vmask, &p, &tm);
  if (rc) return rc;
  int strat = strategy == NFC_STRAT_AUTO ? plan_strategy(cs, p) : strategy;
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
  const size_t slot = state_bytes_per_slot(cs);
  if (strat == NFC_STRAT_SORTED) strat = plan_strategy(cs, p) == NFC_STRAT_HASH ? NFC_STRAT_HASH : NFC_STRAT_DENSE_GLOBAL;
  if (strat == NFC_STRAT_DENSE_SMEM && (size_t)m * slot + 64 > kSmemStateBudget) strat = NFC_STRAT_DENSE_GLOBAL;
  switch (strat) {
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
    stats->launches = tm.launches;
    stats->nstages = tm.finish(stats->stage_ms);
  }
  if (status) {
    set_last_error("device status %d", status);
    return status;
  }
  return ng;
}
