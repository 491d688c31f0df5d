// PARTITION strategy: group-by over a wide dense key span.
//
//   1. histogram   rows -> key-range buckets of W = 2^wb keys (bulk-copy
//                  tiles when the keys and the combined bitmap are 16-byte
//                  aligned)
//   2. plan        bucket offsets, work items (buckets larger than one slice
//                  of kSlice records are split), merge slots
//   3. scatter     rows -> packed records in bucket order.  Aligned inputs:
//                  pass 1 sends TMA-staged row tiles to coarse buckets of 64
//                  fine ones, the refine pass splits the coarse buckets into
//                  fine ones; each tile is ranked by bucket in shared memory
//                  and written as contiguous runs, one global reservation per
//                  bucket and tile.  Otherwise one plain scatter pass (two
//                  sweeps per tile: count, reserve, place).
//   4. aggregate   one CTA per work item folds its records into a shared-
//                  memory state of W groups and writes the bucket's present
//                  groups straight to their final, ascending position
//                  (decoupled look-back over buckets).  Split buckets merge
//                  into a global state; the last slice to finish emits.
//
// Record = u64 words.  Columns are ordered so that 4-byte columns come
// first; word 0 = klow | (first column << 32) when that column is 4 bytes
// (PACK0), and every other column takes one word.  (int32 key + int32 value
// + float64 value = 16 bytes per row.)
//
// Shared-memory state avoids emulated 64-bit atomics: an int32 column's sum
// is one signed 32-bit sum when the scatter saw no value outside +-32767,
// else two native 32-bit sums of its low and high 16-bit halves (both exact
// while a slice holds at most 65,536 records); float64 min/max use native
// 64-bit min/max on an order-preserving encoding; float64 sums use the
// 64-bit float add.
#include <algorithm>
#include <type_traits>

#include "agg_smem.cuh"
#include "bulk.cuh"
#include "groupby_host.h"

namespace nfc {

constexpr int kPartThreads = 512;
constexpr int64_t kScatterTile = 16384;  // rows per CTA tile in the scatter

// ---------------------------------------------------------------- histogram
__global__ void __launch_bounds__(256) k_part_hist(const int32_t* __restrict__ keys,
                                                   const uint32_t* __restrict__ vmask, int64_t n, bool aligned,
                                                   int32_t kmin, int wb, int32_t nb, uint32_t* __restrict__ ghist) {
  extern __shared__ uint32_t s_hist[];
  for (int j = threadIdx.x; j < nb; j += blockDim.x) s_hist[j] = 0u;
  __syncthreads();
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (n + 127) >> 7;
  ColSet none{};
  constexpr int U = 8;  // 128-row tiles in flight per warp
  for (int64_t tile0 = gw * U; tile0 < ntiles; tile0 += nw * U) {
    TileT<0> t[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t row0 = (tile0 + u) * 128 + 4 * lane;
      if (aligned && row0 + 4 <= n) load_tile4_full<false, 0>(keys, vmask, none, row0, t[u]);
      else load_tile4_tail<false, 0>(keys, vmask, none, row0, n, t[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (t[u].valid & (1u << r)) atomicAdd(&s_hist[(uint32_t)((int64_t)t[u].key[r] - kmin) >> wb], 1u);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nb; j += blockDim.x)
    if (s_hist[j]) atomicAdd(&ghist[j], s_hist[j]);
}

// Bulk-copy form over full tiles of kHistTile rows (16-byte aligned keys and
// combined bitmap): each CTA streams its tiles through a shared-memory ring
// and counts from shared memory; the rows after the last full tile go
// through k_part_hist.
constexpr int kHistTile = 4096;
constexpr int kHistStages = 4;
constexpr uint32_t kHistStageBytes = kHistTile * 4 + kHistTile / 8;

__global__ void __launch_bounds__(512) k_part_hist_bulk(const int32_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ vmask, int64_t nfull,
                                                        int32_t kmin, int wb, int32_t nb,
                                                        uint32_t* __restrict__ ghist, int32_t* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);  // [kHistStages]
  unsigned char* stage0 = smem_raw + 128;
  uint32_t* s_hist = reinterpret_cast<uint32_t*>(stage0 + (size_t)kHistStages * kHistStageBytes);
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  for (int j = tid; j < nb; j += blockDim.x) s_hist[j] = 0u;
  if (tid == 0) {
    s_abort = 0;
    for (int i = 0; i < kHistStages; ++i) mbar_init(&bars[i], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int64_t my_tiles = nfull > blockIdx.x ? (nfull - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t pol = l2_policy_evict_first();
  const uint32_t tile_bytes = kHistTile * 4 + (vmask ? kHistTile / 8 : 0);
  auto issue = [&](int64_t k) {
    const int st = (int)(k % kHistStages);
    const int64_t row0 = (blockIdx.x + k * (int64_t)gridDim.x) * kHistTile;
    unsigned char* dst = stage0 + (size_t)st * kHistStageBytes;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[st], tile_bytes);
    bulk_g2s_hint(dst, keys + row0, kHistTile * 4, &bars[st], pol);
    if (vmask) bulk_g2s_hint(dst + kHistTile * 4, vmask + (row0 >> 5), kHistTile / 8, &bars[st], pol);
  };
  if (tid == 0)
    for (int64_t k = 0; k < my_tiles && k < kHistStages; ++k) issue(k);
  int64_t k = 0;
  for (; k < my_tiles; ++k) {
    const int st = (int)(k % kHistStages);
    if (!mbar_wait(&bars[st], (uint32_t)((k / kHistStages) & 1))) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    const unsigned char* sp = stage0 + (size_t)st * kHistStageBytes;
#pragma unroll
    for (int j = 0; j < kHistTile / (4 * 512); ++j) {
      const int i0 = j * 2048 + 4 * tid;
      const int4 kv = *reinterpret_cast<const int4*>(sp + 4 * i0);
      const uint32_t valid =
          vmask ? (*reinterpret_cast<const uint32_t*>(sp + kHistTile * 4 + 4 * (i0 >> 5)) >> (i0 & 31)) & 0xFu : 0xFu;
      if (valid & 1u) atomicAdd(&s_hist[(uint32_t)((int64_t)kv.x - kmin) >> wb], 1u);
      if (valid & 2u) atomicAdd(&s_hist[(uint32_t)((int64_t)kv.y - kmin) >> wb], 1u);
      if (valid & 4u) atomicAdd(&s_hist[(uint32_t)((int64_t)kv.z - kmin) >> wb], 1u);
      if (valid & 8u) atomicAdd(&s_hist[(uint32_t)((int64_t)kv.w - kmin) >> wb], 1u);
    }
    __syncthreads();
    if (tid == 0 && k + kHistStages < my_tiles) issue(k + kHistStages);
  }
  if (s_abort) {
    // Let every copy already issued land before the CTA's shared memory goes away.
    if (tid == 0) {
      atomicExch(err, NFC_ERR_TIMEOUT);
      for (int64_t q = k; q < my_tiles && q < k + kHistStages; ++q)
        mbar_wait(&bars[q % kHistStages], (uint32_t)((q / kHistStages) & 1));
    }
    __syncthreads();
    return;
  }
  for (int j = tid; j < nb; j += blockDim.x)
    if (s_hist[j]) atomicAdd(&ghist[j], s_hist[j]);
}

// ---------------------------------------------------------------- plan
struct PartPlan {
  int64_t* offs;        // [nb+1] record offsets
  uint32_t* cursor;     // [nb]   scatter cursors
  int32_t* item_base;   // [nb+1] work-item offsets (slices)
  int32_t* merge_slot;  // [nb]   -1 or merge-state slot
  int32_t* n_merge;     // [1]
  int32_t* item_bucket; // [items] bucket of each work item
};

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
      for (uint32_t i = 0; i < items; ++i) pl.item_bucket[s_carry_item + (int32_t)(e_items + i)] = (int32_t)b;
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

// ---------------------------------------------------------------- records
template <int NC, bool PACK0>
struct Rec {
  static constexpr int NW = NC == 0 ? 1 : NC + 1 - (PACK0 ? 1 : 0);
  // word index of column c (column 0 shares word 0 when packed)
  static constexpr int word(int c) { return PACK0 ? (c == 0 ? 0 : c) : c + 1; }
};

template <int NC, bool PACK0, bool HINT = false>
NFC_DEV void rec_store(uint64_t* __restrict__ dst, uint32_t klow, const uint64_t* raw, uint64_t policy = 0) {
  // (raw[0] of a packed column is a sign-extended int32; only its low 32 bits are kept)
  uint64_t w[Rec<NC, PACK0>::NW];
  w[0] = klow;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (PACK0 && c == 0) w[0] |= (uint64_t)(uint32_t)raw[0] << 32;
    else w[Rec<NC, PACK0>::word(c)] = raw[c];
  }
  constexpr int NW = Rec<NC, PACK0>::NW;
  if (NW % 2 == 0) {
#pragma unroll
    for (int i = 0; i < NW; i += 2) {
      if (HINT) st_v2_u64_hint(dst + i, w[i], w[i + 1], policy);
      else *reinterpret_cast<ulonglong2*>(dst + i) = make_ulonglong2(w[i], w[i + 1]);
    }
  } else {
#pragma unroll
    for (int i = 0; i < NW; ++i) {
      if (HINT) st_u64_hint(dst + i, w[i], policy);
      else dst[i] = w[i];
    }
  }
}

// Bit c set when int32 column c holds a value outside [-32767, 32767]: the
// aggregate then keeps that column's sum as two 16-bit-half sums instead of
// one signed 32-bit sum.
template <int NC, uint32_t SIG>
NFC_DEV uint32_t wide_bits(const ColSet& cs, const uint64_t* raw) {
  uint32_t w = 0;
#pragma unroll
  for (int c = 0; c < NC; ++c)
    if (col_dt<SIG>(cs, c) == NFC_I32 && (uint32_t)raw[c] + 32767u > 65534u) w |= 1u << c;
  return w;
}

// Fold one thread's wide bits into the call's word (one atomic per warp, and
// only when a bit is set).
NFC_DEV void publish_wide(uint32_t w, uint32_t* gwide) {
  w = __reduce_or_sync(0xffffffffu, w);
  if (lane_id() == 0 && w) atomicOr(gwide, w);
}

// ---------------------------------------------------------------- scatter
template <int NC, bool PACK0, uint32_t SIG>
__global__ void __launch_bounds__(kPartThreads, 2) k_part_scatter(const int32_t* __restrict__ keys,
                                                                 const uint32_t* __restrict__ vmask, ColSet cs,
                                                                 int64_t n, bool aligned, int32_t kmin, int wb,
                                                                 int32_t nb, uint32_t* __restrict__ cursor,
                                                                 uint64_t* __restrict__ rec, uint32_t* gwide) {
  extern __shared__ uint32_t s_part[];
  uint32_t wide = 0;
  uint32_t* s_cnt = s_part;
  uint32_t* s_cur = s_part + nb;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) s_cnt[j] = 0u;
  __syncthreads();
  const int lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int64_t ntiles = (n + kScatterTile - 1) / kScatterTile;
  const uint32_t wmask = (1u << wb) - 1u;
  constexpr int NW = Rec<NC, PACK0>::NW;
  constexpr int U1 = 4;  // 128-row groups in flight per warp, sweep 1
  constexpr int U2 = 2;  // ... sweep 2
  ColSet none{};
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t tbase = tile * kScatterTile;
    // Sweep 1: count rows per bucket (keys stay in L2 for sweep 2).
    for (int wt = warp * U1; wt < kScatterTile / 128; wt += nwarps * U1) {
      TileT<0> t[U1];
#pragma unroll
      for (int u = 0; u < U1; ++u) {
        const int64_t row0 = tbase + (int64_t)(wt + u) * 128 + 4 * lane;
        if (aligned && row0 + 4 <= n) {
          const int4 kv = __ldg(reinterpret_cast<const int4*>(keys + row0));
          t[u].key[0] = kv.x; t[u].key[1] = kv.y; t[u].key[2] = kv.z; t[u].key[3] = kv.w;
          t[u].valid = vmask ? (__ldg(vmask + (row0 >> 5)) >> (row0 & 31)) & 0xFu : 0xFu;
        } else {
          load_tile4_tail<false, 0>(keys, vmask, none, row0, n, t[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < U1; ++u)
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (t[u].valid & (1u << r)) atomicAdd(&s_cnt[(uint32_t)((int64_t)t[u].key[r] - kmin) >> wb], 1u);
    }
    __syncthreads();
    // Reserve each bucket's range for this tile with one global atomic.
    for (int j0 = threadIdx.x; j0 < nb; j0 += 4 * blockDim.x) {
      uint32_t c[4], base[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int j = j0 + u * blockDim.x;
        c[u] = j < nb ? s_cnt[j] : 0u;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c[u]) base[u] = atomicAdd(&cursor[j0 + u * blockDim.x], c[u]);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c[u]) {
          s_cur[j0 + u * blockDim.x] = base[u];
          s_cnt[j0 + u * blockDim.x] = 0u;
        }
    }
    __syncthreads();
    // Sweep 2: place every valid row.
    for (int wt = warp * U2; wt < kScatterTile / 128; wt += nwarps * U2) {
      TileT<NC> t[U2];
#pragma unroll
      for (int u = 0; u < U2; ++u) {
        const int64_t row0 = tbase + (int64_t)(wt + u) * 128 + 4 * lane;
        if (aligned && row0 + 4 <= n) load_tile4_full<true, NC, SIG>(keys, vmask, cs, row0, t[u]);
        else load_tile4_tail<true, NC, SIG>(keys, vmask, cs, row0, n, t[u]);
      }
      // All positions first (independent shared atomics in flight), then stores.
      uint32_t pos[U2][4];
#pragma unroll
      for (int u = 0; u < U2; ++u)
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (t[u].valid & (1u << r))
            pos[u][r] = atomicAdd(&s_cur[(uint32_t)((int64_t)t[u].key[r] - kmin) >> wb], 1u);
#pragma unroll
      for (int u = 0; u < U2; ++u)
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (t[u].valid & (1u << r)) {
            const uint32_t d = (uint32_t)((int64_t)t[u].key[r] - kmin);
            uint64_t raw[NC > 0 ? NC : 1];
#pragma unroll
            for (int c = 0; c < NC; ++c) raw[c] = t[u].raw[c][r];
            wide |= wide_bits<NC, SIG>(cs, raw);
            rec_store<NC, PACK0>(rec + (size_t)pos[u][r] * NW, d & wmask, raw);
          }
    }
    __syncthreads();
  }
  publish_wide(wide, gwide);
}

// ---------------------------------------------------------------- coalesced two-level scatter
// Scattered 16-byte stores are limited by the number of store requests, not
// by bytes, so both scatter passes sort each tile by destination bucket in
// shared memory and write the tile out in contiguous runs.  To keep runs
// long the fan-out per pass stays <= 256: pass 1 sends rows to coarse
// buckets (64 fine buckets each), pass 2 splits every coarse bucket into its
// fine buckets.  Spans of at most 128 fine buckets need pass 1 only.
// Each pass reserves a tile's range of a bucket with one global atomic.
constexpr int kBulkTile = 2048;     // pass-1 rows per tile (TMA-staged)
constexpr int kCoarseShift = 6;     // 64 fine buckets per coarse bucket
constexpr int kMaxPassBins = 256;

struct BulkLayout {
  uint32_t stage_bytes;
  uint32_t off_vmask;
  uint32_t off_col[NFC_MAX_COLS];
  uint32_t bytes_keys, bytes_vmask, bytes_col[NFC_MAX_COLS];
  int32_t stages;
};

// Dynamic shared memory of pass 1: barriers, stages, the tile's index
// permutation (u16) and bucket bytes, three per-bucket tables.
inline size_t pass1_smem(const BulkLayout& L) {
  return 128 + (size_t)L.stages * L.stage_bytes + (size_t)kBulkTile * 3 + 3 * kMaxPassBins * 4;
}
constexpr size_t kPass1SmemPerSm = 226 * 1024;   // two CTAs per SM (1 KB reserved per CTA)
constexpr size_t kPass1SmemPerCta = 227 * 1024;

// Block-wide scan of the per-tile bucket counts (nbins <= kMaxPassBins) and
// the tile's reservation in each bucket (one global atomic per non-empty bucket).
NFC_DEV uint32_t tile_reserve(const uint32_t* s_cnt, uint32_t* s_start, uint32_t* s_gbase, int nbins,
                              uint32_t* __restrict__ gcursor, uint32_t* s_scan) {
  const int tid = threadIdx.x;
  const uint32_t c = tid < nbins ? s_cnt[tid] : 0u;
  uint32_t total;
  const uint32_t e = block_excl_scan(c, s_scan, &total);
  if (tid < nbins) {
    s_start[tid] = e;
    if (c) s_gbase[tid] = atomicAdd(&gcursor[tid], c);
  }
  return total;
}

// Pass 1: full tiles of kBulkTile rows, TMA-staged through a ring of
// L.stages copies.  Each tile is ranked by bucket in shared memory as an
// index permutation (no copy of the rows), reserves one range per bucket
// with one global atomic, and writes each bucket's records as a contiguous
// run, assembling every record from the staged columns.  Record word 0
// holds d = key - kmin (bits kept per keep_mask) and the packed first int32
// column.  Bucket of a row = d >> shift.
template <int NC, bool PACK0, uint32_t SIG>
__global__ void __launch_bounds__(kPartThreads, 2) k_part_pass1(const int32_t* __restrict__ keys,
                                                               const uint32_t* __restrict__ vmask, ColSet cs,
                                                               BulkLayout L, int64_t nfull, int32_t kmin, int shift,
                                                               int nbins, uint32_t keep_mask,
                                                               uint32_t* __restrict__ gcursor,
                                                               uint64_t* __restrict__ out, int32_t* err,
                                                               uint32_t* gwide) {
  constexpr int NW = Rec<NC, PACK0>::NW;
  constexpr int kIter = kBulkTile / (4 * kPartThreads);
  uint32_t wide = 0;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);  // [stages]
  unsigned char* stage0 = smem_raw + 128;
  uint16_t* sidx = reinterpret_cast<uint16_t*>(stage0 + (size_t)L.stages * L.stage_bytes);
  uint8_t* sbin = reinterpret_cast<uint8_t*>(sidx + kBulkTile);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(sbin + kBulkTile);
  uint32_t* s_start = s_cnt + kMaxPassBins;
  uint32_t* s_gbase = s_start + kMaxPassBins;
  __shared__ uint32_t s_scan[33];
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  if (tid < kMaxPassBins) s_cnt[tid] = 0u;
  if (tid == 0) {
    s_abort = 0;
    for (int i = 0; i < L.stages; ++i) mbar_init(&bars[i], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int64_t my_tiles = nfull > blockIdx.x ? (nfull - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t pol_in = l2_policy_evict_first();
  auto issue = [&](int64_t k) {
    const int st = (int)(k % L.stages);
    const int64_t tile = blockIdx.x + k * (int64_t)gridDim.x;
    unsigned char* dst = stage0 + (size_t)st * L.stage_bytes;
    const int64_t row0 = tile * kBulkTile;
    uint32_t total = L.bytes_keys + (vmask ? L.bytes_vmask : 0u);
#pragma unroll
    for (int c = 0; c < NC; ++c) total += L.bytes_col[c];
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[st], total);
    bulk_g2s_hint(dst, keys + row0, L.bytes_keys, &bars[st], pol_in);
    if (vmask) bulk_g2s_hint(dst + L.off_vmask, vmask + (row0 >> 5), L.bytes_vmask, &bars[st], pol_in);
#pragma unroll
    for (int c = 0; c < NC; ++c)
      bulk_g2s_hint(dst + L.off_col[c],
                    static_cast<const unsigned char*>(cs.data[c]) + (size_t)row0 * (L.bytes_col[c] / kBulkTile),
                    L.bytes_col[c], &bars[st], pol_in);
  };
  if (tid == 0)
    for (int64_t k = 0; k < my_tiles && k < L.stages; ++k) issue(k);
  int64_t k = 0;
  for (; k < my_tiles; ++k) {
    const int st = (int)(k % L.stages);
    if (!mbar_wait(&bars[st], (uint32_t)((k / L.stages) & 1))) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    const unsigned char* sp = stage0 + (size_t)st * L.stage_bytes;
    const int32_t* sk = reinterpret_cast<const int32_t*>(sp);
    const uint32_t* sv = reinterpret_cast<const uint32_t*>(sp + L.off_vmask);
    uint32_t bin[kIter][4], rank[kIter][4], valid[kIter];
#pragma unroll
    for (int j = 0; j < kIter; ++j) {
      const int i0 = j * (4 * kPartThreads) + 4 * tid;
      const int4 kv = *reinterpret_cast<const int4*>(sk + i0);
      bin[j][0] = (uint32_t)((int64_t)kv.x - kmin) >> shift; bin[j][1] = (uint32_t)((int64_t)kv.y - kmin) >> shift;
      bin[j][2] = (uint32_t)((int64_t)kv.z - kmin) >> shift; bin[j][3] = (uint32_t)((int64_t)kv.w - kmin) >> shift;
      valid[j] = vmask ? (sv[i0 >> 5] >> (i0 & 31)) & 0xFu : 0xFu;
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (valid[j] & (1u << r)) rank[j][r] = atomicAdd(&s_cnt[bin[j][r]], 1u);
    }
    __syncthreads();
    const uint32_t nvalid = tile_reserve(s_cnt, s_start, s_gbase, nbins, gcursor, s_scan);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kIter; ++j) {
      const int i0 = j * (4 * kPartThreads) + 4 * tid;
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (valid[j] & (1u << r)) {
          const uint32_t p = s_start[bin[j][r]] + rank[j][r];
          sidx[p] = (uint16_t)(i0 + r);
          sbin[p] = (uint8_t)bin[j][r];
        }
    }
    __syncthreads();
    for (int p = tid; p < (int)nvalid; p += kPartThreads) {
      const int i = sidx[p];
      const int b = sbin[p];
      const size_t gp = (size_t)(s_gbase[b] + (uint32_t)(p - s_start[b])) * NW;
      uint64_t rv[NC > 0 ? NC : 1];
#pragma unroll
      for (int c = 0; c < NC; ++c)
        rv[c] = col_dt<SIG>(cs, c) == NFC_I32
                    ? (uint64_t)(int64_t) reinterpret_cast<const int32_t*>(sp + L.off_col[c])[i]
                    : reinterpret_cast<const uint64_t*>(sp + L.off_col[c])[i];
      wide |= wide_bits<NC, SIG>(cs, rv);
      rec_store<NC, PACK0>(out + gp, (uint32_t)((int64_t)sk[i] - kmin) & keep_mask, rv);
    }
    if (tid < kMaxPassBins) s_cnt[tid] = 0u;
    __syncthreads();
    if (tid == 0 && k + L.stages < my_tiles) issue(k + L.stages);
  }
  if (s_abort) {
    // Let every copy already issued land before the CTA's shared memory goes away.
    if (tid == 0) {
      atomicExch(err, NFC_ERR_TIMEOUT);
      for (int64_t q = k; q < my_tiles && q < k + L.stages; ++q)
        mbar_wait(&bars[q % L.stages], (uint32_t)((q / L.stages) & 1));
    }
    __syncthreads();
  }
  publish_wide(wide, gwide);
}

// Pass 1 for the rows after the last full tile (fewer than kBulkTile).
template <int NC, bool PACK0, uint32_t SIG>
__global__ void __launch_bounds__(kPartThreads) k_part_pass1_tail(const int32_t* __restrict__ keys,
                                                                 const uint32_t* __restrict__ vmask, ColSet cs,
                                                                 int64_t row_off, int64_t n, int32_t kmin, int shift,
                                                                 uint32_t keep_mask, uint32_t* __restrict__ gcursor,
                                                                 uint64_t* __restrict__ out, uint32_t* gwide) {
  constexpr int NW = Rec<NC, PACK0>::NW;
  uint32_t wide = 0;
  for (int64_t i = row_off + threadIdx.x; i < n; i += blockDim.x) {
    if (vmask && !((vmask[i >> 5] >> (i & 31)) & 1u)) continue;
    const uint32_t d = (uint32_t)((int64_t)keys[i] - kmin);
    const uint32_t pos = atomicAdd(&gcursor[d >> shift], 1u);
    uint64_t rv[NC > 0 ? NC : 1];
#pragma unroll
    for (int c = 0; c < NC; ++c)
      rv[c] = col_dt<SIG>(cs, c) == NFC_I32 ? (uint64_t)(int64_t) static_cast<const int32_t*>(cs.data[c])[i]
                                            : static_cast<const uint64_t*>(cs.data[c])[i];
    wide |= wide_bits<NC, SIG>(cs, rv);
    rec_store<NC, PACK0>(out + (size_t)pos * NW, d & keep_mask, rv);
  }
  publish_wide(wide, gwide);
}

// Pass-1 cursors and offsets of the coarse buckets (64 fine buckets each)
// from the fine offsets.
__global__ void k_part_plan2(const int64_t* offs, int32_t nb, int32_t nc, uint32_t* ccursor, int64_t* coffs) {
  for (int32_t c = threadIdx.x; c <= nc; c += blockDim.x) {
    const int64_t lo = offs[min((int64_t)c << kCoarseShift, (int64_t)nb)];
    coffs[c] = lo;
    if (c < nc) ccursor[c] = (uint32_t)lo;
  }
}

// Pass 2, persistent form: the pass-1 output is cut into fixed tiles of
// refine2_tile<NW>() records that stream into shared memory through a ring
// of bulk-copy stages (the next tiles are in flight while one is split).
// Pass 1 leaves the records in coarse-bucket order and a coarse bucket
// covers 64 fine buckets, so a tile that touches at most four coarse
// buckets spans at most 256 fine buckets: it is ranked by fine bucket in
// shared memory (an index permutation, not a copy of the records), reserves
// one range per fine bucket with one global atomic and writes each bucket's
// records as a contiguous run.  A tile spanning more fine buckets (only when
// coarse buckets hold a few records each) reserves one slot per record.
template <int NW>
constexpr int refine2_tile() { return NW <= 1 ? 4096 : NW <= 2 ? 2048 : 1024; }
constexpr int kRefineStages = 3;

template <int NW>
constexpr size_t refine2_smem() {
  return 128 + (size_t)kRefineStages * refine2_tile<NW>() * NW * 8 + (size_t)refine2_tile<NW>() * 3 +
         3 * kMaxPassBins * 4;
}

template <int NW>
__global__ void __launch_bounds__(kPartThreads, 2) k_part_refine(const uint64_t* __restrict__ in, int64_t nv, int wb,
                                                                uint32_t* __restrict__ fcursor,
                                                                uint64_t* __restrict__ out, int32_t* err) {
  constexpr int T = refine2_tile<NW>();
  constexpr int PER = T / kPartThreads;
  constexpr uint32_t kStageBytes = (uint32_t)T * NW * 8;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);  // [kRefineStages]
  unsigned char* stage0 = smem_raw + 128;
  uint16_t* sidx = reinterpret_cast<uint16_t*>(stage0 + (size_t)kRefineStages * kStageBytes);
  uint8_t* sbin = reinterpret_cast<uint8_t*>(sidx + T);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(sbin + T);
  uint32_t* s_start = s_cnt + kMaxPassBins;
  uint32_t* s_gbase = s_start + kMaxPassBins;
  __shared__ uint32_t s_scan[33];
  __shared__ uint32_t s_lo, s_hi;
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  const uint32_t keep = (1u << wb) - 1u;
  if (tid < kMaxPassBins) s_cnt[tid] = 0u;
  if (tid == 0) {
    s_abort = 0;
    s_lo = 0xFFFFFFFFu;
    s_hi = 0u;
    for (int i = 0; i < kRefineStages; ++i) mbar_init(&bars[i], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int64_t ntiles = (nv + T - 1) / T;
  const int64_t my_tiles = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t pol_in = l2_policy_evict_first();
  auto issue = [&](int64_t k) {
    const int st = (int)(k % kRefineStages);
    const int64_t r0 = (blockIdx.x + k * (int64_t)gridDim.x) * T;
    const int64_t nrec = min((int64_t)T, nv - r0);
    // Rounded up to 16 bytes: the buffer carries two spare words past nv.
    const uint32_t bytes = ((uint32_t)nrec * NW * 8 + 15u) & ~15u;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[st], bytes);
    bulk_g2s_hint(stage0 + (size_t)st * kStageBytes, in + (size_t)r0 * NW, bytes, &bars[st], pol_in);
  };
  if (tid == 0)
    for (int64_t k = 0; k < my_tiles && k < kRefineStages; ++k) issue(k);
  int64_t k = 0;
  for (; k < my_tiles; ++k) {
    const int st = (int)(k % kRefineStages);
    const int64_t r0 = (blockIdx.x + k * (int64_t)gridDim.x) * T;
    const int nrec = (int)min((int64_t)T, nv - r0);
    if (!mbar_wait(&bars[st], (uint32_t)((k / kRefineStages) & 1))) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    const uint64_t* sr = reinterpret_cast<const uint64_t*>(stage0 + (size_t)st * kStageBytes);
    uint32_t fb[PER];
    uint32_t lo = 0xFFFFFFFFu, hi = 0u;
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int i = u * kPartThreads + tid;
      fb[u] = i < nrec ? (uint32_t)sr[(size_t)i * NW] >> wb : 0u;
      if (i < nrec) { lo = min(lo, fb[u]); hi = max(hi, fb[u]); }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane_id() == 0 && lo <= hi) {
      atomicMin(&s_lo, lo);
      atomicMax(&s_hi, hi);
    }
    __syncthreads();
    const uint32_t tlo = s_lo, thi = s_hi;
    if (thi - tlo < (uint32_t)kMaxPassBins) {
      uint32_t rank[PER];
#pragma unroll
      for (int u = 0; u < PER; ++u)
        if (u * kPartThreads + tid < nrec) rank[u] = atomicAdd(&s_cnt[fb[u] - tlo], 1u);
      __syncthreads();
      tile_reserve(s_cnt, s_start, s_gbase, (int)(thi - tlo + 1), fcursor + tlo, s_scan);
      __syncthreads();
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const int i = u * kPartThreads + tid;
        if (i < nrec) {
          const uint32_t bin = fb[u] - tlo;
          const uint32_t p = s_start[bin] + rank[u];
          sidx[p] = (uint16_t)i;
          sbin[p] = (uint8_t)bin;
        }
      }
      __syncthreads();
      for (int p = tid; p < nrec; p += kPartThreads) {
        const int i = sidx[p];
        const int bin = sbin[p];
        const size_t gp = (size_t)(s_gbase[bin] + (uint32_t)(p - s_start[bin])) * NW;
        uint64_t w[NW];
#pragma unroll
        for (int q = 0; q < NW; ++q) w[q] = sr[(size_t)i * NW + q];
        w[0] = (w[0] & 0xFFFFFFFF00000000ull) | ((uint32_t)w[0] & keep);
        if (NW % 2 == 0) {
#pragma unroll
          for (int q = 0; q < NW; q += 2)
            *reinterpret_cast<ulonglong2*>(out + gp + q) = make_ulonglong2(w[q], w[q + 1]);
        } else {
#pragma unroll
          for (int q = 0; q < NW; ++q) out[gp + q] = w[q];
        }
      }
    } else {
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const int i = u * kPartThreads + tid;
        if (i < nrec) {
          const size_t gp = (size_t)atomicAdd(&fcursor[fb[u]], 1u) * NW;
          uint64_t w[NW];
#pragma unroll
          for (int q = 0; q < NW; ++q) w[q] = sr[(size_t)i * NW + q];
          w[0] = (w[0] & 0xFFFFFFFF00000000ull) | ((uint32_t)w[0] & keep);
#pragma unroll
          for (int q = 0; q < NW; ++q) out[gp + q] = w[q];
        }
      }
      __syncthreads();  // every thread has read s_lo / s_hi before they are reset
    }
    if (tid < kMaxPassBins) s_cnt[tid] = 0u;
    if (tid == 0) {
      s_lo = 0xFFFFFFFFu;
      s_hi = 0u;
    }
    __syncthreads();
    if (tid == 0 && k + kRefineStages < my_tiles) issue(k + kRefineStages);
  }
  if (s_abort) {
    // Let every copy already issued land before the CTA's shared memory goes away.
    if (tid == 0) {
      atomicExch(err, NFC_ERR_TIMEOUT);
      for (int64_t q = k; q < my_tiles && q < k + kRefineStages; ++q)
        mbar_wait(&bars[q % kRefineStages], (uint32_t)((q / kRefineStages) & 1));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- aggregate
struct PartAggArgs {
  ColSet cs;
  const uint64_t* rec;
  const int64_t* offs;
  const int32_t* item_base;
  const int32_t* item_bucket;
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
  const uint32_t* wide;  // bit c: int32 column c has a value outside [-32767, 32767]
};

// Emit the present groups (count > 0) of bucket b in ascending key order.
// Pass 1 counts them and places the bucket after its predecessors (decoupled
// look-back); pass 2 walks the groups in rounds of blockDim, so consecutive
// threads write consecutive output rows.
template <int NC, uint32_t SIG, class CountF, class EmitF>
NFC_DEV void part_emit(const PartAggArgs& a, int32_t b, int32_t wbk, int64_t key0, CountF cnt_of, EmitF emit,
                       uint32_t* s_scan, int64_t* s_base) {
  uint32_t c = 0;
  for (int g = threadIdx.x; g < wbk; g += blockDim.x) c += cnt_of(g) != 0u ? 1u : 0u;
  uint32_t total;
  block_excl_scan(c, s_scan, &total);
  if (threadIdx.x < 32) {
    const int64_t lbx = lookback_exclusive(a.lb, b, total, a.err);  // whole warp
    if (threadIdx.x == 0) {
      *s_base = lbx;
      if (b == a.nb - 1) *a.ng_out = *s_base + total;
    }
  }
  __syncthreads();
  int64_t base = *s_base;
  for (int g0 = 0; g0 < wbk; g0 += blockDim.x) {
    const int g = g0 + threadIdx.x;
    const uint32_t pres = (g < wbk && cnt_of(g) != 0u) ? 1u : 0u;
    uint32_t round_total;
    const uint32_t excl = block_excl_scan(pres, s_scan, &round_total);
    if (pres) emit(g, base + excl);
    base += round_total;
  }
}

template <int NC, bool PACK0, uint32_t SIG>
__global__ void __launch_bounds__(kPartThreads, 2) k_part_agg(PartAggArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_base;
  __shared__ int32_t s_item, s_bucket, s_last;
  if (threadIdx.x == 0) {
    const int32_t it = (int32_t)atomicAdd(a.ticket, 1u);
    s_item = it;
    s_bucket = it < a.item_base[a.nb] ? a.item_bucket[it] : -1;
  }
  __syncthreads();
  const int32_t item = s_item;
  if (s_bucket < 0) return;
  const int32_t b = s_bucket;
  const int32_t W = 1 << a.wb;
  const int64_t key0 = a.kmin + ((int64_t)b << a.wb);
  const int32_t wbk = (int32_t)min((int64_t)W, a.m - ((int64_t)b << a.wb));
  const int32_t nslices = a.item_base[b + 1] - a.item_base[b];
  const int32_t sl = item - a.item_base[b];
  const int64_t r_lo = a.offs[b] + (int64_t)sl * a.slice;
  const int64_t r_hi = min(a.offs[b + 1], r_lo + a.slice);
  constexpr int NW = Rec<NC, PACK0>::NW;
  constexpr int U = 4;  // records in flight per thread

  const AggState<NC> st = carve_agg<NC, SIG>(a.cs, smem_raw, W, ~__ldg(a.wide));
  for (int g = threadIdx.x; g < wbk; g += blockDim.x) agg_init<NC, SIG>(a.cs, st, g);
  __syncthreads();
  const uint64_t* rp = a.rec + (size_t)r_lo * NW;
  const int64_t nrec = r_hi - r_lo;
  for (int64_t i0 = threadIdx.x; i0 < nrec; i0 += (int64_t)U * blockDim.x) {
    uint64_t w[U][NW];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + (int64_t)u * blockDim.x;
      if (i < nrec) {
        if (NW % 2 == 0) {
#pragma unroll
          for (int j = 0; j < NW; j += 2) {
            const ulonglong2 q = __ldcs(reinterpret_cast<const ulonglong2*>(rp + i * NW + j));
            w[u][j] = q.x;
            w[u][j + 1] = q.y;
          }
        } else {
#pragma unroll
          for (int j = 0; j < NW; ++j) w[u][j] = __ldcs(rp + i * NW + j);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (i0 + (int64_t)u * blockDim.x < nrec) {
        uint64_t raw[NC > 0 ? NC : 1];
#pragma unroll
        for (int c = 0; c < NC; ++c) raw[c] = (PACK0 && c == 0) ? (w[u][0] >> 32) : w[u][Rec<NC, PACK0>::word(c)];
        agg_apply<NC, SIG, false>(a.cs, st, (uint32_t)w[u][0], raw);
      }
    }
  }
  __syncthreads();
  if (nslices == 1) {
    part_emit<NC, SIG>(a, b, wbk, key0, [&](int g) { return st.cnt[g]; },
                       [&](int g, int64_t pos) { agg_emit<NC, SIG>(a.cs, st, g, a.o, pos, key0 + g); }, s_scan,
                       &s_base);
    return;
  }
  const int64_t m0 = (int64_t)a.merge_slot[b] * W;
  for (int g = threadIdx.x; g < wbk; g += blockDim.x) agg_merge<NC, SIG>(a.cs, a.gm, m0 + g, st, g);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&a.slice_done[b], 1u) == (uint32_t)(nslices - 1)) ? 1 : 0;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  part_emit<NC, SIG>(a, b, wbk, key0, [&](int g) { return __ldcg(&a.gm.cnt[m0 + g]); },
                     [&](int g, int64_t pos) { state_emit(a.cs, a.gm, m0 + g, a.o, pos, key0 + g); }, s_scan,
                     &s_base);
}

__global__ void k_merge_init(ColSet cs, StateRef gm, const int32_t* n_merge, int64_t w) {
  const int64_t slots = (int64_t)(*n_merge) * w;
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < slots; d += (int64_t)gridDim.x * blockDim.x)
    state_init_slot(cs, gm, d);
}

// ---------------------------------------------------------------- host
constexpr int64_t kMaxBuckets = 16384;
constexpr int64_t kSlice = 65536;  // <= 65536 keeps the 16-bit-split int32 sums exact
constexpr size_t kAggSmemBudget = 200 * 1024;

// Bucket width: the widest whose shared-memory state leaves room for two
// aggregate CTAs per SM (twice the warps to hide shared-atomic latency); if
// that needs more than kMaxBuckets buckets, the widest one CTA can hold.
constexpr size_t kAggSmemBudget2 = 110 * 1024;
int pick_partition_width(size_t slot_bytes, int64_t m, int* wb_out) {
  for (const size_t budget : {kAggSmemBudget2, kAggSmemBudget}) {
    int wb = 16;
    while (wb > 8 && ((size_t)1 << wb) * slot_bytes > budget) --wb;
    if (((size_t)1 << wb) * slot_bytes > budget) continue;
    const int64_t nb = (m + (1ll << wb) - 1) >> wb;
    if (nb <= kMaxBuckets) {
      *wb_out = wb;
      return 0;
    }
  }
  return -1;
}

struct PartLaunch {
  const nfc_groupby_args* a;
  ColSet cs;
  const uint32_t* vmask;
  bool al;
  int32_t kmin;
  int wb;
  int32_t nb;
  bool coalesced;     // two-level coalesced scatter (else the plain one-pass scatter)
  BulkLayout L;
  int64_t nfull;
  int32_t nc;         // coarse buckets (== nb when one level suffices)
  bool two_level;
  uint32_t* ccursor;  // coarse cursors [nc]
  int64_t* coffs;     // [nc+1]
  uint32_t* cursor;   // fine cursors [nb]
  uint64_t* rec_a;    // pass-1 output (two-level)
  uint64_t* rec;      // fine-bucket records (aggregate input)
  size_t agg_smem;
  int64_t max_items;
  int64_t nv;         // valid rows (records)
  uint32_t* wide;     // wide-int32-column bits (zeroed, set by the scatter)
  int32_t* d_err;
};

template <int NC, bool PACK0, uint32_t SIG>
static int launch_part(const PartLaunch& q, PartAggArgs& pa, cudaStream_t s, StageTimer* tm) {
  const nfc_groupby_args* a = q.a;
  constexpr int NW = Rec<NC, PACK0>::NW;
  if (q.coalesced) {
    const int shift = q.two_level ? q.wb + kCoarseShift : q.wb;
    const uint32_t keep = q.two_level ? 0xFFFFFFFFu : (1u << q.wb) - 1u;
    uint32_t* cur1 = q.two_level ? q.ccursor : q.cursor;
    uint64_t* out1 = q.two_level ? q.rec_a : q.rec;
    if (q.nfull > 0) {
      const size_t smem = pass1_smem(q.L);
      NFC_CUDA(cudaFuncSetAttribute(k_part_pass1<NC, PACK0, SIG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
      const int per_sm = 2 * smem <= kPass1SmemPerSm ? 2 : 1;
      const int64_t g = std::max<int64_t>(1, std::min<int64_t>(q.nfull, (int64_t)num_sms() * per_sm));
      k_part_pass1<NC, PACK0, SIG><<<(unsigned)g, kPartThreads, smem, s>>>(a->keys, q.vmask, q.cs, q.L, q.nfull,
                                                                          q.kmin, shift, q.nc, keep, cur1, out1,
                                                                          q.d_err, q.wide);
      NFC_CUDA(cudaGetLastError());
      tm->launched();
    }
    const int64_t row_off = q.nfull * kBulkTile;
    if (a->n > row_off) {
      k_part_pass1_tail<NC, PACK0, SIG><<<1, kPartThreads, 0, s>>>(a->keys, q.vmask, q.cs, row_off, a->n, q.kmin,
                                                                   shift, keep, cur1, out1, q.wide);
      NFC_CUDA(cudaGetLastError());
      tm->launched();
    }
    if (q.two_level) {
      constexpr size_t smem2 = refine2_smem<NW>();
      NFC_CUDA(cudaFuncSetAttribute(k_part_refine<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
      const int64_t nt2 = (q.nv + refine2_tile<NW>() - 1) / refine2_tile<NW>();
      const int64_t g2 = std::max<int64_t>(1, std::min<int64_t>(nt2, (int64_t)num_sms() * 2));
      k_part_refine<NW><<<(unsigned)g2, kPartThreads, smem2, s>>>(q.rec_a, q.nv, q.wb, q.cursor, q.rec, q.d_err);
      NFC_CUDA(cudaGetLastError());
      tm->launched();
    }
  } else {
    const size_t smem = (size_t)q.nb * 8;
    NFC_CUDA(cudaFuncSetAttribute(k_part_scatter<NC, PACK0, SIG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    const int64_t ntiles = (a->n + kScatterTile - 1) / kScatterTile;
    const int64_t g = std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)num_sms() * 2));
    k_part_scatter<NC, PACK0, SIG><<<(unsigned)g, kPartThreads, smem, s>>>(a->keys, q.vmask, q.cs, a->n, q.al,
                                                                          q.kmin, q.wb, q.nb, q.cursor, q.rec,
                                                                          q.wide);
    NFC_CUDA(cudaGetLastError());
    tm->launched();
  }
  tm->mark(s);
  NFC_CUDA(cudaFuncSetAttribute(k_part_agg<NC, PACK0, SIG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)q.agg_smem));
  k_part_agg<NC, PACK0, SIG><<<(unsigned)q.max_items, kPartThreads, q.agg_smem, s>>>(pa);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  return NFC_OK;
}

// Column signatures with a dedicated instantiation (after 4-byte-first ordering).
constexpr uint32_t kSigI32SumMinMax_F64SumMinMax =
    sig_col(0, NFC_I32, NFC_AGG_SUM | NFC_AGG_MIN | NFC_AGG_MAX) | sig_col(1, NFC_F64, NFC_AGG_SUM | NFC_AGG_MIN | NFC_AGG_MAX);
constexpr uint32_t kSigI32Sum = sig_col(0, NFC_I32, NFC_AGG_SUM);

template <int NC>
static int launch_part_nc(bool pack0, const PartLaunch& q, PartAggArgs& pa, cudaStream_t s, StageTimer* tm) {
  const uint32_t sig = sig_of(q.cs);
  if constexpr (NC == 2) {
    if (pack0 && sig == kSigI32SumMinMax_F64SumMinMax)
      return launch_part<2, true, kSigI32SumMinMax_F64SumMinMax>(q, pa, s, tm);
  }
  if constexpr (NC == 1) {
    if (pack0 && sig == kSigI32Sum) return launch_part<1, true, kSigI32Sum>(q, pa, s, tm);
  }
  if (pack0) return launch_part<NC, true, 0>(q, pa, s, tm);
  return launch_part<NC, false, 0>(q, pa, s, tm);
}

int run_partition(const nfc_groupby_args* a, const ColSet& cs_in, const OutSet& o_in, const nfc_probe& p,
                  const uint32_t* vmask, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err,
                  int64_t* buckets_out, StageTimer* tm) {
  // 4-byte columns first (outputs follow their column).
  ColSet cs = cs_in;
  OutSet o = o_in;
  {
    int k = 0;
    for (int pass = 0; pass < 2; ++pass)
      for (int c = 0; c < cs_in.ncols; ++c)
        if ((cs_in.dtype[c] == NFC_I32) == (pass == 0)) {
          cs.dtype[k] = cs_in.dtype[c];
          cs.aggs[k] = cs_in.aggs[c];
          cs.data[k] = cs_in.data[c];
          o.sum[k] = o_in.sum[c];
          o.mn[k] = o_in.mn[c];
          o.mx[k] = o_in.mx[c];
          ++k;
        }
  }
  const bool pack0 = cs.ncols > 0 && cs.dtype[0] == NFC_I32;
  const int nw = cs.ncols == 0 ? 1 : cs.ncols + 1 - (pack0 ? 1 : 0);
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

  PartLaunch q{};
  q.a = a;
  q.cs = cs;
  q.vmask = vmask;
  q.al = inputs_aligned(a);
  q.kmin = (int32_t)p.kmin;
  q.wb = wb;
  q.nb = nb;
  q.d_err = d_err;
  q.nv = p.n_valid;
  q.two_level = nb > 128;
  q.nc = q.two_level ? (int32_t)((nb + (1 << kCoarseShift) - 1) >> kCoarseShift) : nb;
  // Coalesced scatter: 16-byte aligned inputs, coarse fan-out <= kMaxPassBins,
  // TMA stages + the tile's sort buffer fit in shared memory.
  if (q.al && (reinterpret_cast<uintptr_t>(vmask) & 15u) == 0 && q.nc <= kMaxPassBins) {
    BulkLayout& L = q.L;
    uint32_t off = kBulkTile * 4;
    L.bytes_keys = kBulkTile * 4;
    L.off_vmask = off;
    L.bytes_vmask = kBulkTile / 8;
    if (vmask) off += L.bytes_vmask;
    for (int c = 0; c < cs.ncols; ++c) {
      off = (off + 15u) & ~15u;
      L.off_col[c] = off;
      L.bytes_col[c] = kBulkTile * (uint32_t)dtype_bytes(cs.dtype[c]);
      off += L.bytes_col[c];
    }
    L.stage_bytes = (off + 127u) & ~127u;
    // Three stages within half an SM's shared memory (two CTAs per SM), else
    // as many as one CTA can hold.
    for (const size_t budget : {kPass1SmemPerSm / 2, kPass1SmemPerCta}) {
      L.stages = 3;
      while (L.stages >= 2 && pass1_smem(L) > budget) --L.stages;
      if (L.stages >= 2) break;
    }
    if (L.stages >= 2) {
      q.coalesced = true;
      q.nfull = a->n / kBulkTile;
    }
  }

  struct {
    uint32_t* ghist; int64_t* offs; uint32_t* cursor; int32_t* item_base; int32_t* merge_slot;
    int32_t* n_merge; uint32_t* slice_done; uint64_t* lb; uint32_t* ticket;
  } w;
  unsigned char* small = nullptr;
  const size_t nbp = (size_t)nb + 1;
  const size_t ncp = (size_t)q.nc + 1;
  const size_t small_bytes = nbp * (4 + 8 + 4 + 4 + 4 + 4 + 8) + ncp * (4 + 8 + 4) + 128;
  NFC_CUDA(sc.alloc(&small, small_bytes));
  NFC_CUDA(cudaMemsetAsync(small, 0, small_bytes, s));
  unsigned char* qq = small;
  w.offs = reinterpret_cast<int64_t*>(qq); qq += 8 * nbp;
  w.lb = reinterpret_cast<uint64_t*>(qq); qq += 8 * nbp;
  q.coffs = reinterpret_cast<int64_t*>(qq); qq += 8 * ncp;
  w.ghist = reinterpret_cast<uint32_t*>(qq); qq += 4 * nbp;
  w.cursor = reinterpret_cast<uint32_t*>(qq); qq += 4 * nbp;
  w.item_base = reinterpret_cast<int32_t*>(qq); qq += 4 * nbp;
  w.merge_slot = reinterpret_cast<int32_t*>(qq); qq += 4 * nbp;
  w.slice_done = reinterpret_cast<uint32_t*>(qq); qq += 4 * nbp;
  q.ccursor = reinterpret_cast<uint32_t*>(qq); qq += 4 * ncp;
  qq += 4 * ncp;
  w.n_merge = reinterpret_cast<int32_t*>(qq); qq += 8;
  w.ticket = reinterpret_cast<uint32_t*>(qq); qq += 8;
  q.wide = reinterpret_cast<uint32_t*>(qq); qq += 8;
  q.cursor = w.cursor;

  {
    // Full tiles through the bulk-copy histogram when the keys and the
    // combined bitmap are 16-byte aligned; the remaining rows (or all of
    // them) through k_part_hist.
    int64_t hfull = 0;
    if ((reinterpret_cast<uintptr_t>(a->keys) & 15u) == 0 && (reinterpret_cast<uintptr_t>(vmask) & 15u) == 0)
      hfull = a->n / kHistTile;
    if (hfull > 0) {
      const size_t smem = 128 + (size_t)kHistStages * kHistStageBytes + (size_t)nb * 4;
      NFC_CUDA(cudaFuncSetAttribute(k_part_hist_bulk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int per_sm = 2 * (smem + 1024) <= 228 * 1024 ? 2 : 1;
      const int64_t g = std::max<int64_t>(1, std::min<int64_t>(hfull, (int64_t)num_sms() * per_sm));
      k_part_hist_bulk<<<(unsigned)g, 512, smem, s>>>(a->keys, vmask, hfull, q.kmin, wb, nb, w.ghist, d_err);
      NFC_CUDA(cudaGetLastError());
      tm->launched();
    }
    const int64_t r0 = hfull * kHistTile;
    if (a->n > r0) {
      const int64_t ntiles128 = (a->n - r0 + 127) / 128;
      const size_t smem = (size_t)nb * 4;
      NFC_CUDA(cudaFuncSetAttribute(k_part_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int64_t g = std::max<int64_t>(1, std::min<int64_t>((ntiles128 + 15) / 16, (int64_t)num_sms() * 4));
      k_part_hist<<<(unsigned)g, 256, smem, s>>>(a->keys + r0, vmask ? vmask + (r0 >> 5) : nullptr, a->n - r0,
                                                  q.al, q.kmin, wb, nb, w.ghist);
      NFC_CUDA(cudaGetLastError());
      tm->launched();
    }
  }
  const int64_t max_items = nb + nv / kSlice + 1;
  int32_t* item_bucket = nullptr;
  NFC_CUDA(sc.alloc(&item_bucket, (size_t)max_items));
  PartPlan pl{w.offs, w.cursor, w.item_base, w.merge_slot, w.n_merge, item_bucket};
  k_part_plan<<<1, 1024, 0, s>>>(w.ghist, nb, kSlice, pl);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  if (q.coalesced && q.two_level) {
    k_part_plan2<<<1, 1024, 0, s>>>(w.offs, nb, q.nc, q.ccursor, q.coffs);
    NFC_CUDA(cudaGetLastError());
    tm->launched();
    NFC_CUDA(sc.alloc(&q.rec_a, (size_t)std::max<int64_t>(nv, 1) * nw + 2));  // +2: 16-byte tail of the refine copies
  }
  tm->mark(s);

  NFC_CUDA(sc.alloc(&q.rec, (size_t)std::max<int64_t>(nv, 1) * nw));
  const int64_t W = 1ll << wb;
  const int64_t max_merge = nv / (kSlice + 1) + 1;
  unsigned char* gmb = nullptr;
  NFC_CUDA(sc.alloc(&gmb, (size_t)max_merge * W * slot + 64));
  const StateRef gm = carve_state(cs, gmb, max_merge * W);

  PartAggArgs pa;
  pa.cs = cs;
  pa.rec = q.rec;
  pa.offs = w.offs;
  pa.item_base = w.item_base;
  pa.item_bucket = item_bucket;
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
  pa.wide = q.wide;
  q.agg_smem = (size_t)W * slot + 64;
  q.max_items = max_items;
  k_merge_init<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((max_merge * W + 255) / 256, (int64_t)num_sms() * 4)),
                 256, 0, s>>>(cs, gm, w.n_merge, W);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  int rc;
  switch (cs.ncols) {
    case 0: rc = launch_part_nc<0>(pack0, q, pa, s, tm); break;
    case 1: rc = launch_part_nc<1>(pack0, q, pa, s, tm); break;
    case 2: rc = launch_part_nc<2>(pack0, q, pa, s, tm); break;
    case 3: rc = launch_part_nc<3>(pack0, q, pa, s, tm); break;
    default: rc = launch_part_nc<4>(pack0, q, pa, s, tm); break;
  }
  if (rc) return rc;
  tm->mark(s);
  return NFC_OK;
}

}  // namespace nfc
