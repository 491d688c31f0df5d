// SHARED_HASH strategy: per-CTA shared-memory hash tables in front of a
// small global hash table.
//
// Each CTA takes chunks of 65,536 rows.  For every chunk it clears a
// shared-memory table of T keys plus their aggregation state (AggState),
// folds the chunk's valid rows into it with shared-memory atomics, and at the
// end of the chunk merges every occupied slot into the global table
// (hash_core.cuh) with one set of global atomics per distinct key.  A row
// whose key finds no free shared slot within kShProbe probes goes straight to
// the global table.  The global table is sized from the caller's distinct
// hint (room for 4x the hint plus 2^18 keys at load <= 0.5); if an insert
// into it fails within kGlobalProbe probes every CTA stops and the pass is
// repeated with a table 8x larger (at most the upper bound min(span, valid
// rows)); only if that also overflows does the caller rerun the group-by as
// HASH.  A low estimate costs time, never correctness.
//
// Low-cardinality inputs with a key span too wide for a dense table (Zipf
// over a huge domain, sparse identifiers, runs of repeated keys) are where
// this wins: one pass over the rows, shared-memory atomics, and a sort of
// only the distinct keys.  Rows of a warp that share a key are combined with
// warp reductions first (warp_agg_rows), so a run or a hot key costs one
// table update per warp step.
#include <algorithm>

#include "agg_smem.cuh"
#include "groupby_host.h"
#include "hash_core.cuh"

namespace nfc {
namespace {

constexpr int kShThreads = 512;
constexpr int64_t kShChunk = 65536;  // most rows per shared table lifetime (16-bit split sums stay exact)
constexpr int64_t kShMinChunk = 16384;  // fewest rows per chunk when the input is too small to fill the grid
constexpr int kShProbe = 16;
constexpr uint64_t kGlobalProbe = 512;

NFC_DEV uint32_t smem_hash(int32_t key, int lgT) {
  return (uint32_t)(((uint64_t)(uint32_t)key * 0xD6E8FEB86659FD93ull) >> (64 - lgT));
}

template <int NC, uint32_t SIG>
__global__ void __launch_bounds__(kShThreads, 2)
    k_shash_agg(const int32_t* __restrict__ keys, const uint32_t* __restrict__ vmask, ColSet cs, int64_t n,
                int64_t chunk, bool aligned, int lgT, uint64_t* gtable, int glg, StateRef gst, int32_t* ovf) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int T = 1 << lgT;
  unsigned long long* skey = reinterpret_cast<unsigned long long*>(sm);
  const AggState<NC> st = carve_agg<NC, SIG>(cs, sm + 8 * T, T);
  const int warp = threadIdx.x >> 5, lane = lane_id();
  const int64_t nchunks = (n + chunk - 1) / chunk;
  __shared__ int s_stop;
  bool spilled_fail = false;
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    // Once any CTA found the global table too small the pass is void: stop.
    if (threadIdx.x == 0) s_stop = ld_volatile_u32(reinterpret_cast<const uint32_t*>(ovf)) != 0u;
    __syncthreads();
    if (s_stop) break;
    for (int g = threadIdx.x; g < T; g += kShThreads) {
      skey[g] = 0ull;
      agg_init<NC, SIG>(cs, st, g);
    }
    __syncthreads();
    const int64_t r1 = std::min<int64_t>(n, (ch + 1) * chunk);
    for (int64_t t = ch * chunk + (int64_t)warp * 128; t < r1; t += (kShThreads / 32) * 128) {
      const int64_t row0 = t + 4 * lane;
      TileT<NC> tile;
      if (aligned && row0 + 4 <= n) load_tile4_full<true, NC, SIG>(keys, vmask, cs, row0, tile);
      else load_tile4_tail<true, NC, SIG>(keys, vmask, cs, row0, n, tile);
      // Shared slot of a key (inserted if absent), -1 after kShProbe probes.
      auto lookup = [&](int32_t key) -> int {
        const unsigned long long w = (1ull << 32) | (uint32_t)key;
        const uint32_t h = smem_hash(key, lgT);
        for (int i = 0; i < kShProbe; ++i) {
          const uint32_t slot = (h + i) & (uint32_t)(T - 1);
          unsigned long long cur = skey[slot];
          if (cur == 0ull) cur = atomicCAS(&skey[slot], 0ull, w);
          if (cur == 0ull || cur == w) return (int)slot;
        }
        return -1;
      };
      // Row r of every lane in one warp-aggregated step: equal keys of a warp
      // (runs, hot keys) are combined before they touch the table.
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        uint64_t raw[NC > 0 ? NC : 1];
#pragma unroll
        for (int c = 0; c < NC; ++c) raw[c] = tile.raw[c][r];
        warp_agg_rows<NC, SIG>(
            cs, (tile.valid >> r) & 1u, tile.key[r], raw,
            [&](int32_t key, uint32_t k, const uint64_t* sum, const uint64_t* mn, const uint64_t* mx) {
              const int g = lookup(key);
              if (g >= 0) {
                agg_apply_group<NC, SIG>(cs, st, (uint32_t)g, k, sum, mn, mx);
              } else {
                const int64_t gs = hash_slot_bounded(gtable, glg, key, kGlobalProbe);
                if (gs < 0) spilled_fail = true;
                else state_apply_group(cs, gst, gs, k, sum, mn, mx);
              }
            },
            [&](int32_t key, const uint64_t* rw) {
              const int g = lookup(key);
              if (g >= 0) {
                agg_apply<NC, SIG>(cs, st, (uint32_t)g, rw);
              } else {
                const int64_t gs = hash_slot_bounded(gtable, glg, key, kGlobalProbe);
                if (gs < 0) spilled_fail = true;
                else state_apply(cs, gst, gs, rw);
              }
            });
      }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < T; g += kShThreads) {
      const unsigned long long w = skey[g];
      if (w == 0ull || st.cnt[g] == 0u) continue;
      const int64_t gs = hash_slot_bounded(gtable, glg, (int32_t)(uint32_t)w, kGlobalProbe);
      if (gs < 0) spilled_fail = true;
      else agg_merge<NC, SIG>(cs, gst, gs, st, g);
    }
    if (__syncthreads_or(spilled_fail)) {
      if (threadIdx.x == 0) atomicExch(ovf, 1);
      break;
    }
  }
}

constexpr uint32_t kSigI32Sum = sig_col(0, NFC_I32, NFC_AGG_SUM);

struct ShLaunch {
  const int32_t* keys;
  const uint32_t* vmask;
  ColSet cs;
  int64_t n;
  bool aligned;
  uint64_t* gtable;
  int glg;
  StateRef gst;
  int32_t* ovf;
};

template <int NC, uint32_t SIG>
int launch_shash(const ShLaunch& L, size_t slot_bytes, cudaStream_t s) {
  // Two CTAs per SM: up to ~110 KB of shared memory each.
  int lgT = 12;
  while (lgT > 8 && ((size_t)8 + slot_bytes) * ((size_t)1 << lgT) > 110 * 1024) --lgT;
  const size_t smem = ((size_t)8 + slot_bytes) * ((size_t)1 << lgT) + 64;
  NFC_CUDA(cudaFuncSetAttribute(k_shash_agg<NC, SIG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // Grid: one CTA per kShMinChunk rows, at most two per SM.  Equal chunk
  // counts per CTA: the chunk is shrunk (to a multiple of 512 rows, never
  // above kShChunk) until the chunks divide evenly over the grid, so no CTA
  // runs one chunk more than the others at the end.
  const int64_t nchunks = (L.n + kShChunk - 1) / kShChunk;
  const int grid = (int)std::max<int64_t>(
      1, std::min<int64_t>((L.n + kShMinChunk - 1) / kShMinChunk, (int64_t)num_sms() * 2));
  const int64_t rounds = std::max<int64_t>(1, (nchunks + grid - 1) / grid);
  const int64_t per = std::max<int64_t>(1, (L.n + grid * rounds - 1) / (grid * rounds));
  const int64_t chunk = std::min<int64_t>(kShChunk, (per + 511) / 512 * 512);
  k_shash_agg<NC, SIG><<<grid, kShThreads, smem, s>>>(L.keys, L.vmask, L.cs, L.n, chunk, L.aligned, lgT, L.gtable,
                                                      L.glg, L.gst, L.ovf);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

int dispatch_shash(const ShLaunch& L, size_t slot_bytes, cudaStream_t s) {
  switch (L.cs.ncols) {
    case 0: return launch_shash<0, 0>(L, slot_bytes, s);
    case 1:
      if (sig_of(L.cs) == kSigI32Sum) return launch_shash<1, kSigI32Sum>(L, slot_bytes, s);
      return launch_shash<1, 0>(L, slot_bytes, s);
    case 2: return launch_shash<2, 0>(L, slot_bytes, s);
    case 3: return launch_shash<3, 0>(L, slot_bytes, s);
    default: return launch_shash<4, 0>(L, slot_bytes, s);
  }
}

}  // namespace

int run_shared_hash(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
                    const uint32_t* vmask, int64_t distinct_hint, cudaStream_t s, Scratch& sc, int64_t* d_ng,
                    int32_t* d_err, int64_t* slots_out, int* overflow_level, StageTimer* tm) {
  *overflow_level = 0;
  const int64_t span = p.kmax - p.kmin + 1;
  const int64_t bound = std::max<int64_t>(1, std::min<int64_t>(span, p.n_valid));
  // The hint is an estimate (the learned planner's is off by 4x or more on a
  // tenth of its inputs, mostly clustered keys whose first rows show few
  // values), and an overflowing pass costs far more than a larger table to
  // clear: the first table holds 4x the hint plus 2^18 keys, each retry 8x
  // the last, up to the bound min(span, valid rows).
  int64_t target = distinct_hint > 0 ? std::min<int64_t>(bound, 4 * distinct_hint + (1 << 18)) : bound;
  const size_t slot_bytes = state_bytes_per_slot(cs);
  int32_t* ovf = nullptr;
  NFC_CUDA(sc.alloc(&ovf, 1));
  for (int attempt = 0; attempt < 3; ++attempt) {
    int lg = 12;
    while ((1ll << lg) < 2 * target) ++lg;
    const int64_t cap = 1ll << lg;
    *slots_out = cap;
    uint64_t* table = nullptr;
    unsigned char* stb = nullptr;
    NFC_CUDA(sc.alloc(&table, (size_t)cap));
    NFC_CUDA(sc.alloc(&stb, (size_t)cap * slot_bytes + 64));
    NFC_CUDA(cudaMemsetAsync(ovf, 0, sizeof(int32_t), s));
    const StateRef st = carve_state(cs, stb, cap);
    hash_clear_init(cs, st, table, cap, s);
    NFC_CUDA(cudaGetLastError());
    tm->launched(2);
    tm->mark(s);
    ShLaunch L{a->keys, vmask, cs, a->n, inputs_aligned(a), table, lg, st, ovf};
    int rc = dispatch_shash(L, slot_bytes, s);
    if (rc) return rc;
    tm->launched();
    tm->mark(s);
    int32_t h_ovf = 0;
    NFC_CUDA(cudaMemcpyAsync(&h_ovf, ovf, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    NFC_CUDA(cudaStreamSynchronize(s));
    if (!h_ovf) return hash_finish(cs, o, st, table, cap, std::min<int64_t>(bound, cap), s, sc, d_ng, d_err, tm);
    *overflow_level = target >= bound ? 2 : 1;
    if (target >= bound) break;
    target = std::min<int64_t>(bound, 8 * target);
  }
  return NFC_OK;  // level 2: still overflowing at the full size, the caller reruns as HASH
}

}  // namespace nfc
