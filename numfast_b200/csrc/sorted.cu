// SORTED strategy: group-by over keys that are nondecreasing in row order.
//
// The reference plans "sorted" whenever the valid keys are nondecreasing
// (src/Runtime/Planner/_lib/planner.py:226) and reduces each run of equal
// keys in one pass (sorted_fused_aggregate, src/Drivers/CPU/_lib/
// groupindex.py:259-304; sorted_runs, numfast-native/src/groupby/sorted.rs:
// 24-56).  The output contract is the one of every strategy: groups
// ascending by key, int64 counts and integer sums, float64 sums, min/max in
// the value dtype, rows with a NULL anywhere dropped.
//
// Here, with no atomics and no aggregation state in global memory:
//   1. k_sorted_prev    one CTA turns the probe records into the last valid
//                       key before every tile (an exclusive "last non-empty"
//                       scan over the 16,384-row blocks the probe summarised);
//   2. k_sorted_agg     one CTA per tile of 16,384 rows, claimed in order.
//                       The tile's keys and combined validity come into
//                       shared memory with one bulk (TMA) copy.  Pass 1: each
//                       warp marks the run heads of its 2,048-row chunk (a
//                       valid row whose key differs from the previous valid
//                       row's) and counts them; a decoupled look-back gives
//                       the tile its first run number.  Pass 2: each warp
//                       streams its chunk's values in steps of 128 rows (4
//                       per lane, 128-bit loads, the next step in flight) and
//                       reduces the runs with a segmented scan in registers
//                       (lane, then warp shuffles that stop once every lane
//                       has met a head).  Runs that end inside a step go to a
//                       per-warp shared-memory buffer (where the keys were)
//                       and leave in one coalesced pass per step.  The warps'
//                       edge runs are merged by one warp; the tile's first run
//                       (continued from earlier tiles) and last run (possibly
//                       continued by later ones) leave as two partial
//                       "pieces";
//   3. k_sorted_fix     the pieces are merged in order (segmented scan by run
//                       number): chunks of 1,024 in parallel CTAs, then the
//                       chunks' own edge runs in one CTA.
// Output keys are written by the lane holding each run's head.  float64 sums
// are reduced as a tree (order differs from the reference's row loop; within
// 1e-12 relative); everything else is exact.
#include <algorithm>

#include "bulk.cuh"
#include "groupby_host.h"

namespace nfc {
namespace {

constexpr int kSoThreads = 256;
constexpr int kSoWarps = kSoThreads / 32;
constexpr int kSoWarpRows = 2048;                 // rows of one warp chunk
constexpr int kSoTile = kSoWarps * kSoWarpRows;   // rows per CTA tile (16,384)
static_assert(kSoTile == kProbeBlockRows, "one probe record per tile");
constexpr int kSoLaneRows = 4;                    // pass 2: rows per lane and step
constexpr int kSoStepRows = 32 * kSoLaneRows;
constexpr int kSoSteps = kSoWarpRows / kSoStepRows;
constexpr int kRunBuf = kSoStepRows;              // runs ending inside one step
constexpr int kFixThreads = 1024;

// ---------------------------------------------------------------- run aggregate
// Integers are kept as int64 bits (sums wrap like the other strategies' int64
// atomics), float64 min/max as the ordered encodings of nfc_common.cuh;
// int32 min/max use int32 identities and 32-bit compares.  A count never
// exceeds the row count (< 2^31).
template <int NC>
struct Seg {
  uint32_t cnt;
  uint64_t sum[NC > 0 ? NC : 1], mn[NC > 0 ? NC : 1], mx[NC > 0 ? NC : 1];
};

template <int NC, uint32_t SIG>
NFC_DEV void seg_identity(const ColSet& cs, Seg<NC>& a) {
  a.cnt = 0;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    a.sum[c] = 0;
    if (col_dt<SIG>(cs, c) == NFC_F64) {
      a.mn[c] = ~0ull;
      a.mx[c] = 0ull;
    } else if (col_dt<SIG>(cs, c) == NFC_I32) {
      a.mn[c] = (uint64_t)(int64_t)INT_MAX;
      a.mx[c] = (uint64_t)(int64_t)INT_MIN;
    } else {
      a.mn[c] = (uint64_t)LLONG_MAX;
      a.mx[c] = (uint64_t)LLONG_MIN;
    }
  }
}

NFC_DEV uint64_t i32_min64(uint64_t a, uint64_t b) { return (uint64_t)(int64_t)min((int32_t)a, (int32_t)b); }
NFC_DEV uint64_t i32_max64(uint64_t a, uint64_t b) { return (uint64_t)(int64_t)max((int32_t)a, (int32_t)b); }
NFC_DEV uint64_t f64_add_bits(uint64_t a, uint64_t b) {
  return (uint64_t)__double_as_longlong(__longlong_as_double((long long)a) + __longlong_as_double((long long)b));
}

// a = a then b.
template <int NC, uint32_t SIG>
NFC_DEV void seg_combine(const ColSet& cs, Seg<NC>& a, const Seg<NC>& b) {
  a.cnt += b.cnt;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    if (dt == NFC_F64) {
      if (ag & NFC_AGG_SUM) a.sum[c] = f64_add_bits(a.sum[c], b.sum[c]);
      if (ag & NFC_AGG_MIN) a.mn[c] = min(a.mn[c], b.mn[c]);
      if (ag & NFC_AGG_MAX) a.mx[c] = max(a.mx[c], b.mx[c]);
    } else if (dt == NFC_I32) {
      if (ag & NFC_AGG_SUM) a.sum[c] += b.sum[c];
      if (ag & NFC_AGG_MIN) a.mn[c] = i32_min64(a.mn[c], b.mn[c]);
      if (ag & NFC_AGG_MAX) a.mx[c] = i32_max64(a.mx[c], b.mx[c]);
    } else {
      if (ag & NFC_AGG_SUM) a.sum[c] += b.sum[c];
      if (ag & NFC_AGG_MIN) a.mn[c] = (uint64_t)min((long long)a.mn[c], (long long)b.mn[c]);
      if (ag & NFC_AGG_MAX) a.mx[c] = (uint64_t)max((long long)a.mx[c], (long long)b.mx[c]);
    }
  }
}

// Fold one row: int32 values as their 32-bit word, 8-byte values as bits.
template <int NC, uint32_t SIG>
NFC_DEV void seg_add_row(const ColSet& cs, Seg<NC>& a, const uint64_t* raw) {
  a.cnt += 1;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    const uint64_t r = raw[c];
    if (dt == NFC_F64) {
      if (ag & NFC_AGG_SUM) a.sum[c] = f64_add_bits(a.sum[c], r);
      if (ag & (NFC_AGG_MIN | NFC_AGG_MAX)) {
        // One order-preserving word for both lanes (the encodings of
        // nfc_common.cuh); NaN wins both.
        const uint32_t hi = (uint32_t)(r >> 32), lo = (uint32_t)r;
        const uint32_t s = (uint32_t)((int32_t)hi >> 31);
        const uint64_t ord = r ^ (((uint64_t)(s | 0x80000000u) << 32) | s);
        const uint32_t ah = hi & 0x7FFFFFFFu;
        const bool nan = ah > 0x7FF00000u || (ah == 0x7FF00000u && lo != 0u);
        if (ag & NFC_AGG_MIN) a.mn[c] = min(a.mn[c], nan ? (uint64_t)0 : ord);
        if (ag & NFC_AGG_MAX) a.mx[c] = max(a.mx[c], nan ? ~(uint64_t)0 : ord);
      }
    } else if (dt == NFC_I32) {
      if (ag & NFC_AGG_SUM) a.sum[c] += (uint64_t)(int64_t)(int32_t)r;
      if (ag & NFC_AGG_MIN) a.mn[c] = i32_min64(a.mn[c], r);
      if (ag & NFC_AGG_MAX) a.mx[c] = i32_max64(a.mx[c], r);
    } else {
      if (ag & NFC_AGG_SUM) a.sum[c] += r;
      if (ag & NFC_AGG_MIN) a.mn[c] = (uint64_t)min((long long)a.mn[c], (long long)r);
      if (ag & NFC_AGG_MAX) a.mx[c] = (uint64_t)max((long long)a.mx[c], (long long)r);
    }
  }
}

// Shuffles of a run aggregate: only the requested aggregates move, counts
// and int32 min/max as 32-bit words.
template <int NC, uint32_t SIG, bool UP>
NFC_DEV void seg_shfl(const ColSet& cs, const Seg<NC>& a, Seg<NC>& out, int arg) {
  auto sh32 = [&](uint32_t v) { return UP ? __shfl_up_sync(0xffffffffu, v, arg) : __shfl_sync(0xffffffffu, v, arg); };
  auto sh64 = [&](uint64_t v) { return UP ? __shfl_up_sync(0xffffffffu, v, arg) : __shfl_sync(0xffffffffu, v, arg); };
  out.cnt = sh32(a.cnt);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int ag = col_ag<SIG>(cs, c);
    if (ag & NFC_AGG_SUM) out.sum[c] = sh64(a.sum[c]);
    if (col_dt<SIG>(cs, c) == NFC_I32) {
      if (ag & NFC_AGG_MIN) out.mn[c] = (uint64_t)(int64_t)(int32_t)sh32((uint32_t)a.mn[c]);
      if (ag & NFC_AGG_MAX) out.mx[c] = (uint64_t)(int64_t)(int32_t)sh32((uint32_t)a.mx[c]);
    } else {
      if (ag & NFC_AGG_MIN) out.mn[c] = sh64(a.mn[c]);
      if (ag & NFC_AGG_MAX) out.mx[c] = sh64(a.mx[c]);
    }
  }
}

// Output row g of run aggregate a (keys are written at the heads).
template <int NC, uint32_t SIG>
NFC_DEV void seg_emit(const ColSet& cs, const OutSet& o, int64_t g, const Seg<NC>& a) {
  o.counts[g] = (int64_t)a.cnt;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    if (ag & NFC_AGG_SUM) static_cast<uint64_t*>(o.sum[c])[g] = a.sum[c];
    if (dt == NFC_I32) {
      if (ag & NFC_AGG_MIN) static_cast<int32_t*>(o.mn[c])[g] = (int32_t)a.mn[c];
      if (ag & NFC_AGG_MAX) static_cast<int32_t*>(o.mx[c])[g] = (int32_t)a.mx[c];
    } else if (dt == NFC_I64) {
      if (ag & NFC_AGG_MIN) static_cast<uint64_t*>(o.mn[c])[g] = a.mn[c];
      if (ag & NFC_AGG_MAX) static_cast<uint64_t*>(o.mx[c])[g] = a.mx[c];
    } else {
      if (ag & NFC_AGG_MIN) static_cast<uint64_t*>(o.mn[c])[g] = f64_min_dec(a.mn[c]);
      if (ag & NFC_AGG_MAX) static_cast<uint64_t*>(o.mx[c])[g] = f64_max_dec(a.mx[c]);
    }
  }
}

// Partial runs at tile (or chunk) edges: slot 2t = the run continued from
// before tile t, slot 2t+1 = the tile's last run; idx -1 = none.
struct Pieces {
  int64_t* idx;
  uint64_t* cnt;
  uint64_t* sum[NFC_MAX_COLS];
  uint64_t* mn[NFC_MAX_COLS];
  uint64_t* mx[NFC_MAX_COLS];
};

template <int NC>
NFC_DEV void piece_store(const Pieces& P, int64_t slot, int64_t idx, const Seg<NC>& a) {
  P.idx[slot] = idx;
  P.cnt[slot] = a.cnt;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    P.sum[c][slot] = a.sum[c];
    P.mn[c][slot] = a.mn[c];
    P.mx[c][slot] = a.mx[c];
  }
}

template <int NC>
NFC_DEV void piece_load(const Pieces& P, int64_t slot, Seg<NC>& a) {
  a.cnt = (uint32_t)P.cnt[slot];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    a.sum[c] = P.sum[c][slot];
    a.mn[c] = P.mn[c][slot];
    a.mx[c] = P.mx[c][slot];
  }
}

// Warp-wide segmented scan.  Lane l holds (f, a): f = a run starts inside
// the lane.  The operator is (f1,a1) then (f2,a2) = (f1|f2, f2 ? a2 : a1+a2).
// (cf, ca) is the warp-uniform open run before lane 0.  Returns in ex the
// exclusive value of every lane (carry included) and advances the carry past
// lane 31.  The scan stops as soon as every lane has met a head.
template <int NC, uint32_t SIG>
NFC_DEV void warp_seg_scan(const ColSet& cs, uint32_t f, const Seg<NC>& a, uint32_t& cf, Seg<NC>& ca, Seg<NC>& ex) {
  const int lane = lane_id();
  uint32_t incf = f;
  Seg<NC> inc = a;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    if (__all_sync(0xffffffffu, incf)) break;
    Seg<NC> y;
    seg_shfl<NC, SIG, true>(cs, inc, y, o);
    const uint32_t yf = __shfl_up_sync(0xffffffffu, incf, o);
    if (lane >= o) {
      if (!incf) {
        seg_combine<NC, SIG>(cs, y, inc);
        inc = y;
      }
      incf |= yf;
    }
  }
  Seg<NC> w;
  seg_shfl<NC, SIG, true>(cs, inc, w, 1);
  const uint32_t wf = __shfl_up_sync(0xffffffffu, incf, 1);
  if (lane == 0 || !wf) {
    ex = ca;
    if (lane != 0) seg_combine<NC, SIG>(cs, ex, w);
  } else {
    ex = w;
  }
  Seg<NC> last;
  seg_shfl<NC, SIG, false>(cs, inc, last, 31);
  const uint32_t lastf = __shfl_sync(0xffffffffu, incf, 31);
  if (lastf) ca = last;
  else seg_combine<NC, SIG>(cs, ca, last);
  cf |= lastf;
}

// Block-wide segmented scan (same operator), blockDim a multiple of 32.
template <int NC, uint32_t SIG>
struct SegScanSmem {
  Seg<NC> tot[32];
  uint32_t totf[32];
  Seg<NC> wcarry[32];
  uint32_t wcarryf[32];
  Seg<NC> carry;
  uint32_t carryf;
};

template <int NC, uint32_t SIG>
NFC_DEV void block_seg_scan(const ColSet& cs, uint32_t f, const Seg<NC>& a, uint32_t& carry_f, Seg<NC>& carry,
                            Seg<NC>& excl, SegScanSmem<NC, SIG>& sm) {
  const int lane = lane_id(), warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // Within the warp, from an empty carry: wex = the lanes before this one
  // (back to the nearest head), wtot = the whole warp.
  uint32_t wf = 0;
  Seg<NC> wtot, wex;
  seg_identity<NC, SIG>(cs, wtot);
  warp_seg_scan<NC, SIG>(cs, f, a, wf, wtot, wex);
  const bool head_before = (__ballot_sync(0xffffffffu, f) & ((1u << lane) - 1u)) != 0u;
  if (lane == 0) {
    sm.tot[warp] = wtot;
    sm.totf[warp] = wf;
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t tf = 0;
    Seg<NC> t;
    seg_identity<NC, SIG>(cs, t);
    if (lane < nw) {
      t = sm.tot[lane];
      tf = sm.totf[lane];
    }
    uint32_t c2f = carry_f;
    Seg<NC> c2 = carry, ex;
    warp_seg_scan<NC, SIG>(cs, tf, t, c2f, c2, ex);  // ex = carry-in of warp `lane`
    if (lane < nw) sm.wcarry[lane] = ex;
    if (lane == 0) {
      sm.carry = c2;
      sm.carryf = c2f;
    }
  }
  __syncthreads();
  if (head_before) {
    excl = wex;
  } else {
    excl = sm.wcarry[warp];
    seg_combine<NC, SIG>(cs, excl, wex);
  }
  carry = sm.carry;
  carry_f = sm.carryf;
  __syncthreads();
}

// Last valid key before each tile: prev[t] = (1 << 32 | key) or 0 when no
// valid row precedes tile t.  One CTA walks the probe records (one per tile)
// in order.
__global__ void __launch_bounds__(1024) k_sorted_prev(const ProbeRec* recs, int64_t nrec, uint64_t* prev) {
  __shared__ uint64_t s_w[32];
  __shared__ uint64_t s_carry;
  const int lane = lane_id(), warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nrec; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    uint64_t v = 0;  // inclusive "last valid" of record i
    if (i < nrec) {
      const ProbeRec r = recs[i];
      if (r.flags & 1u) v = (1ull << 32) | (uint32_t)r.last;
    }
    uint64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o && !(inc >> 32)) inc = y;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    uint64_t before = s_carry;
    for (int w = 0; w < warp; ++w)
      if (s_w[w] >> 32) before = s_w[w];
    uint64_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) ex = 0;
    const uint64_t mine = (ex >> 32) ? ex : before;
    if (i < nrec) prev[i] = mine;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = (inc >> 32) ? inc : mine;
    __syncthreads();
  }
}

// Values of one pass-2 step for one lane (kSoLaneRows consecutive rows):
// 32-bit words, the high words only for 8-byte columns.
template <int NC>
struct StepVals {
  uint32_t lo[NC > 0 ? NC : 1][kSoLaneRows];
  uint32_t hi[NC > 0 ? NC : 1][kSoLaneRows];
};

template <int NC, uint32_t SIG>
NFC_DEV void load_step(const ColSet& cs, int64_t n, bool aligned, int64_t row, StepVals<NC>& b) {
  if (row >= n) return;
  if (aligned && row + kSoLaneRows <= n) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (col_dt<SIG>(cs, c) == NFC_I32) {
        const int4 x = __ldcs(reinterpret_cast<const int4*>(static_cast<const int32_t*>(cs.data[c]) + row));
        b.lo[c][0] = x.x; b.lo[c][1] = x.y; b.lo[c][2] = x.z; b.lo[c][3] = x.w;
      } else {
        const int4* q = reinterpret_cast<const int4*>(static_cast<const uint64_t*>(cs.data[c]) + row);
        const int4 x = __ldcs(q), y = __ldcs(q + 1);
        b.lo[c][0] = x.x; b.hi[c][0] = x.y; b.lo[c][1] = x.z; b.hi[c][1] = x.w;
        b.lo[c][2] = y.x; b.hi[c][2] = y.y; b.lo[c][3] = y.z; b.hi[c][3] = y.w;
      }
    }
  } else {
#pragma unroll
    for (int r = 0; r < kSoLaneRows; ++r)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (row + r >= n) continue;
        if (col_dt<SIG>(cs, c) == NFC_I32) {
          b.lo[c][r] = (uint32_t) static_cast<const int32_t*>(cs.data[c])[row + r];
        } else {
          const uint64_t v = static_cast<const uint64_t*>(cs.data[c])[row + r];
          b.lo[c][r] = (uint32_t)v;
          b.hi[c][r] = (uint32_t)(v >> 32);
        }
      }
  }
}

// Runs that end inside one pass-2 step, buffered per warp: entry j = run
// (first run of the step - 1 + j).
template <int NC>
struct RunBuf {
  uint64_t sum[NC > 0 ? NC : 1][kRunBuf];
  uint64_t mn[NC > 0 ? NC : 1][kRunBuf];
  uint64_t mx[NC > 0 ? NC : 1][kRunBuf];
  uint32_t cnt[kRunBuf];
};

template <int NC, uint32_t SIG>
NFC_DEV void rb_store(const ColSet& cs, RunBuf<NC>& rb, int j, const Seg<NC>& a) {
  rb.cnt[j] = a.cnt;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int ag = col_ag<SIG>(cs, c);
    if (ag & NFC_AGG_SUM) rb.sum[c][j] = a.sum[c];
    if (ag & NFC_AGG_MIN) rb.mn[c][j] = a.mn[c];
    if (ag & NFC_AGG_MAX) rb.mx[c][j] = a.mx[c];
  }
}

template <int NC, uint32_t SIG>
NFC_DEV void rb_load(const ColSet& cs, const RunBuf<NC>& rb, int j, Seg<NC>& a) {
  a.cnt = rb.cnt[j];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int ag = col_ag<SIG>(cs, c);
    if (ag & NFC_AGG_SUM) a.sum[c] = rb.sum[c][j];
    if (ag & NFC_AGG_MIN) a.mn[c] = rb.mn[c][j];
    if (ag & NFC_AGG_MAX) a.mx[c] = rb.mx[c][j];
  }
}

template <int NC, uint32_t SIG>
struct SortedSmem {
  union {
    int32_t keys[kSoTile];       // pass 1: the tile's keys
    RunBuf<NC> rb[kSoWarps];     // pass 2: per-warp run buffers
  } u;
  alignas(16) uint32_t vbits[kSoTile / 32];
  uint32_t hbits[kSoTile / 32];
  uint64_t bar;
  uint32_t wheads[kSoWarps];
  int64_t wbase[kSoWarps];
  int64_t pidx[2 * kSoWarps];  // warp pieces: 2w = run continued into chunk w, 2w+1 = its last run
  Seg<NC> pseg[2 * kSoWarps];
  int64_t excl;
  int64_t tile;
  int32_t abort;
};

template <int NC, uint32_t SIG>
__global__ void __launch_bounds__(kSoThreads, 2) k_sorted_agg(const int32_t* __restrict__ keys,
                                                              const uint32_t* __restrict__ vmask, ColSet cs,
                                                              int64_t n, bool aligned, bool bulk_ok,
                                                              const uint64_t* __restrict__ prev, OutSet o,
                                                              int64_t cap, Pieces P, uint64_t* lb, uint32_t* ticket,
                                                              int64_t* ng_out, int32_t* err) {
  extern __shared__ __align__(128) unsigned char sm_raw[];
  SortedSmem<NC, SIG>& sm = *reinterpret_cast<SortedSmem<NC, SIG>*>(sm_raw);
  const int tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  if (tid == 0) {
    sm.tile = atomicAdd(ticket, 1u);
    sm.abort = 0;
    mbar_init(&sm.bar, 1);
    mbar_fence_init();
  }
  if (tid < 2 * kSoWarps) sm.pidx[tid] = -1;
  __syncthreads();
  const int64_t tile = sm.tile;
  const int64_t ntiles = (n + kSoTile - 1) / kSoTile;
  if (tile >= ntiles) return;
  const int64_t tbase = tile * kSoTile;
  const int c0 = warp * kSoWarpRows;  // chunk start (tile row)

  // The values do not depend on the keys: the first step's loads go out now
  // and land while the keys are staged, the heads counted and the tile's run
  // number looked up.
  StepVals<NC> va, vb2;
  load_step<NC, SIG>(cs, n, aligned, tbase + c0 + kSoLaneRows * lane, va);

  // ---- keys and validity of the tile -> shared memory.
  const bool full = tbase + kSoTile <= n;
  if (full && bulk_ok) {
    if (tid == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&sm.bar, (uint32_t)(kSoTile * 4 + (vmask ? kSoTile / 8 : 0)));
      bulk_g2s(sm.u.keys, keys + tbase, (uint32_t)(kSoTile * 4), &sm.bar);
      if (vmask) bulk_g2s(sm.vbits, vmask + tbase / 32, (uint32_t)(kSoTile / 8), &sm.bar);
    }
    if (!vmask)
      for (int w = tid; w < kSoTile / 32; w += kSoThreads) sm.vbits[w] = 0xFFFFFFFFu;
    if (!mbar_wait(&sm.bar, 0)) sm.abort = 1;
  } else {
    for (int i = tid; i < kSoTile; i += kSoThreads) sm.u.keys[i] = tbase + i < n ? __ldg(keys + tbase + i) : 0;
    for (int w = tid; w < kSoTile / 32; w += kSoThreads) {
      const int64_t r0 = tbase + 32 * (int64_t)w;
      uint32_t b = 0;
      if (r0 < n) {
        b = vmask ? __ldg(vmask + (r0 >> 5)) : 0xFFFFFFFFu;
        if (n - r0 < 32) b &= (1u << (n - r0)) - 1u;
      }
      sm.vbits[w] = b;
    }
  }
  __syncthreads();
  if (sm.abort) {
    // Let the copy land before the shared memory goes away.
    if (tid == 0) {
      atomicExch(err, NFC_ERR_TIMEOUT);
      mbar_wait(&sm.bar, 0);
    }
    __syncthreads();
    return;
  }

  // ---- pass 1: run heads of every warp chunk, 8 rows per lane and step.
  uint64_t carry = prev[tile];  // (1 << 32 | key) of the last valid row before the chunk
  if (warp > 0) {
    // Last valid row before the chunk inside the tile, if any: the warp reads
    // 32 validity words per round, nearest first.
    for (int w0 = c0 / 32 - 1; w0 >= 0; w0 -= 32) {
      const int wi = w0 - lane;
      const uint32_t b = wi >= 0 ? sm.vbits[wi] : 0u;
      const unsigned nz = __ballot_sync(0xffffffffu, b != 0u);
      if (nz) {
        const int l = __ffs(nz) - 1;
        const uint32_t bs = __shfl_sync(0xffffffffu, b, l);
        const int row = (w0 - l) * 32 + (31 - __clz(bs));
        carry = (1ull << 32) | (uint32_t)sm.u.keys[row];
        break;
      }
    }
  }
  uint32_t heads = 0;
  for (int st = 0; st < kSoWarpRows / 256; ++st) {
    const int r0 = c0 + st * 256 + 8 * lane;
    const int4 ka = *reinterpret_cast<const int4*>(&sm.u.keys[r0]);
    const int4 kb = *reinterpret_cast<const int4*>(&sm.u.keys[r0 + 4]);
    const int32_t k[8] = {ka.x, ka.y, ka.z, ka.w, kb.x, kb.y, kb.z, kb.w};
    const uint32_t vb = (sm.vbits[r0 >> 5] >> (r0 & 31)) & 0xFFu;
    uint64_t mine = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (vb & (1u << r)) mine = (1ull << 32) | (uint32_t)k[r];
    uint64_t inc = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      if (__all_sync(0xffffffffu, inc >> 32)) break;
      const uint64_t y = __shfl_up_sync(0xffffffffu, inc, off);
      if (lane >= off && !(inc >> 32)) inc = y;
    }
    uint64_t p = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0 || !(p >> 32)) p = carry;
    uint32_t hb = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (vb & (1u << r)) {
        if (!(p >> 32) || (int32_t)(uint32_t)p != k[r]) hb |= 1u << r;
        p = (1ull << 32) | (uint32_t)k[r];
      }
    reinterpret_cast<uint8_t*>(sm.hbits)[r0 >> 3] = (uint8_t)hb;
    heads += __popc(hb);
    const uint64_t l31 = __shfl_sync(0xffffffffu, inc, 31);
    if (l31 >> 32) carry = l31;
  }
  heads = warp_sum(heads);
  if (lane == 0) sm.wheads[warp] = heads;
  __syncthreads();  // also: every warp is done with the staged keys
  if (warp == 0) {
    const uint32_t h = lane < kSoWarps ? sm.wheads[lane] : 0u;
    uint32_t hi = h;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, hi, off);
      if (lane >= off) hi += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, hi, 31);
    const int64_t ex = lookback_exclusive(lb, tile, total, err);  // whole warp
    if (lane < kSoWarps) sm.wbase[lane] = ex + hi - h;
    if (lane == 0) {
      sm.excl = ex;
      if (tile == ntiles - 1) *ng_out = ex + total;
    }
  }
  __syncthreads();
  const int64_t excl_tile = sm.excl;
  const int64_t wbase = sm.wbase[warp];
  RunBuf<NC>& rb = sm.u.rb[warp];

  // ---- pass 2: values; runs reduced by a segmented scan per warp step.
  uint32_t cf = 0;
  Seg<NC> ca;
  seg_identity<NC, SIG>(cs, ca);
  int64_t hrun = wbase;  // run number of the next head in the chunk
  auto step = [&](int st, const StepVals<NC>& vals) {
    const int r0 = c0 + st * kSoStepRows + kSoLaneRows * lane;  // tile row
    const uint32_t vb = (sm.vbits[r0 >> 5] >> (r0 & 31)) & 0xFu;
    const uint32_t hb = (sm.hbits[r0 >> 5] >> (r0 & 31)) & 0xFu;
    const uint32_t hc = __popc(hb);
    uint32_t hi = hc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, hi, off);
      if (lane >= off) hi += y;
    }
    const uint32_t H = __shfl_sync(0xffffffffu, hi, 31);
    // Head j of the step starts run hrun + j and ends run hrun + j - 1, which
    // is buffer entry j.
    const int j0 = (int)(hi - hc);  // this lane's first head
    Seg<NC> lead, cur;
    seg_identity<NC, SIG>(cs, lead);
    seg_identity<NC, SIG>(cs, cur);
    bool seen = false;
    int j = j0;
#pragma unroll
    for (int r = 0; r < kSoLaneRows; ++r) {
      if (!(vb & (1u << r))) continue;
      if (hb & (1u << r)) {
        if (!seen) {
          lead = cur;
          seen = true;
        } else {
          rb_store<NC, SIG>(cs, rb, j, cur);  // a run that began and ended in this lane
        }
        // Runs never outnumber min(span, valid rows) <= cap for sorted keys;
        // the check only keeps a broken sortedness flag from writing past it.
        const int64_t g = hrun + j;
        if (g < cap) o.ukeys[g] = (int64_t)__ldg(keys + tbase + r0 + r);
        else atomicExch(err, NFC_ERR_RANGE);
        ++j;
        seg_identity<NC, SIG>(cs, cur);
      }
      uint64_t rv[NC > 0 ? NC : 1];
#pragma unroll
      for (int c = 0; c < NC; ++c)
        rv[c] = col_dt<SIG>(cs, c) == NFC_I32 ? (uint64_t)vals.lo[c][r]
                                              : ((uint64_t)vals.hi[c][r] << 32) | vals.lo[c][r];
      seg_add_row<NC, SIG>(cs, cur, rv);
    }
    if (!seen) lead = cur;
    Seg<NC> ex;
    warp_seg_scan<NC, SIG>(cs, seen ? 1u : 0u, seen ? cur : lead, cf, ca, ex);
    if (seen) {
      // The run that ends just before this lane's first head (run hrun+j0-1).
      seg_combine<NC, SIG>(cs, ex, lead);
      if (hrun + j0 - 1 < wbase) {
        // It began before the chunk: the warp's front piece.
        if (ex.cnt > 0) {
          sm.pidx[2 * warp] = hrun + j0 - 1;
          sm.pseg[2 * warp] = ex;
        }
      } else {
        rb_store<NC, SIG>(cs, rb, j0, ex);
      }
    }
    __syncwarp();
    // Runs hrun - 1 + j (j < H) ended in this step: out in one coalesced pass.
    for (int jj = lane; jj < (int)H; jj += 32) {
      const int64_t g = hrun - 1 + jj;
      if (g < wbase || g >= cap) continue;
      Seg<NC> a;
      rb_load<NC, SIG>(cs, rb, jj, a);
      seg_emit<NC, SIG>(cs, o, g, a);
    }
    __syncwarp();
    hrun += H;
  };
  for (int st = 0; st < kSoSteps; st += 2) {
    load_step<NC, SIG>(cs, n, aligned, tbase + c0 + (st + 1) * kSoStepRows + kSoLaneRows * lane, vb2);
    step(st, va);
    if (st + 2 < kSoSteps)
      load_step<NC, SIG>(cs, n, aligned, tbase + c0 + (st + 2) * kSoStepRows + kSoLaneRows * lane, va);
    step(st + 1, vb2);
  }
  if (lane == 0) {
    if (hrun > wbase) {
      sm.pidx[2 * warp + 1] = hrun - 1;
      sm.pseg[2 * warp + 1] = ca;
    } else if (ca.cnt > 0) {
      sm.pidx[2 * warp] = wbase - 1;  // no head in the chunk: it continues one run
      sm.pseg[2 * warp] = ca;
    }
  }
  __syncthreads();

  // ---- warp pieces -> runs of the tile (one warp, one piece per lane).
  if (warp == 0) {
    const int64_t idx = lane < 2 * kSoWarps ? sm.pidx[lane] : -1;
    Seg<NC> a;
    if (idx >= 0) a = sm.pseg[lane];
    else seg_identity<NC, SIG>(cs, a);
    int64_t mx = idx;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, mx, off);
      if (lane >= off) mx = max(mx, y);
    }
    int64_t before = __shfl_up_sync(0xffffffffu, mx, 1);
    if (lane == 0) before = -1;
    const bool head = idx >= 0 && idx > before;
    uint32_t tcf = 0;
    Seg<NC> tca, ex;
    seg_identity<NC, SIG>(cs, tca);
    warp_seg_scan<NC, SIG>(cs, head ? 1u : 0u, a, tcf, tca, ex);
    if (head && before >= 0) {
      if (before < excl_tile) piece_store<NC>(P, 2 * tile, before, ex);
      else if (before < cap) seg_emit<NC, SIG>(cs, o, before, ex);
    }
    const int64_t last = __shfl_sync(0xffffffffu, mx, 31);
    if (lane == 0 && last >= 0) piece_store<NC>(P, last < excl_tile ? 2 * tile : 2 * tile + 1, last, tca);
  }
}

__global__ void k_pieces_clear(int64_t* idx, int64_t m) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    idx[i] = -1;
}

// Merge pieces (nondecreasing run numbers; -1 = none) by run number.
// With Q.idx null one CTA walks every piece and writes every run.  Otherwise
// CTA b takes chunk b (blockDim pieces): the runs that start and end inside
// it are written, and its first and last runs -- which may continue in the
// neighbouring chunks -- become pieces 2b and 2b+1 of Q for a second pass.
template <int NC, uint32_t SIG>
__global__ void __launch_bounds__(kFixThreads) k_sorted_fix(ColSet cs, Pieces P, int64_t npieces, OutSet o,
                                                            int64_t cap, Pieces Q) {
  __shared__ SegScanSmem<NC, SIG> sm;
  __shared__ int64_t s_wmax[32];
  __shared__ int64_t s_cmax, s_first;
  const int lane = lane_id(), warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool level1 = Q.idx != nullptr;
  if (threadIdx.x == 0) {
    s_cmax = -1;
    s_first = -1;
  }
  uint32_t carry_f = 0;
  Seg<NC> carry_a;
  seg_identity<NC, SIG>(cs, carry_a);
  __syncthreads();
  const int64_t begin = level1 ? (int64_t)blockIdx.x * blockDim.x : 0;
  const int64_t end = level1 ? min(npieces, begin + (int64_t)blockDim.x) : npieces;
  for (int64_t base = begin; base < end; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int64_t idx = i < end ? P.idx[i] : -1;
    Seg<NC> a;
    if (idx >= 0) piece_load<NC>(P, i, a);
    else seg_identity<NC, SIG>(cs, a);
    // Exclusive running max of the run numbers (the run of the previous piece).
    int64_t inc = idx;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, inc, off);
      if (lane >= off) inc = max(inc, y);
    }
    if (lane == 31) s_wmax[warp] = inc;
    __syncthreads();
    int64_t before = s_cmax;
    for (int w = 0; w < warp; ++w) before = max(before, s_wmax[w]);
    int64_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) ex = -1;
    const int64_t runmax = max(before, ex);
    const bool head = idx >= 0 && idx > runmax;
    if (level1 && head && runmax < 0) s_first = idx;  // the chunk's first run (one thread)
    int64_t new_cmax = s_cmax;
    for (int w = 0; w < nw; ++w) new_cmax = max(new_cmax, s_wmax[w]);
    Seg<NC> ea;
    block_seg_scan<NC, SIG>(cs, head ? 1u : 0u, a, carry_f, carry_a, ea, sm);  // syncs: s_first visible
    if (head && runmax >= 0) {
      if (level1 && runmax == s_first) piece_store<NC>(Q, 2 * blockIdx.x, runmax, ea);
      else if (runmax < cap) seg_emit<NC, SIG>(cs, o, runmax, ea);
    }
    if (threadIdx.x == 0) s_cmax = new_cmax;
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_cmax >= 0) {
    if (level1) piece_store<NC>(Q, s_cmax == s_first ? 2 * blockIdx.x : 2 * blockIdx.x + 1, s_cmax, carry_a);
    else if (s_cmax < cap) seg_emit<NC, SIG>(cs, o, s_cmax, carry_a);
  }
}

template <int NC, uint32_t SIG>
int launch_sorted(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const uint32_t* vmask,
                  const uint64_t* prev, const Pieces& P, const Pieces& Q, int64_t ntiles, int64_t nchunks,
                  uint64_t* lb, uint32_t* ticket, int64_t* d_ng, int32_t* d_err, cudaStream_t s, StageTimer* tm) {
  const size_t smem = sizeof(SortedSmem<NC, SIG>);
  NFC_CUDA(cudaFuncSetAttribute(k_sorted_agg<NC, SIG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // Bulk copies need 16-byte aligned sources (the combined bitmap is ours).
  const bool bulk_ok = (reinterpret_cast<uintptr_t>(a->keys) & 15u) == 0 &&
                       (reinterpret_cast<uintptr_t>(vmask) & 15u) == 0;
  k_sorted_agg<NC, SIG><<<(unsigned)ntiles, kSoThreads, smem, s>>>(a->keys, vmask, cs, a->n, inputs_aligned(a),
                                                                   bulk_ok, prev, o, a->out_cap, P, lb, ticket,
                                                                   d_ng, d_err);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);
  Pieces none{};
  if (nchunks > 1) {
    k_sorted_fix<NC, SIG><<<(unsigned)nchunks, kFixThreads, 0, s>>>(cs, P, 2 * ntiles, o, a->out_cap, Q);
    NFC_CUDA(cudaGetLastError());
    k_sorted_fix<NC, SIG><<<1, kFixThreads, 0, s>>>(cs, Q, 2 * nchunks, o, a->out_cap, none);
    tm->launched(2);
  } else {
    k_sorted_fix<NC, SIG><<<1, kFixThreads, 0, s>>>(cs, P, 2 * ntiles, o, a->out_cap, none);
    tm->launched();
  }
  NFC_CUDA(cudaGetLastError());
  tm->mark(s);
  return NFC_OK;
}

constexpr uint32_t kSigI32SumMinMax_F64SumMinMax =
    sig_col(0, NFC_I32, NFC_AGG_SUM | NFC_AGG_MIN | NFC_AGG_MAX) | sig_col(1, NFC_F64, NFC_AGG_SUM | NFC_AGG_MIN | NFC_AGG_MAX);
constexpr uint32_t kSigI32Sum = sig_col(0, NFC_I32, NFC_AGG_SUM);

Pieces carve_pieces(uint64_t*& q, int64_t np) {
  Pieces P{};
  P.idx = reinterpret_cast<int64_t*>(q); q += np;
  P.cnt = q; q += np;
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    P.sum[c] = q; q += np;
    P.mn[c] = q; q += np;
    P.mx[c] = q; q += np;
  }
  return P;
}

}  // namespace

int run_sorted(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
               const uint32_t* vmask, const ProbeRec* recs, cudaStream_t s, Scratch& sc, int64_t* d_ng,
               int32_t* d_err, StageTimer* tm) {
  const int64_t n = a->n;
  const int64_t ntiles = (n + kSoTile - 1) / kSoTile;
  const int64_t nrec = (n + kProbeBlockRows - 1) / kProbeBlockRows;  // == ntiles
  const int64_t np = 2 * ntiles;
  const int64_t nchunks = (np + kFixThreads - 1) / kFixThreads;
  const int64_t nq = 2 * nchunks;
  // One allocation: prev[ntiles], lb[ntiles], ticket, tile pieces, chunk pieces.
  const size_t per_piece = 2 + 3 * NFC_MAX_COLS;
  const size_t words = (size_t)ntiles * 2 + 2 + (size_t)(np + nq) * per_piece;
  uint64_t* w = nullptr;
  NFC_CUDA(sc.alloc(&w, words));
  uint64_t* prev = w;
  uint64_t* lb = prev + ntiles;
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles);
  uint64_t* q = lb + ntiles + 2;
  const Pieces P = carve_pieces(q, np);
  const Pieces Q = carve_pieces(q, nq);
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * ((size_t)ntiles + 2), s));
  k_pieces_clear<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((np + 255) / 256, (int64_t)num_sms() * 4)), 256,
                   0, s>>>(P.idx, np);
  NFC_CUDA(cudaGetLastError());
  k_pieces_clear<<<1, 256, 0, s>>>(Q.idx, nq);
  NFC_CUDA(cudaGetLastError());
  k_sorted_prev<<<1, 1024, 0, s>>>(recs, nrec, prev);
  NFC_CUDA(cudaGetLastError());
  tm->launched(3);
  tm->mark(s);
  const uint32_t sig = sig_of(cs);
#define NFC_SORTED_LAUNCH(NCV, SIGV) \
  launch_sorted<NCV, SIGV>(a, cs, o, vmask, prev, P, Q, ntiles, nchunks, lb, ticket, d_ng, d_err, s, tm)
  switch (cs.ncols) {
    case 0: return NFC_SORTED_LAUNCH(0, 0);
    case 1:
      if (sig == kSigI32Sum) return NFC_SORTED_LAUNCH(1, kSigI32Sum);
      return NFC_SORTED_LAUNCH(1, 0);
    case 2:
      if (sig == kSigI32SumMinMax_F64SumMinMax) return NFC_SORTED_LAUNCH(2, kSigI32SumMinMax_F64SumMinMax);
      return NFC_SORTED_LAUNCH(2, 0);
    case 3: return NFC_SORTED_LAUNCH(3, 0);
    default: return NFC_SORTED_LAUNCH(4, 0);
  }
#undef NFC_SORTED_LAUNCH
}

}  // namespace nfc
