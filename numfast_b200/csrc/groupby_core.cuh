// Device building blocks of the group-by path: column descriptors, the
// 128-row warp tile loader (128-bit vector loads), aggregation state
// (identity, atomic apply, merge, decode) and the decoupled look-back
// used to place compacted groups.
#pragma once

#include <limits.h>

#include "nfc_common.cuh"

namespace nfc {

// Column set passed by value to every kernel (kernel params, uniform reads).
struct ColSet {
  int32_t ncols;
  int32_t dtype[NFC_MAX_COLS];
  int32_t aggs[NFC_MAX_COLS];
  const void* data[NFC_MAX_COLS];
};

NFC_HD int dtype_bytes(int dt) { return dt == NFC_I32 ? 4 : 8; }

// Compile-time column signature: column c uses bits [5c, 5c+2) for its
// dtype and [5c+2, 5c+5) for its NFC_AGG_* mask.  SIG == 0 means "read the
// dtype/aggs from the ColSet at run time" (generic instantiation).
constexpr uint32_t sig_col(int c, int dtype, int aggs) { return (uint32_t)(dtype | (aggs << 2)) << (5 * c); }
template <uint32_t SIG>
NFC_DEV int col_dt(const ColSet& cs, int c) {
  if constexpr (SIG != 0) return (int)((SIG >> (5 * c)) & 3u);
  else return cs.dtype[c];
}
template <uint32_t SIG>
NFC_DEV int col_ag(const ColSet& cs, int c) {
  if constexpr (SIG != 0) return (int)((SIG >> (5 * c + 2)) & 7u);
  else return cs.aggs[c];
}
static inline uint32_t sig_of(const ColSet& cs) {
  uint32_t s = 0;
  for (int c = 0; c < cs.ncols; ++c) s |= sig_col(c, cs.dtype[c], cs.aggs[c]);
  return s;
}

// ---------------------------------------------------------------------
// Aggregation state: SoA arrays of `slots` entries.
//   cnt       u32
//   sum[c]    i64 (integer columns) / f64
//   mn[c]     i32 / i64 / ordered-u64 (f64 MIN lane encoding)
//   mx[c]     i32 / i64 / ordered-u64 (f64 MAX lane encoding)
// The same layout is used in shared memory and in global memory.
// ---------------------------------------------------------------------
struct StateRef {
  uint32_t* cnt;
  void* sum[NFC_MAX_COLS];
  void* mn[NFC_MAX_COLS];
  void* mx[NFC_MAX_COLS];
};

// Bytes of state per slot for a column set.
static inline size_t state_bytes_per_slot(const ColSet& cs) {
  size_t b = 4;
  for (int c = 0; c < cs.ncols; ++c) {
    const int w = dtype_bytes(cs.dtype[c]);
    if (cs.aggs[c] & NFC_AGG_SUM) b += 8;
    if (cs.aggs[c] & NFC_AGG_MIN) b += w;
    if (cs.aggs[c] & NFC_AGG_MAX) b += w;
  }
  return b;
}

// Carve a StateRef for `slots` entries out of base (8-byte arrays first).
NFC_HD StateRef carve_state(const ColSet& cs, void* base, int64_t slots) {
  StateRef st;
  char* p = static_cast<char*>(base);
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    st.sum[c] = st.mn[c] = st.mx[c] = nullptr;
  }
  for (int c = 0; c < cs.ncols; ++c) {
    if (cs.aggs[c] & NFC_AGG_SUM) { st.sum[c] = p; p += 8 * slots; }
    if (dtype_bytes(cs.dtype[c]) == 8) {
      if (cs.aggs[c] & NFC_AGG_MIN) { st.mn[c] = p; p += 8 * slots; }
      if (cs.aggs[c] & NFC_AGG_MAX) { st.mx[c] = p; p += 8 * slots; }
    }
  }
  for (int c = 0; c < cs.ncols; ++c) {
    if (dtype_bytes(cs.dtype[c]) == 4) {
      if (cs.aggs[c] & NFC_AGG_MIN) { st.mn[c] = p; p += 4 * slots; }
      if (cs.aggs[c] & NFC_AGG_MAX) { st.mx[c] = p; p += 4 * slots; }
    }
  }
  st.cnt = reinterpret_cast<uint32_t*>(p);
  return st;
}

NFC_DEV void state_init_slot(const ColSet& cs, const StateRef& st, int64_t d) {
  st.cnt[d] = 0u;
#pragma unroll
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    if (c >= cs.ncols) break;
    const int dt = cs.dtype[c], ag = cs.aggs[c];
    if (ag & NFC_AGG_SUM) static_cast<uint64_t*>(st.sum[c])[d] = 0ull;
    if (dt == NFC_I32) {
      if (ag & NFC_AGG_MIN) static_cast<int32_t*>(st.mn[c])[d] = INT_MAX;
      if (ag & NFC_AGG_MAX) static_cast<int32_t*>(st.mx[c])[d] = INT_MIN;
    } else if (dt == NFC_I64) {
      if (ag & NFC_AGG_MIN) static_cast<int64_t*>(st.mn[c])[d] = LLONG_MAX;
      if (ag & NFC_AGG_MAX) static_cast<int64_t*>(st.mx[c])[d] = LLONG_MIN;
    } else {
      if (ag & NFC_AGG_MIN) static_cast<uint64_t*>(st.mn[c])[d] = ~0ull;
      if (ag & NFC_AGG_MAX) static_cast<uint64_t*>(st.mx[c])[d] = 0ull;
    }
  }
}

// Fold one row (raw value bits per column) into slot d.  Integer values
// arrive sign-extended to 64 bits; float64 values as their bit pattern.
NFC_DEV void state_apply(const ColSet& cs, const StateRef& st, int64_t d, const uint64_t* raw) {
  atomicAdd(&st.cnt[d], 1u);
#pragma unroll
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    if (c >= cs.ncols) break;
    const int dt = cs.dtype[c], ag = cs.aggs[c];
    const uint64_t r = raw[c];
    if (dt == NFC_F64) {
      if (ag & NFC_AGG_SUM) atomicAdd(static_cast<double*>(st.sum[c]) + d, __longlong_as_double((long long)r));
      if (ag & NFC_AGG_MIN)
        atomicMin(static_cast<unsigned long long*>(st.mn[c]) + d, (unsigned long long)f64_min_enc(r));
      if (ag & NFC_AGG_MAX)
        atomicMax(static_cast<unsigned long long*>(st.mx[c]) + d, (unsigned long long)f64_max_enc(r));
    } else {
      if (ag & NFC_AGG_SUM) atomicAdd(static_cast<unsigned long long*>(st.sum[c]) + d, (unsigned long long)r);
      if (dt == NFC_I32) {
        if (ag & NFC_AGG_MIN) atomicMin(static_cast<int*>(st.mn[c]) + d, (int)(int64_t)r);
        if (ag & NFC_AGG_MAX) atomicMax(static_cast<int*>(st.mx[c]) + d, (int)(int64_t)r);
      } else {
        if (ag & NFC_AGG_MIN) atomicMin(static_cast<long long*>(st.mn[c]) + d, (long long)r);
        if (ag & NFC_AGG_MAX) atomicMax(static_cast<long long*>(st.mx[c]) + d, (long long)r);
      }
    }
  }
}

// Fold a combined row group -- k rows with the given per-column sums (int64
// bits / float64 bits), minima and maxima (int64 / ordered float64 lanes) --
// into slot d with one set of atomics.
NFC_DEV void state_apply_group(const ColSet& cs, const StateRef& st, int64_t d, uint32_t k, const uint64_t* sum,
                               const uint64_t* mn, const uint64_t* mx) {
  atomicAdd(&st.cnt[d], k);
#pragma unroll
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    if (c >= cs.ncols) break;
    const int dt = cs.dtype[c], ag = cs.aggs[c];
    if (dt == NFC_F64) {
      if (ag & NFC_AGG_SUM) atomicAdd(static_cast<double*>(st.sum[c]) + d, __longlong_as_double((long long)sum[c]));
      if (ag & NFC_AGG_MIN) atomicMin(static_cast<unsigned long long*>(st.mn[c]) + d, (unsigned long long)mn[c]);
      if (ag & NFC_AGG_MAX) atomicMax(static_cast<unsigned long long*>(st.mx[c]) + d, (unsigned long long)mx[c]);
    } else {
      if (ag & NFC_AGG_SUM) atomicAdd(static_cast<unsigned long long*>(st.sum[c]) + d, (unsigned long long)sum[c]);
      if (dt == NFC_I32) {
        if (ag & NFC_AGG_MIN) atomicMin(static_cast<int*>(st.mn[c]) + d, (int)(long long)mn[c]);
        if (ag & NFC_AGG_MAX) atomicMax(static_cast<int*>(st.mx[c]) + d, (int)(long long)mx[c]);
      } else {
        if (ag & NFC_AGG_MIN) atomicMin(static_cast<long long*>(st.mn[c]) + d, (long long)mn[c]);
        if (ag & NFC_AGG_MAX) atomicMax(static_cast<long long*>(st.mx[c]) + d, (long long)mx[c]);
      }
    }
  }
}

// Warp-aggregated rows, called by all 32 lanes (active = the lane has a
// row).  Lanes holding the same key find each other with __match_any_sync;
// a lane alone with its key hands its row to apply_row(key, raw), and each
// group of equal keys is reduced with warp reductions and handed once, by its
// lowest lane, to apply_group(key, k, sum, mn, mx) (k rows; per column the
// int64 / float64-bit sum and the int64 / ordered-float64 min and max) -- so a
// hot key or a run of one key costs one update per warp instead of one per
// row.  At most kWarpAggRounds groups are reduced per call; lanes of further
// groups apply their own rows.
constexpr int kWarpAggRounds = 4;

template <int NC, uint32_t SIG, class GroupF, class RowF>
NFC_DEV void warp_agg_rows(const ColSet& cs, bool active, int32_t key, const uint64_t* raw, GroupF&& apply_group,
                           RowF&& apply_row) {
  constexpr int M = NC > 0 ? NC : 1;
  const unsigned lane = lane_id();
  const unsigned act = __ballot_sync(0xffffffffu, active);
  if (act == 0u) return;
  const unsigned peers = __match_any_sync(0xffffffffu, key) & act;
  const bool solo = active && peers == (1u << lane);
  unsigned todo = __ballot_sync(0xffffffffu, active && !solo);
  for (int round = 0; round < kWarpAggRounds && todo; ++round) {
    const int leader = __ffs(todo) - 1;
    const unsigned grp = __shfl_sync(0xffffffffu, peers, leader);
    const bool in = (grp >> lane) & 1u;
    uint64_t sum[M], mn[M], mx[M];
#pragma unroll
    for (int c = 0; c < M; ++c) {
      sum[c] = 0;
      mn[c] = mx[c] = 0;
      if (c >= NC || (SIG == 0 && c >= cs.ncols)) continue;
      const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
      const uint64_t r = raw[c];
      if (dt == NFC_I32) {
        const int32_t v = (int32_t)(uint32_t)r;
        if (ag & NFC_AGG_SUM) {
          // Two exact 32-bit reductions of the 16-bit halves (32 lanes).
          const int lo = __reduce_add_sync(0xffffffffu, in ? (int)(v & 0xFFFF) : 0);
          const int hi = __reduce_add_sync(0xffffffffu, in ? (v >> 16) : 0);
          sum[c] = (uint64_t)((int64_t)hi * 65536 + (int64_t)lo);
        }
        if (ag & NFC_AGG_MIN) mn[c] = (uint64_t)(int64_t)__reduce_min_sync(0xffffffffu, in ? v : INT_MAX);
        if (ag & NFC_AGG_MAX) mx[c] = (uint64_t)(int64_t)__reduce_max_sync(0xffffffffu, in ? v : INT_MIN);
      } else if (dt == NFC_I64) {
        uint64_t s = in ? r : 0ull;
        long long lo = in ? (long long)r : LLONG_MAX, hi = in ? (long long)r : LLONG_MIN;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          s += __shfl_xor_sync(0xffffffffu, s, o);
          lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
          hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        sum[c] = s;
        mn[c] = (uint64_t)lo;
        mx[c] = (uint64_t)hi;
      } else {
        double s = in ? __longlong_as_double((long long)r) : 0.0;
        uint64_t lo = in ? f64_min_enc(r) : ~0ull, hi = in ? f64_max_enc(r) : 0ull;
        if (ag & NFC_AGG_SUM) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        }
        if (ag & (NFC_AGG_MIN | NFC_AGG_MAX)) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
          }
        }
        sum[c] = (uint64_t)__double_as_longlong(s);
        mn[c] = lo;
        mx[c] = hi;
      }
    }
    if ((int)lane == leader) apply_group(key, (uint32_t)__popc(grp), sum, mn, mx);
    todo &= ~grp;
  }
  if (solo || ((todo >> lane) & 1u)) apply_row(key, raw);
}

// Warp-aggregated update of a global state: slot_of(key) gives the slot
// (called only by lanes that apply; -1 skips).
template <class SlotF>
NFC_DEV void warp_agg_apply(const ColSet& cs, const StateRef& st, bool active, int32_t key, const uint64_t* raw,
                            SlotF&& slot_of) {
  warp_agg_rows<NFC_MAX_COLS, 0>(
      cs, active, key, raw,
      [&](int32_t k, uint32_t cnt, const uint64_t* sum, const uint64_t* mn, const uint64_t* mx) {
        const int64_t d = slot_of(k);
        if (d >= 0) state_apply_group(cs, st, d, cnt, sum, mn, mx);
      },
      [&](int32_t k, const uint64_t* r) {
        const int64_t d = slot_of(k);
        if (d >= 0) state_apply(cs, st, d, r);
      });
}

// Merge slot s of `src` into slot d of `dst` (dst shared by many CTAs).
NFC_DEV void state_merge(const ColSet& cs, const StateRef& dst, int64_t d, const StateRef& src, int64_t s) {
  const uint32_t k = src.cnt[s];
  if (k == 0u) return;
  atomicAdd(&dst.cnt[d], k);
#pragma unroll
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    if (c >= cs.ncols) break;
    const int dt = cs.dtype[c], ag = cs.aggs[c];
    if (dt == NFC_F64) {
      if (ag & NFC_AGG_SUM) atomicAdd(static_cast<double*>(dst.sum[c]) + d, static_cast<const double*>(src.sum[c])[s]);
      if (ag & NFC_AGG_MIN)
        atomicMin(static_cast<unsigned long long*>(dst.mn[c]) + d, static_cast<const unsigned long long*>(src.mn[c])[s]);
      if (ag & NFC_AGG_MAX)
        atomicMax(static_cast<unsigned long long*>(dst.mx[c]) + d, static_cast<const unsigned long long*>(src.mx[c])[s]);
    } else {
      if (ag & NFC_AGG_SUM)
        atomicAdd(static_cast<unsigned long long*>(dst.sum[c]) + d, static_cast<const unsigned long long*>(src.sum[c])[s]);
      if (dt == NFC_I32) {
        if (ag & NFC_AGG_MIN) atomicMin(static_cast<int*>(dst.mn[c]) + d, static_cast<const int*>(src.mn[c])[s]);
        if (ag & NFC_AGG_MAX) atomicMax(static_cast<int*>(dst.mx[c]) + d, static_cast<const int*>(src.mx[c])[s]);
      } else {
        if (ag & NFC_AGG_MIN) atomicMin(static_cast<long long*>(dst.mn[c]) + d, static_cast<const long long*>(src.mn[c])[s]);
        if (ag & NFC_AGG_MAX) atomicMax(static_cast<long long*>(dst.mx[c]) + d, static_cast<const long long*>(src.mx[c])[s]);
      }
    }
  }
}

// Output pointers of one group-by call.
struct OutSet {
  int64_t* ukeys;
  int64_t* counts;
  void* sum[NFC_MAX_COLS];
  void* mn[NFC_MAX_COLS];
  void* mx[NFC_MAX_COLS];
};

// Write compacted group `pos` from state slot s (key value `key`).
NFC_DEV void state_emit(const ColSet& cs, const StateRef& st, int64_t s, const OutSet& o, int64_t pos, int64_t key) {
  o.ukeys[pos] = key;
  o.counts[pos] = static_cast<int64_t>(st.cnt[s]);
#pragma unroll
  for (int c = 0; c < NFC_MAX_COLS; ++c) {
    if (c >= cs.ncols) break;
    const int dt = cs.dtype[c], ag = cs.aggs[c];
    if (ag & NFC_AGG_SUM) static_cast<uint64_t*>(o.sum[c])[pos] = static_cast<const uint64_t*>(st.sum[c])[s];
    if (dt == NFC_I32) {
      if (ag & NFC_AGG_MIN) static_cast<int32_t*>(o.mn[c])[pos] = static_cast<const int32_t*>(st.mn[c])[s];
      if (ag & NFC_AGG_MAX) static_cast<int32_t*>(o.mx[c])[pos] = static_cast<const int32_t*>(st.mx[c])[s];
    } else if (dt == NFC_I64) {
      if (ag & NFC_AGG_MIN) static_cast<int64_t*>(o.mn[c])[pos] = static_cast<const int64_t*>(st.mn[c])[s];
      if (ag & NFC_AGG_MAX) static_cast<int64_t*>(o.mx[c])[pos] = static_cast<const int64_t*>(st.mx[c])[s];
    } else {
      if (ag & NFC_AGG_MIN) static_cast<uint64_t*>(o.mn[c])[pos] = f64_min_dec(static_cast<const uint64_t*>(st.mn[c])[s]);
      if (ag & NFC_AGG_MAX) static_cast<uint64_t*>(o.mx[c])[pos] = f64_max_dec(static_cast<const uint64_t*>(st.mx[c])[s]);
    }
  }
}

// ---------------------------------------------------------------------
// 128-row warp tile: lane l owns rows base + 4l .. base + 4l + 3.
// Keys and 4-byte values use one 128-bit load per lane; 8-byte values two.
// `vmask` is the combined validity bitmap (u32 words, LSB = first row) or
// null when every row is valid.
// ---------------------------------------------------------------------
template <int NC>
struct TileT {
  int32_t key[4];
  uint32_t valid;  // bit r = row r of this lane is valid
  uint64_t raw[NC > 0 ? NC : 1][4];
};
using Tile4 = TileT<NFC_MAX_COLS>;

template <bool LOAD_VALUES, int NC = NFC_MAX_COLS, uint32_t SIG = 0>
NFC_DEV void load_tile4_full(const int32_t* __restrict__ keys, const uint32_t* __restrict__ vmask,
                             const ColSet& cs, int64_t row0, TileT<NC>& t) {
  const int4 k = __ldcs(reinterpret_cast<const int4*>(keys + row0));
  t.key[0] = k.x; t.key[1] = k.y; t.key[2] = k.z; t.key[3] = k.w;
  if (vmask) {
    const uint32_t w = __ldg(vmask + (row0 >> 5));
    t.valid = (w >> (row0 & 31)) & 0xFu;
  } else {
    t.valid = 0xFu;
  }
  if (LOAD_VALUES) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (SIG == 0 && c >= cs.ncols) break;
      if (col_dt<SIG>(cs, c) == NFC_I32) {
        const int4 v = __ldcs(reinterpret_cast<const int4*>(static_cast<const int32_t*>(cs.data[c]) + row0));
        t.raw[c][0] = (uint64_t)(int64_t)v.x; t.raw[c][1] = (uint64_t)(int64_t)v.y;
        t.raw[c][2] = (uint64_t)(int64_t)v.z; t.raw[c][3] = (uint64_t)(int64_t)v.w;
      } else {
        const ulonglong2* p = reinterpret_cast<const ulonglong2*>(static_cast<const uint64_t*>(cs.data[c]) + row0);
        const ulonglong2 a = __ldcs(p), b = __ldcs(p + 1);
        t.raw[c][0] = a.x; t.raw[c][1] = a.y; t.raw[c][2] = b.x; t.raw[c][3] = b.y;
      }
    }
  }
}

// Scalar loader for the ragged tail (rows >= n are invalid).
template <bool LOAD_VALUES, int NC = NFC_MAX_COLS, uint32_t SIG = 0>
NFC_DEV void load_tile4_tail(const int32_t* __restrict__ keys, const uint32_t* __restrict__ vmask,
                             const ColSet& cs, int64_t row0, int64_t n, TileT<NC>& t) {
  t.valid = 0u;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int64_t i = row0 + r;
    t.key[r] = 0;
    if (i < n) {
      t.key[r] = keys[i];
      const bool v = vmask ? ((vmask[i >> 5] >> (i & 31)) & 1u) : true;
      t.valid |= (v ? 1u : 0u) << r;
      if (LOAD_VALUES) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          if (SIG == 0 && c >= cs.ncols) break;
          t.raw[c][r] = col_dt<SIG>(cs, c) == NFC_I32
                            ? (uint64_t)(int64_t) static_cast<const int32_t*>(cs.data[c])[i]
                            : static_cast<const uint64_t*>(cs.data[c])[i];
        }
      }
    } else if (LOAD_VALUES) {
#pragma unroll
      for (int c = 0; c < NC; ++c) t.raw[c][r] = 0;
    }
  }
}

// ---------------------------------------------------------------------
// Decoupled look-back over an ordered sequence of tiles.  Status word:
// bits 62-63 flag (0 none, 1 aggregate, 2 inclusive prefix), bits 0-61
// value.  Called by one full warp per tile; returns the exclusive prefix.
// A predecessor that never publishes ends the wait after kSpinLimit polls
// with *err = NFC_ERR_TIMEOUT (the tile then uses a partial prefix; the
// call reports the error instead of hanging).
// ---------------------------------------------------------------------
constexpr uint64_t kLbAgg = 1ull << 62;
constexpr uint64_t kLbInc = 2ull << 62;
constexpr uint64_t kLbVal = (1ull << 62) - 1;

NFC_DEV void lb_store(uint64_t* p, uint64_t v) {
  __threadfence();
  atomicExch(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}

// Decoupled look-back run by ONE FULL WARP (all 32 lanes call it; every lane
// gets the exclusive prefix; lane 0 publishes).  Lane i reads the status of
// tile j - i, so one round covers 32 predecessors with independent loads
// instead of one dependent L2 round trip per tile -- what bounds a serial
// walk when a whole wave of tiles starts together.  Statuses up to the
// nearest inclusive one are summed with a warp reduction; if one of them has
// not been published yet, the published run before it is consumed and the
// walk polls again from there.
NFC_DEV int64_t lookback_exclusive(uint64_t* status, int64_t tile, uint64_t aggregate, int32_t* err,
                                   uint32_t spin_limit = kSpinLimit) {
  const unsigned lane = lane_id();
  if (tile == 0) {
    if (lane == 0) lb_store(status, kLbInc | aggregate);
    return 0;
  }
  if (lane == 0) lb_store(status + tile, kLbAgg | aggregate);
  uint64_t excl = 0;
  int64_t j = tile - 1;  // nearest predecessor not yet accounted for
  uint32_t spins = 0;
  while (true) {
    const int64_t t = j - (int64_t)lane;
    // Lanes past tile 0 read as an inclusive zero: tile 0 ends every walk.
    const uint64_t w = t >= 0 ? ld_volatile_u64(status + t) : kLbInc;
    const uint64_t flag = w & ~kLbVal;
    const unsigned inc = __ballot_sync(0xffffffffu, flag == kLbInc);
    const unsigned pending = __ballot_sync(0xffffffffu, flag == 0);
    const unsigned upto = inc ? (((inc & (0u - inc)) << 1) - 1u) : 0xffffffffu;  // lanes 0 .. first inclusive
    const unsigned wait = pending & upto;
    const int take = wait ? __ffs(wait) - 1 : 32;  // lanes before the first unpublished one
    const uint64_t v = (int)lane < take && ((upto >> lane) & 1u) ? (w & kLbVal) : 0ull;
    excl += warp_sum(v);
    if (!wait && inc) break;
    if (take == 0 && ++spins > spin_limit) {
      if (lane == 0) atomicExch(err, NFC_ERR_TIMEOUT);
      break;
    }
    j -= take;
  }
  if (lane == 0) {
    __threadfence();
    lb_store(status + tile, kLbInc | (excl + aggregate));
  }
  return static_cast<int64_t>(excl);
}

// Block-wide exclusive scan of one u32 per thread (blockDim multiple of 32,
// <= 1024).  `smem` needs 33 words.  Returns exclusive prefix; *total gets
// the block sum.
NFC_DEV uint32_t block_excl_scan(uint32_t v, uint32_t* smem, uint32_t* total) {
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nw ? smem[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (unsigned)o) s += y;
    }
    if (lane < nw) smem[lane] = s;  // inclusive per-warp
    if (lane == nw - 1) smem[32] = s;
  }
  __syncthreads();
  const uint32_t warp_excl = warp ? smem[warp - 1] : 0u;
  *total = smem[32];
  __syncthreads();
  return warp_excl + x - v;
}

}  // namespace nfc
