// Shared-memory aggregation state for one CTA's groups, shared by the
// partition aggregate and the shared-hash strategy.
//
// 64-bit shared-memory atomics on integers are emulated, so an int32
// column's sum is kept as two native 32-bit sums of its low and high 16-bit
// halves (exact while a state slot sees at most 65,536 rows) -- or, when
// the caller knows every value of the column lies in [-32767, 32767]
// (bit c of `narrow`), as one signed 32-bit sum in the low array (exact for
// the same 65,536 rows); float64
// min/max use native 64-bit min/max on an order-preserving encoding;
// float64 sums use the 64-bit float add.  agg_merge folds a slot into the
// global state layout (StateRef) with global atomics.
#pragma once

#include "groupby_core.cuh"

namespace nfc {

template <int NC>
struct AggState {
  uint32_t* cnt;
  uint32_t* slo[NC > 0 ? NC : 1];   // int32 columns: sum of low 16-bit halves
  int32_t* shi[NC > 0 ? NC : 1];    // int32 columns: sum of high 16-bit halves
  uint64_t* s64[NC > 0 ? NC : 1];   // int64 / float64 columns: sum
  void* mn[NC > 0 ? NC : 1];
  void* mx[NC > 0 ? NC : 1];
  uint32_t narrow;  // bit c: int32 column c summed with one signed 32-bit atomic
};

template <int NC, uint32_t SIG>
NFC_DEV AggState<NC> carve_agg(const ColSet& cs, unsigned char* base, int w, uint32_t narrow = 0u) {
  AggState<NC> st;
  st.narrow = narrow;
  unsigned char* p = base;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    st.slo[c] = nullptr; st.shi[c] = nullptr; st.s64[c] = nullptr; st.mn[c] = nullptr; st.mx[c] = nullptr;
    const bool wide = col_dt<SIG>(cs, c) != NFC_I32;
    const int ag = col_ag<SIG>(cs, c);
    if (wide && (ag & NFC_AGG_SUM)) { st.s64[c] = reinterpret_cast<uint64_t*>(p); p += 8 * w; }
    if (wide && (ag & NFC_AGG_MIN)) { st.mn[c] = p; p += 8 * w; }
    if (wide && (ag & NFC_AGG_MAX)) { st.mx[c] = p; p += 8 * w; }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (col_dt<SIG>(cs, c) != NFC_I32) continue;
    const int ag = col_ag<SIG>(cs, c);
    if (ag & NFC_AGG_SUM) {
      st.slo[c] = reinterpret_cast<uint32_t*>(p); p += 4 * w;
      st.shi[c] = reinterpret_cast<int32_t*>(p); p += 4 * w;
    }
    if (ag & NFC_AGG_MIN) { st.mn[c] = p; p += 4 * w; }
    if (ag & NFC_AGG_MAX) { st.mx[c] = p; p += 4 * w; }
  }
  st.cnt = reinterpret_cast<uint32_t*>(p);
  return st;
}

template <int NC, uint32_t SIG>
NFC_DEV void agg_init(const ColSet& cs, const AggState<NC>& st, int g) {
  st.cnt[g] = 0u;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    if (dt == NFC_I32) {
      if (ag & NFC_AGG_SUM) { st.slo[c][g] = 0u; st.shi[c][g] = 0; }
      if (ag & NFC_AGG_MIN) static_cast<int32_t*>(st.mn[c])[g] = INT_MAX;
      if (ag & NFC_AGG_MAX) static_cast<int32_t*>(st.mx[c])[g] = INT_MIN;
    } else {
      if (ag & NFC_AGG_SUM) st.s64[c][g] = 0ull;
      if (dt == NFC_I64) {
        if (ag & NFC_AGG_MIN) static_cast<int64_t*>(st.mn[c])[g] = LLONG_MAX;
        if (ag & NFC_AGG_MAX) static_cast<int64_t*>(st.mx[c])[g] = LLONG_MIN;
      } else {
        if (ag & NFC_AGG_MIN) static_cast<uint64_t*>(st.mn[c])[g] = ~0ull;
        if (ag & NFC_AGG_MAX) static_cast<uint64_t*>(st.mx[c])[g] = 0ull;
      }
    }
  }
}

// READ_FIRST: min/max read the slot first and skip the atomic when the value
// cannot win (the stored extreme only moves one way, so a value that does
// not beat it now can never beat the final one).  That pays when slots see
// many rows each; with a few rows per slot (the partition aggregate: ~8 on
// average) the read costs more shared-memory wavefronts than the atomics it
// saves, so that caller issues the atomics directly.
template <int NC, uint32_t SIG, bool READ_FIRST = true>
NFC_DEV void agg_apply(const ColSet& cs, const AggState<NC>& st, uint32_t g, const uint64_t* raw) {
  atomicAdd(&st.cnt[g], 1u);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    const uint64_t r = raw[c];
    if (dt == NFC_I32) {
      const int32_t v = (int32_t)(uint32_t)r;
      if (ag & NFC_AGG_SUM) {
        if ((st.narrow >> c) & 1u) {
          atomicAdd(reinterpret_cast<int*>(st.slo[c]) + g, v);
        } else {
          atomicAdd(&st.slo[c][g], (uint32_t)v & 0xFFFFu);
          atomicAdd(&st.shi[c][g], v >> 16);
        }
      }
      if ((ag & NFC_AGG_MIN) && (!READ_FIRST || v < static_cast<volatile int32_t*>(st.mn[c])[g]))
        atomicMin(static_cast<int*>(st.mn[c]) + g, v);
      if ((ag & NFC_AGG_MAX) && (!READ_FIRST || v > static_cast<volatile int32_t*>(st.mx[c])[g]))
        atomicMax(static_cast<int*>(st.mx[c]) + g, v);
    } else if (dt == NFC_I64) {
      if (ag & NFC_AGG_SUM) atomicAdd(reinterpret_cast<unsigned long long*>(st.s64[c]) + g, (unsigned long long)r);
      if ((ag & NFC_AGG_MIN) && (!READ_FIRST || (long long)r < static_cast<volatile long long*>(st.mn[c])[g]))
        atomicMin(static_cast<long long*>(st.mn[c]) + g, (long long)r);
      if ((ag & NFC_AGG_MAX) && (!READ_FIRST || (long long)r > static_cast<volatile long long*>(st.mx[c])[g]))
        atomicMax(static_cast<long long*>(st.mx[c]) + g, (long long)r);
    } else {
      if (ag & NFC_AGG_SUM) atomicAdd(reinterpret_cast<double*>(st.s64[c]) + g, __longlong_as_double((long long)r));
      if (ag & NFC_AGG_MIN) {
        const unsigned long long e = f64_min_enc(r);
        if (!READ_FIRST || e < static_cast<volatile unsigned long long*>(st.mn[c])[g])
          atomicMin(static_cast<unsigned long long*>(st.mn[c]) + g, e);
      }
      if (ag & NFC_AGG_MAX) {
        const unsigned long long e = f64_max_enc(r);
        if (!READ_FIRST || e > static_cast<volatile unsigned long long*>(st.mx[c])[g])
          atomicMax(static_cast<unsigned long long*>(st.mx[c]) + g, e);
      }
    }
  }
}

// Fold k rows combined by warp_agg_rows (sums as int64 / float64 bits,
// minima / maxima as int64 / ordered float64 lanes) into slot g.  An int32
// sum goes into the split halves as its own low 16 bits and the rest, which
// keeps value = high * 65536 + low and the same bounds as k single rows.
template <int NC, uint32_t SIG>
NFC_DEV void agg_apply_group(const ColSet& cs, const AggState<NC>& st, uint32_t g, uint32_t k, const uint64_t* sum,
                             const uint64_t* mn, const uint64_t* mx) {
  atomicAdd(&st.cnt[g], k);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    if (dt == NFC_I32) {
      if (ag & NFC_AGG_SUM) {
        const int64_t s = (int64_t)sum[c];
        if ((st.narrow >> c) & 1u) {
          atomicAdd(reinterpret_cast<int*>(st.slo[c]) + g, (int)s);
        } else {
          atomicAdd(&st.slo[c][g], (uint32_t)(s & 0xFFFF));
          atomicAdd(&st.shi[c][g], (int32_t)(s >> 16));
        }
      }
      if (ag & NFC_AGG_MIN) atomicMin(static_cast<int*>(st.mn[c]) + g, (int)(int64_t)mn[c]);
      if (ag & NFC_AGG_MAX) atomicMax(static_cast<int*>(st.mx[c]) + g, (int)(int64_t)mx[c]);
    } else if (dt == NFC_I64) {
      if (ag & NFC_AGG_SUM) atomicAdd(reinterpret_cast<unsigned long long*>(st.s64[c]) + g, (unsigned long long)sum[c]);
      if (ag & NFC_AGG_MIN) atomicMin(static_cast<long long*>(st.mn[c]) + g, (long long)mn[c]);
      if (ag & NFC_AGG_MAX) atomicMax(static_cast<long long*>(st.mx[c]) + g, (long long)mx[c]);
    } else {
      if (ag & NFC_AGG_SUM) atomicAdd(reinterpret_cast<double*>(st.s64[c]) + g, __longlong_as_double((long long)sum[c]));
      if (ag & NFC_AGG_MIN) atomicMin(static_cast<unsigned long long*>(st.mn[c]) + g, (unsigned long long)mn[c]);
      if (ag & NFC_AGG_MAX) atomicMax(static_cast<unsigned long long*>(st.mx[c]) + g, (unsigned long long)mx[c]);
    }
  }
}

template <int NC, uint32_t SIG>
NFC_DEV int64_t agg_sum_bits(const ColSet& cs, const AggState<NC>& st, int c, int g) {
  if (col_dt<SIG>(cs, c) == NFC_I32) {
    if ((st.narrow >> c) & 1u) return (int64_t)(int32_t)st.slo[c][g];
    return (int64_t)st.shi[c][g] * 65536 + (int64_t)st.slo[c][g];
  }
  return (int64_t)st.s64[c][g];
}

// Merge shared slot g into the global merge state (StateRef layout) slot d.
template <int NC, uint32_t SIG>
NFC_DEV void agg_merge(const ColSet& cs, const StateRef& dst, int64_t d, const AggState<NC>& st, int g) {
  const uint32_t k = st.cnt[g];
  if (k == 0u) return;
  atomicAdd(&dst.cnt[d], k);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    if (ag & NFC_AGG_SUM) {
      if (dt == NFC_F64) atomicAdd(static_cast<double*>(dst.sum[c]) + d, __longlong_as_double((long long)st.s64[c][g]));
      else atomicAdd(static_cast<unsigned long long*>(dst.sum[c]) + d, (unsigned long long)agg_sum_bits<NC, SIG>(cs, st, c, g));
    }
    if (dt == NFC_I32) {
      if (ag & NFC_AGG_MIN) atomicMin(static_cast<int*>(dst.mn[c]) + d, static_cast<const int*>(st.mn[c])[g]);
      if (ag & NFC_AGG_MAX) atomicMax(static_cast<int*>(dst.mx[c]) + d, static_cast<const int*>(st.mx[c])[g]);
    } else if (dt == NFC_I64) {
      if (ag & NFC_AGG_MIN) atomicMin(static_cast<long long*>(dst.mn[c]) + d, static_cast<const long long*>(st.mn[c])[g]);
      if (ag & NFC_AGG_MAX) atomicMax(static_cast<long long*>(dst.mx[c]) + d, static_cast<const long long*>(st.mx[c])[g]);
    } else {
      if (ag & NFC_AGG_MIN)
        atomicMin(static_cast<unsigned long long*>(dst.mn[c]) + d, static_cast<const unsigned long long*>(st.mn[c])[g]);
      if (ag & NFC_AGG_MAX)
        atomicMax(static_cast<unsigned long long*>(dst.mx[c]) + d, static_cast<const unsigned long long*>(st.mx[c])[g]);
    }
  }
}

template <int NC, uint32_t SIG>
NFC_DEV void agg_emit(const ColSet& cs, const AggState<NC>& st, int g, const OutSet& o, int64_t pos, int64_t key) {
  o.ukeys[pos] = key;
  o.counts[pos] = (int64_t)st.cnt[g];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int dt = col_dt<SIG>(cs, c), ag = col_ag<SIG>(cs, c);
    if (ag & NFC_AGG_SUM) static_cast<int64_t*>(o.sum[c])[pos] = agg_sum_bits<NC, SIG>(cs, st, c, g);
    if (dt == NFC_I32) {
      if (ag & NFC_AGG_MIN) static_cast<int32_t*>(o.mn[c])[pos] = static_cast<const int32_t*>(st.mn[c])[g];
      if (ag & NFC_AGG_MAX) static_cast<int32_t*>(o.mx[c])[pos] = static_cast<const int32_t*>(st.mx[c])[g];
    } else if (dt == NFC_I64) {
      if (ag & NFC_AGG_MIN) static_cast<int64_t*>(o.mn[c])[pos] = static_cast<const int64_t*>(st.mn[c])[g];
      if (ag & NFC_AGG_MAX) static_cast<int64_t*>(o.mx[c])[pos] = static_cast<const int64_t*>(st.mx[c])[g];
    } else {
      if (ag & NFC_AGG_MIN) static_cast<uint64_t*>(o.mn[c])[pos] = f64_min_dec(static_cast<const uint64_t*>(st.mn[c])[g]);
      if (ag & NFC_AGG_MAX) static_cast<uint64_t*>(o.mx[c])[pos] = f64_max_dec(static_cast<const uint64_t*>(st.mx[c])[g]);
    }
  }
}

}  // namespace nfc
