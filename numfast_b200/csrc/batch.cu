// Batched group-by: thousands of independent `group(key, {v: (sum, count)})`
// queries over one concatenated int32 key column and one int32 value column,
// run by ONE persistent kernel (optionally replayed from a CUDA graph).
//
// Per query the arithmetic is the executor's groupby_multi branch with ops
// ("sum", "count") on one int32 value column (src/Drivers/CPU/_lib/cpu.py:
// 3435-3704): rows whose key or value is NULL are dropped (_valid_mask,
// cpu.py:1374-1382), groups come out in ascending key order, counts and sums
// are int64.  The batch itself has no counterpart in the reference, which
// runs one query per executor node.
//
// Work is a static list of items built on the host, claimed in list order
// through one global ticket.  Items of a query depend only on items that
// come earlier in the list, so the smallest unfinished item is always being
// executed by a resident CTA and every bounded wait ends:
//   PROBE (query, chunk)  key min/max/valid count -> the last one plans the
//                         query (dense span, shared-memory or global state,
//                         state slice of the arena, output reservation)
//   SOLO  (query)         a small query done start to finish by one CTA
//   AGG   (query, chunk)  rows -> shared-memory table flushed to the global
//                         state, or warp-aggregated global reductions
//   EMIT  (query, slice)  state slice -> compacted ascending groups, with a
//                         decoupled look-back across the query's slices;
//                         the slice is cleared so the arena stays zero.
//
// Global state: one u64 per key slot holding count << SH plus the signed sum
// (SH = 64 - bitlen(rows)); a query whose |value| * rows could reach
// 2^(SH-1) is flagged and finished by the single-query path on the host,
// like any query whose span or reservation does not fit (deferred).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "groupby_core.cuh"
#include "groupby_host.h"

namespace nfc {
namespace {

constexpr int kBThreads = 512;
constexpr int kBWarps = kBThreads / 32;
constexpr int kBPer = 16;                    // rows per thread per sub-tile
constexpr int kBSub = kBThreads * kBPer;     // 8192 rows per sub-tile
constexpr int kBEmitRound = kBThreads * 4;   // slots per emit round

enum : uint32_t { kItProbe = 0, kItSolo = 1, kItAgg = 2, kItEmit = 3 };

struct QDesc {
  int64_t row_off;
  int64_t rows;
  uint32_t n_probe;
  uint32_t n_agg;
  uint32_t n_emit;
  uint32_t emit_slice;
  uint32_t lb_base;
  uint32_t solo;
  uint32_t chunk;  // rows per aggregate item of this query
  uint32_t pad1;
};
static_assert(sizeof(QDesc) == 48, "QDesc layout");

// Per-query runtime state, zeroed before every launch.
struct QRt {
  uint32_t kmax_o;   // max over valid keys of (key ^ 0x80000000)
  uint32_t kmin_c;   // max over valid keys of ~(key ^ 0x80000000)
  uint32_t nvalid;
  uint32_t probe_done;
  uint32_t agg_done;
  uint32_t plan_ready;
  uint32_t plan;
  uint32_t flags;
  int64_t kmin;
  int64_t span;
  int64_t state_off;
  int64_t out_base;
  uint32_t sh;
  uint32_t pad;
};
static_assert(sizeof(QRt) == 72, "QRt layout");

constexpr uint32_t kFlUnsafe = 1;
constexpr uint32_t kPlanEmpty = NFC_BATCH_PLAN_EMPTY;
constexpr uint32_t kPlanSmem = NFC_BATCH_PLAN_SMEM;
constexpr uint32_t kPlanGlobal = NFC_BATCH_PLAN_GLOBAL;
constexpr uint32_t kPlanDeferred = NFC_BATCH_PLAN_DEFERRED;
constexpr uint32_t kPlanSolo = NFC_BATCH_PLAN_SOLO;

// Fields written by other CTAs during the launch are read through L2 only
// (a line cached in this SM's L1 by an earlier item could be stale).
NFC_DEV int64_t ldcg_i64(const int64_t* p) { return (int64_t)__ldcg(reinterpret_cast<const long long*>(p)); }
NFC_DEV uint32_t ldcg_u32(const uint32_t* p) { return __ldcg(p); }
NFC_DEV unsigned long long ldcg_u64(const unsigned long long* p) { return __ldcg(p); }

struct BatchHdr {
  uint32_t ticket;
  int32_t err;
  unsigned long long arena_cursor;
  unsigned long long out_cursor;
  uint64_t pad;
  unsigned long long cycles[6];  // SM cycles per item type (thread 0 of each CTA); [4], [5]:
  unsigned long long items[6];   // aggregate items of shared-memory / global plans
};

struct BatchParams {
  const int32_t* keys;
  const uint8_t* kvalid;
  const int32_t* vals;
  const uint8_t* vvalid;
  int64_t n_total;
  const QDesc* qd;
  QRt* qr;
  const uint64_t* items;
  int64_t n_items;
  uint64_t* lb;
  unsigned long long* arena;
  int64_t arena_words;
  int64_t out_cap;
  int64_t* ukeys;
  int64_t* sums;
  int64_t* counts;
  int64_t* group_offsets;
  int64_t* ngroups;
  int32_t* qstatus;
  BatchHdr* hdr;
  int32_t smem_slots;
  int32_t smem_span_div;
  int32_t chunk_rows;
  int32_t probe_rows;
  int32_t warp_agg;
  int32_t pad;
};

bool operator==(const BatchParams& a, const BatchParams& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

struct BSmem {
  uint64_t item;
  int64_t a64[4];
  uint32_t u32[8];
  uint32_t scan[33];
  uint32_t red[kBWarps];
  uint32_t wv[kBWarps][32];
};

NFC_DEV uint32_t block_max_u32(uint32_t v, BSmem& S) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane_id() == 0) S.red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t r = 0;
#pragma unroll
  for (int w = 0; w < kBWarps; ++w) r = max(r, S.red[w]);
  return r;
}

NFC_DEV uint32_t block_sum_u32(uint32_t v, BSmem& S) {
  v = warp_sum(v);
  __syncthreads();
  if (lane_id() == 0) S.red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t r = 0;
#pragma unroll
  for (int w = 0; w < kBWarps; ++w) r += S.red[w];
  return r;
}

// Sub-tile of kBSub rows at 4-row aligned base g0 (rows g0 .. g0+8191 in
// groups of 4 per thread per step), masked to [a, b).  Bit e of `mask` says
// row e of the thread's 16 is in range and has valid key (and value).
template <bool VEC, bool VALS>
NFC_DEV void load_sub(const BatchParams& P, int64_t g0, int64_t a, int64_t b, int32_t (&k)[kBPer],
                      int32_t (&v)[kBPer], uint32_t& mask) {
  mask = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t r4 = g0 + ((int64_t)j * kBThreads + threadIdx.x) * 4;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      k[4 * j + e] = 0;
      v[4 * j + e] = 0;
    }
    if (r4 >= b) continue;
    if (VEC && r4 + 4 <= P.n_total) {
      const int4 kk = __ldcs(reinterpret_cast<const int4*>(P.keys + r4));
      k[4 * j] = kk.x; k[4 * j + 1] = kk.y; k[4 * j + 2] = kk.z; k[4 * j + 3] = kk.w;
      if (VALS) {
        const int4 vv = __ldcs(reinterpret_cast<const int4*>(P.vals + r4));
        v[4 * j] = vv.x; v[4 * j + 1] = vv.y; v[4 * j + 2] = vv.z; v[4 * j + 3] = vv.w;
      }
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (r4 + e < b) {
          k[4 * j + e] = P.keys[r4 + e];
          if (VALS) v[4 * j + e] = P.vals[r4 + e];
        }
      }
    }
    uint32_t m = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) m |= (r4 + e >= a && r4 + e < b) ? (1u << e) : 0u;
    if (P.kvalid) m &= (uint32_t)(P.kvalid[r4 >> 3] >> (r4 & 7)) & 0xFu;
    if (VALS && P.vvalid) m &= (uint32_t)(P.vvalid[r4 >> 3] >> (r4 & 7)) & 0xFu;
    mask |= m << (4 * j);
  }
}

NFC_DEV int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
NFC_DEV int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }
NFC_DEV uint32_t umax32(uint32_t a, uint32_t b) { return a > b ? a : b; }

NFC_DEV uint32_t ord32(int32_t k) { return (uint32_t)k ^ 0x80000000u; }

NFC_DEV uint32_t bitlen64(uint64_t x) { return x ? 64u - (uint32_t)__clzll((long long)x) : 0u; }

// Largest |value| for which rows * |value| < 2^(sh-1).
NFC_DEV uint64_t packed_limit(int64_t rows, uint32_t sh) {
  return ((1ull << (sh - 1)) - 1ull) / (uint64_t)imax64(rows, 1);
}

NFC_DEV uint32_t absu(int32_t v) { return v < 0 ? 0u - (uint32_t)v : (uint32_t)v; }

// Bounded wait (thread 0) until *p >= target; false on timeout, or at once
// once any wait of the launch has timed out (the launch then drains quickly).
// A legitimate wait covers at most a few items in flight (well under 1 ms);
// the bound is about a second.
constexpr uint32_t kBatchSpinLimit = 1u << 21;

NFC_DEV bool wait_ge(const uint32_t* p, uint32_t target, int32_t* err) {
  for (uint32_t i = 0; i < kBatchSpinLimit; ++i) {
    if (ld_volatile_u32(p) >= target) {
      __threadfence();
      return true;
    }
    if ((i & 255u) == 255u && ld_volatile_u32(reinterpret_cast<const uint32_t*>(err)) != 0u) return false;
    __nanosleep(256);
  }
  atomicExch(err, NFC_ERR_TIMEOUT);
  return false;
}

// Reserve `need` units of a bump allocator only if they fit under `cap`;
// returns the start or -1 (a failed request leaves the cursor unchanged, so
// the rest stays usable for later queries and the host-side fallback).
NFC_DEV int64_t reserve(unsigned long long* cursor, int64_t need, int64_t cap) {
  unsigned long long cur = ldcg_u64(cursor);
  for (int i = 0; i < 1 << 20; ++i) {
    if ((int64_t)cur + need > cap) return -1;
    const unsigned long long old = atomicCAS(cursor, cur, cur + (unsigned long long)need);
    if (old == cur) return (int64_t)cur;
    cur = old;
  }
  return -1;
}

// Called by thread 0 of the CTA that finished the query's last probe item.
NFC_DEV void plan_query(const BatchParams& P, const QDesc& qd, QRt* qr, int q) {
  const uint32_t nvalid = ld_volatile_u32(&qr->nvalid);
  uint32_t plan = kPlanEmpty;
  if (nvalid == 0) {
    P.ngroups[q] = 0;
    P.group_offsets[q] = 0;
  } else {
    const int32_t kmax = (int32_t)(ld_volatile_u32(&qr->kmax_o) ^ 0x80000000u);
    const int32_t kmin = (int32_t)((~ld_volatile_u32(&qr->kmin_c)) ^ 0x80000000u);
    const int64_t span = (int64_t)kmax - (int64_t)kmin + 1;
    const int64_t cap = (int64_t)qd.n_emit * qd.emit_slice;
    if (span <= P.smem_slots && span * P.smem_span_div <= (int64_t)qd.chunk) plan = kPlanSmem;
    else if (span <= cap) plan = kPlanGlobal;
    else plan = kPlanDeferred;
    if (plan != kPlanDeferred) {
      const int64_t words = (span + 3) & ~3ll;  // 32-byte aligned slices
      const int64_t need = imin64(nvalid, span);
      const int64_t off = reserve(&P.hdr->arena_cursor, words, P.arena_words);
      const int64_t ob = off < 0 ? -1 : reserve(&P.hdr->out_cursor, need, P.out_cap);
      // A state slice whose output reservation failed stays untouched (zero).
      if (ob < 0) plan = kPlanDeferred;
      qr->state_off = off < 0 ? 0 : off;
      qr->out_base = ob;
    }
    qr->kmin = kmin;
    qr->span = span;
    qr->sh = 64u - bitlen64((uint64_t)qd.rows);
  }
  if (plan == kPlanDeferred) P.qstatus[q] = 1;
  qr->plan = plan;
  __threadfence();
  atomicExch(&qr->plan_ready, 1u);
}

template <bool VEC>
NFC_DEV void do_probe(const BatchParams& P, BSmem& S, int q, uint32_t idx) {
  const QDesc qd = P.qd[q];
  QRt* qr = P.qr + q;
  const int64_t a = qd.row_off + (int64_t)idx * P.probe_rows;
  const int64_t b = imin64(a + P.probe_rows, qd.row_off + qd.rows);
  uint32_t mx = 0, mnc = 0, cnt = 0;
  int32_t k[kBPer], v[kBPer];
  for (int64_t g0 = a & ~3ll; g0 < b; g0 += kBSub) {
    uint32_t m;
    load_sub<VEC, false>(P, g0, a, b, k, v, m);
#pragma unroll
    for (int e = 0; e < kBPer; ++e) {
      if (m & (1u << e)) {
        const uint32_t o = ord32(k[e]);
        mx = max(mx, o);
        mnc = max(mnc, ~o);
        ++cnt;
      }
    }
  }
  mx = block_max_u32(mx, S);
  mnc = block_max_u32(mnc, S);
  cnt = block_sum_u32(cnt, S);
  if (threadIdx.x == 0) {
    if (cnt) {
      atomicMax(&qr->kmax_o, mx);
      atomicMax(&qr->kmin_c, mnc);
      atomicAdd(&qr->nvalid, cnt);
    }
    __threadfence();
    if (atomicAdd(&qr->probe_done, 1u) == qd.n_probe - 1) {
      __threadfence();
      plan_query(P, qd, qr, q);
    }
  }
}

// Global packed reductions for one loaded sub-tile.  Returns false if a
// value breaks the packed bound (the query is then flagged).
NFC_DEV bool global_apply(const BatchParams& P, BSmem& S, const int32_t (&k)[kBPer], const int32_t (&v)[kBPer],
                          uint32_t m, int64_t kmin, unsigned long long* st, uint32_t sh, uint64_t lim) {
  bool ok = true;
  const uint64_t one = 1ull << sh;
  const int warp = threadIdx.x >> 5, lane = lane_id();
#pragma unroll
  for (int e = 0; e < kBPer; ++e) {
    const bool in = (m >> e) & 1u;
    if (in && absu(v[e]) > lim) ok = false;
    if (P.warp_agg == 2) {
      // Hot-key combine: the rows of the warp that share the key of its first
      // valid lane are folded into one reduction (exact: 16-bit halves);
      // every other row reduces on its own.  Cheap enough to leave on for
      // high-cardinality queries, and it catches Zipf heads.
      const unsigned vm = __ballot_sync(0xffffffffu, in);
      if (vm == 0u) continue;
      const int leader = __ffs(vm) - 1;
      const uint32_t slot = in ? (uint32_t)((int64_t)k[e] - kmin) : 0xFFFFFFFFu;
      const uint32_t hot = __shfl_sync(0xffffffffu, slot, leader);
      const bool is_hot = in && slot == hot;
      const unsigned hm = __ballot_sync(0xffffffffu, is_hot);
      if (__popc(hm) > 1) {
        const uint32_t lo = __reduce_add_sync(0xffffffffu, is_hot ? ((uint32_t)v[e] & 0xFFFFu) : 0u);
        const int hi = __reduce_add_sync(0xffffffffu, is_hot ? (v[e] >> 16) : 0);
        if (lane == leader)
          atomicAdd(st + hot, (unsigned long long)__popc(hm) * one +
                                  (unsigned long long)((int64_t)hi * 65536 + (int64_t)lo));
        if (in && !is_hot) atomicAdd(st + slot, one + (unsigned long long)(int64_t)v[e]);
      } else if (in) {
        atomicAdd(st + slot, one + (unsigned long long)(int64_t)v[e]);
      }
    } else if (P.warp_agg) {
      // Spans are below 2^31, so 0xFFFFFFFF never names a real slot.
      const uint32_t slot = in ? (uint32_t)((int64_t)k[e] - kmin) : 0xFFFFFFFFu;
      const unsigned peers = __match_any_sync(0xffffffffu, slot);
      S.wv[warp][lane] = (uint32_t)v[e];
      __syncwarp();
      if (in && (__ffs(peers) - 1) == lane) {
        int64_t s = 0;
        for (unsigned pm = peers; pm; pm &= pm - 1) s += (int32_t)S.wv[warp][__ffs(pm) - 1];
        atomicAdd(st + slot, (unsigned long long)__popc(peers) * one + (unsigned long long)s);
      }
      __syncwarp();
    } else if (in) {
      atomicAdd(st + ((int64_t)k[e] - kmin), one + (unsigned long long)(int64_t)v[e]);
    }
  }
  return ok;
}

template <bool VEC>
NFC_DEV void global_chunk(const BatchParams& P, BSmem& S, const QDesc& qd, QRt* qr, int64_t a, int64_t b,
                          int64_t kmin, unsigned long long* st, uint32_t sh) {
  const uint64_t lim = packed_limit(qd.rows, sh);
  int32_t k[kBPer], v[kBPer];
  bool ok = true;
  for (int64_t g0 = a & ~3ll; g0 < b; g0 += kBSub) {
    uint32_t m;
    load_sub<VEC, true>(P, g0, a, b, k, v, m);
    ok &= global_apply(P, S, k, v, m, kmin, st, sh, lim);
  }
  if (!ok) atomicOr(&qr->flags, kFlUnsafe);
}

// Global plan with a shared-memory hash cache (warp_agg == 3): rows fold into
// a per-CTA table of T key slots (slot + 1 as the key, 0 = empty; count and
// int32 partial sum), flushed to the global state at the end of the chunk
// with one reduction per cached key.  A row whose key is not cached within
// kCacheProbe probes, or arrives once the table is 3/4 full, or whose value
// could overflow the int32 partial sum, reduces straight into the global
// state.  Zipf-like queries then cost shared atomics instead of one global
// reduction per row.
constexpr int kCacheProbe = 8;

template <bool VEC>
NFC_DEV void cached_chunk(const BatchParams& P, BSmem& S, uint32_t* skey, uint32_t* s_cnt, int32_t* s_sum, int lgT,
                          const QDesc& qd, QRt* qr, int64_t a, int64_t b, int64_t kmin, unsigned long long* st,
                          uint32_t sh) {
  const int T = 1 << lgT;
  for (int i = threadIdx.x; i < T; i += kBThreads) {
    skey[i] = 0u;
    s_cnt[i] = 0u;
    s_sum[i] = 0;
  }
  if (threadIdx.x == 0) S.u32[4] = 0u;  // slots taken
  __syncthreads();
  const uint64_t lim = packed_limit(qd.rows, sh);
  const uint32_t lim_s = (uint32_t)(0x7FFFFFFFu / (uint32_t)imax64(b - a, 1));
  const uint64_t one = 1ull << sh;
  const uint32_t fill_cap = (uint32_t)(T - T / 4);
  int32_t k[kBPer], v[kBPer];
  bool ok = true;
  for (int64_t g0 = a & ~3ll; g0 < b; g0 += kBSub) {
    uint32_t m;
    load_sub<VEC, true>(P, g0, a, b, k, v, m);
    const bool can_insert = *reinterpret_cast<volatile uint32_t*>(&S.u32[4]) < fill_cap;
#pragma unroll
    for (int e = 0; e < kBPer; ++e) {
      if (!(m & (1u << e))) continue;
      const uint32_t av = absu(v[e]);
      ok &= av <= lim;
      const uint32_t slot = (uint32_t)((int64_t)k[e] - kmin);
      int g = -1;
      if (av <= lim_s) {
        const uint32_t want = slot + 1u;
        const uint32_t h = lgT ? (slot * 0x9E3779B1u) >> (32 - lgT) : 0u;
        for (int i = 0; i < kCacheProbe; ++i) {
          const uint32_t pos = (h + i) & (uint32_t)(T - 1);
          uint32_t cur = skey[pos];
          if (cur == 0u && can_insert) {
            cur = atomicCAS(&skey[pos], 0u, want);
            if (cur == 0u) atomicAdd(&S.u32[4], 1u);
          }
          if (cur == 0u || cur == want) {
            if (cur == want || can_insert) g = (int)pos;
            break;
          }
        }
      }
      if (g >= 0) {
        atomicAdd(&s_cnt[g], 1u);
        atomicAdd(&s_sum[g], v[e]);
      } else {
        atomicAdd(st + slot, one + (unsigned long long)(int64_t)v[e]);
      }
    }
  }
  if (!ok) atomicOr(&qr->flags, kFlUnsafe);
  __syncthreads();
  for (int i = threadIdx.x; i < T; i += kBThreads) {
    const uint32_t w = skey[i];
    const uint32_t c = s_cnt[i];
    if (w && c) atomicAdd(st + (w - 1u), (unsigned long long)c * one + (unsigned long long)(int64_t)s_sum[i]);
  }
}

// Shared-memory table: s_cnt[span], s_sum[span] (int32 partial sums, safe
// while rows * |value| < 2^31 for the chunk).
template <bool VEC>
NFC_DEV uint32_t do_agg(const BatchParams& P, BSmem& S, uint32_t* s_cnt, int32_t* s_sum, int q, uint32_t idx) {
  const QDesc qd = P.qd[q];
  QRt* qr = P.qr + q;
  if (threadIdx.x == 0) {
    wait_ge(&qr->plan_ready, 1u, &P.hdr->err);
    S.u32[0] = ldcg_u32(&qr->plan);
    S.a64[0] = ldcg_i64(&qr->kmin);
    S.a64[1] = ldcg_i64(&qr->span);
    S.a64[2] = ldcg_i64(&qr->state_off);
    S.u32[1] = ldcg_u32(&qr->sh);
  }
  __syncthreads();
  const uint32_t plan = S.u32[0];
  const int64_t kmin = S.a64[0], span = S.a64[1];
  unsigned long long* st = P.arena + S.a64[2];
  const uint32_t sh = S.u32[1];
  const int64_t a = qd.row_off + (int64_t)idx * qd.chunk;
  const int64_t b = imin64(a + qd.chunk, qd.row_off + qd.rows);
  if (plan == kPlanGlobal && P.warp_agg == 3) {
    // The cache reuses the dynamic shared memory (smem_slots x 8 bytes) as
    // count[T] | sum[T] | key[T] with T the largest power of two that fits.
    int lgT = 0;
    while ((2 << lgT) * 12 <= P.smem_slots * 8) ++lgT;
    const int T = 1 << lgT;
    uint32_t* base = s_cnt;
    cached_chunk<VEC>(P, S, base + 2 * T, base, reinterpret_cast<int32_t*>(base + T), lgT, qd, qr, a, b, kmin, st,
                      sh);
  } else if (plan == kPlanGlobal) {
    global_chunk<VEC>(P, S, qd, qr, a, b, kmin, st, sh);
  } else if (plan == kPlanSmem) {
    for (int64_t i = threadIdx.x; i < span; i += kBThreads) {
      s_cnt[i] = 0;
      s_sum[i] = 0;
    }
    __syncthreads();
    const uint32_t lim_s = (uint32_t)(0x7FFFFFFFu / (uint32_t)imax64(b - a, 1));
    const uint64_t lim_q = packed_limit(qd.rows, sh);
    bool small = true, ok = true;
    int32_t k[kBPer], v[kBPer];
    for (int64_t g0 = a & ~3ll; g0 < b; g0 += kBSub) {
      uint32_t m;
      load_sub<VEC, true>(P, g0, a, b, k, v, m);
#pragma unroll
      for (int e = 0; e < kBPer; ++e) {
        if (m & (1u << e)) {
          const uint32_t av = absu(v[e]);
          small &= av <= lim_s;
          ok &= av <= lim_q;
          const int64_t slot = (int64_t)k[e] - kmin;
          atomicAdd(&s_cnt[slot], 1u);
          atomicAdd(&s_sum[slot], v[e]);
        }
      }
    }
    if (!ok) atomicOr(&qr->flags, kFlUnsafe);
    if (__syncthreads_and(small)) {
      const uint64_t one = 1ull << sh;
      for (int64_t i = threadIdx.x; i < span; i += kBThreads) {
        const uint32_t c = s_cnt[i];
        if (c) atomicAdd(st + i, (unsigned long long)c * one + (unsigned long long)(int64_t)s_sum[i]);
      }
    } else {
      // Some |value| could overflow the int32 partial sums: redo the chunk
      // with 64-bit global reductions.
      global_chunk<VEC>(P, S, qd, qr, a, b, kmin, st, sh);
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(&qr->agg_done, 1u);
  return plan;
}

// Decode a packed slot.
NFC_DEV void unpack(uint64_t w, uint32_t sh, int64_t& cnt, int64_t& sum) {
  const uint64_t lo = w & ((1ull << sh) - 1ull);
  const int64_t s = (int64_t)(lo << (64 - sh)) >> (64 - sh);
  sum = s;
  cnt = (int64_t)((w - (uint64_t)s) >> sh);
}

NFC_DEV void do_emit(const BatchParams& P, BSmem& S, int q, uint32_t j) {
  const QDesc qd = P.qd[q];
  QRt* qr = P.qr + q;
  if (threadIdx.x == 0) {
    bool ok = wait_ge(&qr->plan_ready, 1u, &P.hdr->err);
    if (ok) ok = wait_ge(&qr->agg_done, qd.n_agg, &P.hdr->err);
    S.u32[0] = ok ? ldcg_u32(&qr->plan) : kPlanDeferred;
    S.u32[1] = ldcg_u32(&qr->sh);
    S.u32[2] = ldcg_u32(&qr->flags);
    S.a64[0] = ldcg_i64(&qr->kmin);
    S.a64[1] = ldcg_i64(&qr->span);
    S.a64[2] = ldcg_i64(&qr->state_off);
    S.a64[3] = ldcg_i64(&qr->out_base);
  }
  __syncthreads();
  const uint32_t plan = S.u32[0];
  if (plan != kPlanSmem && plan != kPlanGlobal) return;
  const uint32_t sh = S.u32[1];
  const bool unsafe = S.u32[2] & kFlUnsafe;
  const int64_t kmin = S.a64[0], span = S.a64[1], out_base = S.a64[3];
  unsigned long long* st = P.arena + S.a64[2];
  const int64_t lo = (int64_t)j * qd.emit_slice;
  if (lo >= span) return;
  const int64_t hi = imin64(lo + qd.emit_slice, span);
  if (unsafe) {
    for (int64_t i = lo + threadIdx.x; i < hi; i += kBThreads) st[i] = 0ull;
    if (threadIdx.x == 0 && hi == span) P.qstatus[q] = 1;
    return;
  }
  // Pass 1: groups in the slice.
  uint32_t c = 0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kBThreads) c += ldcg_u64(st + i) != 0ull;
  const uint32_t total = block_sum_u32(c, S);
  if (threadIdx.x < 32) {
    const int64_t lbx = lookback_exclusive(P.lb + qd.lb_base, j, total, &P.hdr->err);  // whole warp
    if (threadIdx.x == 0) {
      S.a64[0] = lbx;
      if (hi == span) {
        P.ngroups[q] = S.a64[0] + total;
        P.group_offsets[q] = out_base;
      }
    }
  }
  __syncthreads();
  int64_t pos = out_base + S.a64[0];
  // Pass 2: compact in ascending slot order and clear.
  for (int64_t r = lo; r < hi; r += kBEmitRound) {
    const int64_t i0 = r + (int64_t)threadIdx.x * 4;
    uint64_t w[4];
    uint32_t cnt = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      w[e] = i0 + e < hi ? ldcg_u64(st + i0 + e) : 0ull;
      cnt += w[e] != 0ull;
    }
    uint32_t rt;
    const uint32_t ex = block_excl_scan(cnt, S.scan, &rt);
    int64_t o = pos + ex;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (w[e]) {
        int64_t gc, gs;
        unpack(w[e], sh, gc, gs);
        P.ukeys[o] = kmin + i0 + e;
        P.sums[o] = gs;
        P.counts[o] = gc;
        ++o;
        st[i0 + e] = 0ull;
      }
    }
    pos += rt;
  }
}

// One CTA: packed reductions into an arena slice, then an ascending
// compaction of the slice by the same CTA (which also clears it).
template <bool VEC>
NFC_DEV void solo_global(const BatchParams& P, BSmem& S, const QDesc& qd, int q, int64_t a, int64_t b,
                         int64_t kmin, int64_t span, unsigned long long* st, int64_t out_base) {
  const uint32_t sh = 64u - bitlen64((uint64_t)qd.rows);
  const uint64_t lim = packed_limit(qd.rows, sh);
  int32_t k[kBPer], v[kBPer];
  bool ok = true;
  for (int64_t g0 = a & ~3ll; g0 < b; g0 += kBSub) {
    uint32_t m;
    load_sub<VEC, true>(P, g0, a, b, k, v, m);
    ok &= global_apply(P, S, k, v, m, kmin, st, sh, lim);
  }
  __threadfence();
  const bool all_ok = __syncthreads_and(ok);
  int64_t pos = out_base;
  for (int64_t r = 0; r < span; r += kBEmitRound) {
    const int64_t i0 = r + (int64_t)threadIdx.x * 4;
    uint64_t w[4];
    uint32_t cnt = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      w[e] = i0 + e < span ? ldcg_u64(st + i0 + e) : 0ull;
      cnt += w[e] != 0ull;
      if (w[e]) st[i0 + e] = 0ull;
    }
    uint32_t rt;
    const uint32_t ex = block_excl_scan(cnt, S.scan, &rt);
    int64_t o = pos + ex;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (w[e] && all_ok) {
        int64_t gc, gs;
        unpack(w[e], sh, gc, gs);
        P.ukeys[o] = kmin + i0 + e;
        P.sums[o] = gs;
        P.counts[o] = gc;
        ++o;
      }
    }
    pos += rt;
  }
  if (threadIdx.x == 0) {
    if (all_ok) {
      P.ngroups[q] = pos - out_base;
      P.group_offsets[q] = out_base;
    } else {
      P.qstatus[q] = 1;
      P.qr[q].plan = kPlanDeferred;
    }
  }
}

template <bool VEC>
NFC_DEV void do_solo(const BatchParams& P, BSmem& S, uint32_t* s_cnt, int32_t* s_sum, int q) {
  const QDesc qd = P.qd[q];
  const int64_t a = qd.row_off, b = qd.row_off + qd.rows;
  uint32_t mx = 0, mnc = 0, cnt = 0;
  int32_t k[kBPer], v[kBPer];
  for (int64_t g0 = a & ~3ll; g0 < b; g0 += kBSub) {
    uint32_t m;
    load_sub<VEC, false>(P, g0, a, b, k, v, m);
#pragma unroll
    for (int e = 0; e < kBPer; ++e) {
      if (m & (1u << e)) {
        const uint32_t o = ord32(k[e]);
        mx = max(mx, o);
        mnc = max(mnc, ~o);
        ++cnt;
      }
    }
  }
  mx = block_max_u32(mx, S);
  mnc = block_max_u32(mnc, S);
  cnt = block_sum_u32(cnt, S);
  QRt* qr = P.qr + q;
  if (cnt == 0) {
    if (threadIdx.x == 0) {
      P.ngroups[q] = 0;
      P.group_offsets[q] = 0;
      qr->plan = kPlanEmpty;
    }
    return;
  }
  const int64_t kmin = (int32_t)((~mnc) ^ 0x80000000u);
  const int64_t span = (int64_t)(int32_t)(mx ^ 0x80000000u) - kmin + 1;
  const bool in_smem = span <= P.smem_slots;
  if (threadIdx.x == 0) {
    int64_t ob = -1, off = 0;
    if (in_smem) {
      ob = reserve(&P.hdr->out_cursor, imin64(cnt, span), P.out_cap);
    } else if (span <= 4 * qd.rows + P.smem_slots) {
      // Too wide for the shared table: packed global state in the arena,
      // still finished by this CTA alone.
      off = reserve(&P.hdr->arena_cursor, (span + 3) & ~3ll, P.arena_words);
      if (off >= 0) ob = reserve(&P.hdr->out_cursor, imin64(cnt, span), P.out_cap);
    }
    S.a64[0] = ob;
    S.a64[1] = off;
    qr->plan = ob < 0 ? kPlanDeferred : kPlanSolo;
    if (ob < 0) P.qstatus[q] = 1;
  }
  __syncthreads();
  const int64_t out_base = S.a64[0];
  if (out_base < 0) return;
  if (!in_smem) {
    solo_global<VEC>(P, S, qd, q, a, b, kmin, span, P.arena + S.a64[1], out_base);
    return;
  }
  for (int64_t i = threadIdx.x; i < span; i += kBThreads) {
    s_cnt[i] = 0;
    s_sum[i] = 0;
  }
  __syncthreads();
  const uint32_t lim_s = (uint32_t)(0x7FFFFFFFu / umax32(cnt, 1u));
  bool small = true;
  for (int64_t g0 = a & ~3ll; g0 < b; g0 += kBSub) {
    uint32_t m;
    load_sub<VEC, true>(P, g0, a, b, k, v, m);
#pragma unroll
    for (int e = 0; e < kBPer; ++e) {
      if (m & (1u << e)) {
        small &= absu(v[e]) <= lim_s;
        const int64_t slot = (int64_t)k[e] - kmin;
        atomicAdd(&s_cnt[slot], 1u);
        atomicAdd(&s_sum[slot], v[e]);
      }
    }
  }
  if (!__syncthreads_and(small)) {
    // int32 partial sums could have wrapped: leave the query to the host.
    if (threadIdx.x == 0) {
      P.qstatus[q] = 1;
      qr->plan = kPlanDeferred;
    }
    return;
  }
  int64_t pos = out_base;
  for (int64_t r = 0; r < span; r += kBEmitRound) {
    const int64_t i0 = r + (int64_t)threadIdx.x * 4;
    uint32_t c4[4];
    uint32_t n = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      c4[e] = i0 + e < span ? s_cnt[i0 + e] : 0u;
      n += c4[e] != 0u;
    }
    uint32_t rt;
    const uint32_t ex = block_excl_scan(n, S.scan, &rt);
    int64_t o = pos + ex;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (c4[e]) {
        P.ukeys[o] = kmin + i0 + e;
        P.sums[o] = s_sum[i0 + e];
        P.counts[o] = c4[e];
        ++o;
      }
    }
    pos += rt;
  }
  if (threadIdx.x == 0) {
    P.ngroups[q] = pos - out_base;
    P.group_offsets[q] = out_base;
  }
}

template <bool VEC, int MINB>
__global__ void __launch_bounds__(kBThreads, MINB) k_batch(const BatchParams P) {
  extern __shared__ __align__(16) unsigned char bsm[];
  __shared__ BSmem S;
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(bsm);
  int32_t* s_sum = reinterpret_cast<int32_t*>(bsm) + P.smem_slots;
  uint32_t next = 0;
  if (threadIdx.x == 0) next = atomicAdd(&P.hdr->ticket, 1u);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      S.item = next < P.n_items ? P.items[next] : ~0ull;
      if (next < P.n_items) next = atomicAdd(&P.hdr->ticket, 1u);
    }
    __syncthreads();
    const uint64_t it = S.item;
    if (it == ~0ull) break;
    const uint32_t type = (uint32_t)(it >> 62);
    const int q = (int)((it >> 32) & 0x3FFFFFFFull);
    const uint32_t idx = (uint32_t)it;
    const long long t0 = clock64();
    uint32_t plan = 0;
    switch (type) {
      case kItProbe: do_probe<VEC>(P, S, q, idx); break;
      case kItSolo: do_solo<VEC>(P, S, s_cnt, s_sum, q); break;
      case kItAgg: plan = do_agg<VEC>(P, S, s_cnt, s_sum, q, idx); break;
      default: do_emit(P, S, q, idx); break;
    }
    if (threadIdx.x == 0) {
      const unsigned long long dt = (unsigned long long)(clock64() - t0);
      atomicAdd(&P.hdr->cycles[type], dt);
      atomicAdd(&P.hdr->items[type], 1ull);
      if (plan == kPlanSmem || plan == kPlanGlobal) {
        const int k = plan == kPlanSmem ? 4 : 5;
        atomicAdd(&P.hdr->cycles[k], dt);
        atomicAdd(&P.hdr->items[k], 1ull);
      }
    }
  }
}

// Bits [off, off+n) of a bitmap, re-based to bit 0.
__global__ void k_bitmap_slice(const uint8_t* __restrict__ src, int64_t off, int64_t n, uint8_t* __restrict__ dst) {
  const int64_t nb = (n + 7) >> 3;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t byte = 0;
    for (int bit = 0; bit < 8; ++bit) {
      const int64_t r = i * 8 + bit;
      if (r < n) byte |= (uint32_t)((src[(off + r) >> 3] >> ((off + r) & 7)) & 1u) << bit;
    }
    dst[i] = (uint8_t)byte;
  }
}

template <bool VEC, int MINB>
cudaError_t launch_batch(const BatchParams& P, int grid, size_t smem, cudaStream_t s) {
  k_batch<VEC, MINB><<<grid, kBThreads, smem, s>>>(P);
  return cudaGetLastError();
}

// Dynamic shared memory limits are raised once per batch object, outside any
// stream capture.
cudaError_t set_batch_attributes(size_t smem) {
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return e;
}

size_t static_smem_bytes() { return sizeof(BSmem) + 64; }

}  // namespace
}  // namespace nfc

using namespace nfc;

struct nfc_batch {
  int device = 0;
  int64_t nq = 0;
  int64_t n_total = 0;
  nfc_batch_tuning tune{};
  std::vector<int64_t> row_off;
  std::vector<QDesc> hqd;
  int64_t n_items = 0;
  int64_t n_emit_total = 0;
  int64_t counts_by_type[4] = {};
  QDesc* d_qd = nullptr;
  uint64_t* d_items = nullptr;
  void* d_rt = nullptr;  // QRt[nq] | lb[n_emit_total] | hdr | qstatus[nq]
  size_t rt_bytes = 0;
  QRt* d_qr = nullptr;
  uint64_t* d_lb = nullptr;
  BatchHdr* d_hdr = nullptr;
  int32_t* d_qstatus = nullptr;
  unsigned long long* d_arena = nullptr;
  int64_t arena_words = 0;
  bool arena_dirty = true;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  BatchParams graph_params{};
  BatchParams last_params{};
  bool pending = false;
  std::mutex mu;
};

namespace {

void batch_free(nfc_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  cudaFree(b->d_qd);
  cudaFree(b->d_items);
  cudaFree(b->d_rt);
  cudaFree(b->d_arena);
  delete b;
}

void default_tuning(nfc_batch_tuning* t) {
  t->solo_rows = 32768;
  t->chunk_rows = 65536;
  t->probe_rows = 262144;
  t->emit_slice = 65536;
  t->emit_max_items = 8;
  t->smem_slots = 16384;
  t->smem_span_div = 2;
  t->warp_agg = 1;
  t->ctas_per_sm = 1;
  t->schedule = 0;
  t->agg_split = 0;
  t->arena_bytes = 0;
}

int check_tuning(const nfc_batch_tuning& t) {
  auto pow2ok = [](int32_t x, int32_t lo, int32_t hi) { return x >= lo && x <= hi && x % kBSub == 0; };
  if (t.solo_rows < 0 || t.solo_rows > (1 << 20)) return 0;
  if (!pow2ok(t.chunk_rows, kBSub, 1 << 24) || !pow2ok(t.probe_rows, kBSub, 1 << 26)) return 0;
  if (t.emit_slice < kBEmitRound || t.emit_slice % kBEmitRound) return 0;
  if (t.emit_max_items < 1 || t.emit_max_items > 4096) return 0;
  if (t.ctas_per_sm != 1 && t.ctas_per_sm != 2) return 0;
  if (t.smem_slots < 1024 || t.smem_slots % 1024) return 0;
  const size_t per_cta = (size_t)(227 * 1024) / (size_t)t.ctas_per_sm - static_smem_bytes() - 1024;
  if ((size_t)t.smem_slots * 8 > per_cta) return 0;
  if (t.smem_span_div < 1 || t.smem_span_div > 1024) return 0;
  if (t.warp_agg < 0 || t.warp_agg > 3) return 0;
  if (t.schedule < 0 || t.schedule > 2) return 0;
  if (t.agg_split < 0 || t.agg_split > 4096) return 0;
  if (t.arena_bytes < 0) return 0;
  return 1;
}

uint64_t item(uint32_t type, int64_t q, uint32_t idx) {
  return ((uint64_t)type << 62) | ((uint64_t)q << 32) | idx;
}

}  // namespace

extern "C" void nfc_batch_default_tuning(nfc_batch_tuning* t) {
  if (t) default_tuning(t);
}

extern "C" nfc_batch* nfc_batch_create(int64_t nq, const int64_t* row_offsets, const nfc_batch_tuning* tuning) {
  if (nq < 1 || nq >= (1 << 24) || !row_offsets) {
    set_last_error("nfc_batch_create: nq=%lld out of [1, 2^24) or null row_offsets", (long long)nq);
    return nullptr;
  }
  nfc_batch_tuning t;
  default_tuning(&t);
  if (tuning) t = *tuning;
  if (!check_tuning(t)) {
    set_last_error("nfc_batch_create: invalid tuning (chunk/probe rows multiples of %d, emit_slice multiple of %d, "
                   "smem_slots multiple of 1024 within the per-CTA shared memory, ctas_per_sm 1 or 2)",
                   kBSub, kBEmitRound);
    return nullptr;
  }
  if (row_offsets[0] != 0) {
    set_last_error("nfc_batch_create: row_offsets[0] must be 0");
    return nullptr;
  }
  for (int64_t q = 0; q < nq; ++q) {
    const int64_t r = row_offsets[q + 1] - row_offsets[q];
    if (r < 0 || r >= (1ll << 31)) {
      set_last_error("nfc_batch_create: query %lld has %lld rows (need 0 <= rows < 2^31)", (long long)q, (long long)r);
      return nullptr;
    }
  }
  nfc_batch* b = new (std::nothrow) nfc_batch();
  if (!b) return nullptr;
  b->nq = nq;
  b->tune = t;
  b->row_off.assign(row_offsets, row_offsets + nq + 1);
  b->n_total = row_offsets[nq];
  cudaGetDevice(&b->device);
  b->hqd.resize(nq);
  std::vector<int64_t> order(nq);
  for (int64_t q = 0; q < nq; ++q) order[q] = q;
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
    return (row_offsets[x + 1] - row_offsets[x]) > (row_offsets[y + 1] - row_offsets[y]);
  });
  uint32_t lb = 0;
  for (int64_t q = 0; q < nq; ++q) {
    QDesc& d = b->hqd[q];
    std::memset(&d, 0, sizeof(d));
    d.row_off = row_offsets[q];
    d.rows = row_offsets[q + 1] - row_offsets[q];
    d.solo = d.rows <= t.solo_rows ? 1u : 0u;
    if (!d.solo) {
      d.n_probe = (uint32_t)((d.rows + t.probe_rows - 1) / t.probe_rows);
      // Large queries are cut into at least agg_split items, so the CTAs
      // working at one time share few queries and their state stays in L2.
      int64_t chunk = t.chunk_rows;
      if (t.agg_split > 0) {
        const int64_t want = (d.rows + t.agg_split - 1) / t.agg_split;
        chunk = std::min<int64_t>(chunk, std::max<int64_t>(kBSub, (want + kBSub - 1) / kBSub * kBSub));
      }
      d.chunk = (uint32_t)chunk;
      d.n_agg = (uint32_t)((d.rows + chunk - 1) / chunk);
      const int64_t cap = std::max<int64_t>(d.rows, t.smem_slots);
      int64_t ne = std::min<int64_t>((cap + t.emit_slice - 1) / t.emit_slice, t.emit_max_items);
      int64_t slice = (cap + ne - 1) / ne;
      slice = (slice + kBEmitRound - 1) / kBEmitRound * kBEmitRound;
      d.n_emit = (uint32_t)ne;
      d.emit_slice = (uint32_t)slice;
      d.lb_base = lb;
      lb += (uint32_t)ne;
    }
  }
  b->n_emit_total = lb;
  // Item list.
  std::vector<uint64_t> items;
  auto add_probe = [&]() {
    for (int64_t q : order) {
      const QDesc& d = b->hqd[q];
      if (d.solo) continue;
      for (uint32_t i = 0; i < d.n_probe; ++i) items.push_back(item(kItProbe, q, i));
    }
  };
  auto add_solo = [&]() {
    for (int64_t q : order)
      if (b->hqd[q].solo) items.push_back(item(kItSolo, q, 0));
  };
  auto add_agg_q = [&](int64_t q) {
    for (uint32_t i = 0; i < b->hqd[q].n_agg; ++i) items.push_back(item(kItAgg, q, i));
  };
  auto add_emit_q = [&](int64_t q) {
    for (uint32_t i = 0; i < b->hqd[q].n_emit; ++i) items.push_back(item(kItEmit, q, i));
  };
  std::vector<int64_t> multi;
  for (int64_t q : order)
    if (!b->hqd[q].solo) multi.push_back(q);
  add_probe();
  if (t.schedule != 2) add_solo();
  if (t.schedule == 1) {
    // Emit items of a query follow the aggregate items of the query two
    // places later, so its state is read back while still in L2.
    const size_t lag = 2;
    for (size_t i = 0; i < multi.size(); ++i) {
      add_agg_q(multi[i]);
      if (i >= lag) add_emit_q(multi[i - lag]);
    }
    for (size_t i = multi.size() > lag ? multi.size() - lag : 0; i < multi.size(); ++i) add_emit_q(multi[i]);
  } else {
    for (int64_t q : multi) add_agg_q(q);
    for (int64_t q : multi) add_emit_q(q);
  }
  if (t.schedule == 2) add_solo();
  b->n_items = (int64_t)items.size();
  for (uint64_t it : items) b->counts_by_type[it >> 62]++;
  // Arena default: 2 bytes per row (at least 256 MiB), never more than every
  // non-solo query's largest accepted span nor a quarter of free memory.  A
  // query whose span does not fit in what is left is deferred.
  int64_t want = 0;
  for (const QDesc& d : b->hqd)
    if (!d.solo) want += ((int64_t)d.n_emit * d.emit_slice + 3) & ~3ll;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  int64_t words = t.arena_bytes ? t.arena_bytes / 8
                                 : std::min<int64_t>({want, std::max<int64_t>(b->n_total / 4, (256ll << 20) / 8),
                                                      (int64_t)(free_b / 4 / 8)});
  words = std::max<int64_t>(words, 4);
  b->arena_words = words;
  b->rt_bytes = sizeof(QRt) * nq + sizeof(uint64_t) * (b->n_emit_total + 1) + sizeof(BatchHdr) + sizeof(int32_t) * nq;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&b->d_qd, sizeof(QDesc) * nq);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_items, sizeof(uint64_t) * std::max<int64_t>(b->n_items, 1));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_rt, b->rt_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_arena, sizeof(unsigned long long) * words);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_qd, b->hqd.data(), sizeof(QDesc) * nq, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && b->n_items)
    e = cudaMemcpy(b->d_items, items.data(), sizeof(uint64_t) * b->n_items, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = set_batch_attributes((size_t)t.smem_slots * 8);
  if (e == cudaSuccess) num_sms();
  if (e != cudaSuccess) {
    cuda_fail(e, "nfc_batch_create");
    batch_free(b);
    return nullptr;
  }
  char* p = static_cast<char*>(b->d_rt);
  b->d_qr = reinterpret_cast<QRt*>(p);
  p += sizeof(QRt) * nq;
  b->d_lb = reinterpret_cast<uint64_t*>(p);
  p += sizeof(uint64_t) * (b->n_emit_total + 1);
  b->d_hdr = reinterpret_cast<BatchHdr*>(p);
  p += sizeof(BatchHdr);
  b->d_qstatus = reinterpret_cast<int32_t*>(p);
  return b;
}

extern "C" void nfc_batch_destroy(nfc_batch* b) {
  if (!b) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  batch_free(b);
  cudaSetDevice(cur);
}

extern "C" int32_t nfc_batch_info(const nfc_batch* b, int64_t* out, int32_t nout) {
  if (!b || !out) return NFC_ERR_NULL;
  const int64_t v[8] = {b->nq, b->n_total, b->n_items, b->counts_by_type[kItProbe], b->counts_by_type[kItSolo],
                        b->counts_by_type[kItAgg], b->counts_by_type[kItEmit], b->arena_words * 8};
  for (int i = 0; i < nout && i < 8; ++i) out[i] = v[i];
  return NFC_OK;
}

namespace {

// Enqueue zeroing of the runtime state and the persistent kernel.
int enqueue_batch(nfc_batch* b, const BatchParams& P, bool vec, cudaStream_t s) {
  NFC_CUDA(cudaMemsetAsync(b->d_rt, 0, b->rt_bytes, s));
  if (P.n_items == 0) return NFC_OK;
  const int cps = b->tune.ctas_per_sm;
  const int grid = (int)std::min<int64_t>((int64_t)num_sms() * cps, P.n_items);
  const size_t smem = (size_t)b->tune.smem_slots * 8;
  cudaError_t e;
  if (vec) e = cps == 2 ? launch_batch<true, 2>(P, grid, smem, s) : launch_batch<true, 1>(P, grid, smem, s);
  else e = cps == 2 ? launch_batch<false, 2>(P, grid, smem, s) : launch_batch<false, 1>(P, grid, smem, s);
  NFC_CUDA(e);
  return NFC_OK;
}

// The single-query path for one deferred query; results land at *cursor.
int run_deferred(nfc_batch* b, const BatchParams& P, int64_t q, int64_t* cursor, cudaStream_t s) {
  const int64_t a = b->row_off[q], n = b->row_off[q + 1] - b->row_off[q];
  Scratch sc(s);
  uint8_t* kv = nullptr;
  uint8_t* vv = nullptr;
  const int64_t nb = (n + 7) / 8;
  if (P.kvalid) {
    NFC_CUDA(sc.alloc(&kv, nb));
    k_bitmap_slice<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((nb + 255) / 256, 4096)), 256, 0, s>>>(
        P.kvalid, a, n, kv);
    NFC_CUDA(cudaGetLastError());
  }
  if (P.vvalid) {
    NFC_CUDA(sc.alloc(&vv, nb));
    k_bitmap_slice<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((nb + 255) / 256, 4096)), 256, 0, s>>>(
        P.vvalid, a, n, vv);
    NFC_CUDA(cudaGetLastError());
  }
  int64_t* tmp = nullptr;
  const int64_t cap = std::max<int64_t>(n, 1);
  NFC_CUDA(sc.alloc(&tmp, 3 * cap));
  nfc_value_col col{};
  col.dtype = NFC_I32;
  col.aggs = NFC_AGG_SUM;
  col.data = P.vals + a;
  col.validity = vv;
  col.sum_out = tmp + cap;
  nfc_groupby_args ga{};
  ga.n = n;
  ga.keys = P.keys + a;
  ga.key_validity = kv;
  ga.ncols = 1;
  ga.cols = &col;
  ga.out_cap = cap;
  ga.ukeys_out = tmp;
  ga.counts_out = tmp + 2 * cap;
  const int64_t ng = nfc_groupby(&ga, NFC_STRAT_AUTO, s, nullptr);
  if (ng < 0) return (int)ng;
  if (*cursor + ng > P.out_cap) {
    set_last_error("nfc_batch_run: output capacity %lld too small for deferred query %lld", (long long)P.out_cap,
                   (long long)q);
    return NFC_ERR_OVERFLOW;
  }
  if (ng) {
    NFC_CUDA(cudaMemcpyAsync(P.ukeys + *cursor, tmp, ng * 8, cudaMemcpyDeviceToDevice, s));
    NFC_CUDA(cudaMemcpyAsync(P.sums + *cursor, tmp + cap, ng * 8, cudaMemcpyDeviceToDevice, s));
    NFC_CUDA(cudaMemcpyAsync(P.counts + *cursor, tmp + 2 * cap, ng * 8, cudaMemcpyDeviceToDevice, s));
  }
  const int64_t go[2] = {*cursor, ng};
  NFC_CUDA(cudaMemcpyAsync(P.group_offsets + q, &go[0], 8, cudaMemcpyHostToDevice, s));
  NFC_CUDA(cudaMemcpyAsync(P.ngroups + q, &go[1], 8, cudaMemcpyHostToDevice, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  *cursor += ng;
  return NFC_OK;
}

// Read back the launch's status (error word, output cursor, deferred
// queries) and finish every deferred query with the single-query path.
int64_t batch_finish_locked(nfc_batch* b, cudaStream_t s) {
  const BatchParams& P = b->last_params;
  b->pending = false;
  BatchHdr hdr{};
  std::vector<int32_t> st((size_t)b->nq);
  NFC_CUDA(cudaMemcpyAsync(&hdr, b->d_hdr, sizeof(hdr), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaMemcpyAsync(st.data(), b->d_qstatus, sizeof(int32_t) * b->nq, cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if (hdr.err) {
    b->arena_dirty = true;
    set_last_error("nfc_batch_run: a bounded wait timed out in the batch kernel");
    return hdr.err;
  }
  int64_t cursor = std::min<int64_t>((int64_t)hdr.out_cursor, P.out_cap);
  int64_t ndef = 0;
  for (int64_t q = 0; q < b->nq; ++q) {
    if (!st[q]) continue;
    const int rc = run_deferred(b, P, q, &cursor, s);
    if (rc != NFC_OK) return rc;
    ++ndef;
  }
  return ndef;
}

}  // namespace

extern "C" int64_t nfc_batch_run(nfc_batch* b, const int32_t* keys, const uint8_t* key_validity, const int32_t* values,
                                 const uint8_t* value_validity, int64_t out_cap, int64_t* ukeys_out,
                                 int64_t* sums_out, int64_t* counts_out, int64_t* group_offsets,
                                 int64_t* ngroups, int32_t flags, void* stream) {
  if (!b) return NFC_ERR_NULL;
  if (b->n_total > 0 && (!keys || !values)) return NFC_ERR_NULL;
  if (!group_offsets || !ngroups || (out_cap > 0 && (!ukeys_out || !sums_out || !counts_out))) return NFC_ERR_NULL;
  if (out_cap < 0) return NFC_ERR_MALFORMED;
  std::lock_guard<std::mutex> lock(b->mu);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BatchParams P{};
  P.keys = keys;
  P.kvalid = key_validity;
  P.vals = values;
  P.vvalid = value_validity;
  P.n_total = b->n_total;
  P.qd = b->d_qd;
  P.qr = b->d_qr;
  P.items = b->d_items;
  P.n_items = b->n_items;
  P.lb = b->d_lb;
  P.arena = b->d_arena;
  P.arena_words = b->arena_words;
  P.out_cap = out_cap;
  P.ukeys = ukeys_out;
  P.sums = sums_out;
  P.counts = counts_out;
  P.group_offsets = group_offsets;
  P.ngroups = ngroups;
  P.qstatus = b->d_qstatus;
  P.hdr = b->d_hdr;
  P.smem_slots = b->tune.smem_slots;
  P.smem_span_div = b->tune.smem_span_div;
  P.chunk_rows = b->tune.chunk_rows;
  P.probe_rows = b->tune.probe_rows;
  P.warp_agg = b->tune.warp_agg;
  const bool vec = ((uintptr_t)keys % 16 == 0) && ((uintptr_t)values % 16 == 0);
  if (b->arena_dirty) {
    NFC_CUDA(cudaMemsetAsync(b->d_arena, 0, sizeof(unsigned long long) * b->arena_words, s));
    b->arena_dirty = false;
  }
  const bool use_graph = flags & NFC_BATCH_GRAPH;
  if (use_graph) {
    if (!b->exec || !(b->graph_params == P)) {
      if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
      }
      cudaGraph_t g = nullptr;
      NFC_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue_batch(b, P, vec, b->cap_stream);
      const cudaError_t ce = cudaStreamEndCapture(b->cap_stream, &g);
      if (rc != NFC_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      NFC_CUDA(ce);
      const cudaError_t ie = cudaGraphInstantiate(&b->exec, g, 0);
      cudaGraphDestroy(g);
      NFC_CUDA(ie);
      b->graph_params = P;
    }
    NFC_CUDA(cudaGraphLaunch(b->exec, s));
  } else {
    const int rc = enqueue_batch(b, P, vec, s);
    if (rc != NFC_OK) return rc;
  }
  b->last_params = P;
  b->pending = true;
  if (flags & NFC_BATCH_NO_SYNC) return 0;
  return batch_finish_locked(b, s);
}

extern "C" int64_t nfc_batch_finish(nfc_batch* b, void* stream) {
  if (!b) return NFC_ERR_NULL;
  std::lock_guard<std::mutex> lock(b->mu);
  if (!b->pending) return 0;
  return batch_finish_locked(b, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t nfc_batch_profile(nfc_batch* b, int64_t* out, void* stream) {
  if (!b || !out) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BatchHdr hdr{};
  NFC_CUDA(cudaMemcpyAsync(&hdr, b->d_hdr, sizeof(hdr), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < 6; ++i) {
    out[i] = (int64_t)hdr.cycles[i];
    out[6 + i] = (int64_t)hdr.items[i];
  }
  return NFC_OK;
}

extern "C" int32_t nfc_batch_query_plans(nfc_batch* b, int32_t* plans_out, void* stream) {
  if (!b || !plans_out) return NFC_ERR_NULL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<QRt> rt((size_t)b->nq);
  NFC_CUDA(cudaMemcpyAsync(rt.data(), b->d_qr, sizeof(QRt) * b->nq, cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  for (int64_t q = 0; q < b->nq; ++q) plans_out[q] = (int32_t)rt[q].plan;
  return NFC_OK;
}
