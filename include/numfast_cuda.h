/*
 * libnumfast_cuda — B200 (sm_100a) group-by hot path for NumFast.
 *
 * Two C-ABI surfaces live in one shared library:
 *
 *  1. nf_*  — the numfast-native ABI the reference's Python host binds
 *             through ctypes (src/Drivers/CPU/_lib/native_cpu.py:93-143 and
 *             the optional-ABI probes it runs later).  Same names, same
 *             argument meaning, same return codes; buffers are HOST memory,
 *             the library stages them to the GPU and back.  Each entry cites
 *             the numfast-native/src/lib.rs export it replaces.
 *
 *  2. nfc_* — the device-resident extension: device pointers, Arrow-style
 *             LSB validity bitmaps, min/max lanes, an explicit CUDA stream.
 *             No counterpart in numfast-native (validity is compacted in
 *             Python before the native call there, cpu.py:3508-3511); these
 *             entries replace the executor's groupby_multi / sort /
 *             unique_inverse branches (cpu.py:3435-3704, :3177-3187,
 *             :4006-4040) when the data already lives in HBM.
 *
 * Every call but one is reentrant: scratch memory is stream-ordered and
 * private to the call, so concurrent calls on distinct streams (or from
 * distinct host threads through nf_*) never share state.  The exception is
 * nfc_groupby_dense_noalloc, whose calls all share one static device array
 * (see its comment).
 */
#ifndef NUMFAST_CUDA_H
#define NUMFAST_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes (numfast-native/src/core/errors.rs:13-38) ---------- */
#define NFC_OK 0
#define NFC_ERR_NULL (-1)      /* null pointer; unsorted abort on *_sorted_run_* */
#define NFC_ERR_RANGE (-2)     /* out-of-range key; null state on carry/sorted */
#define NFC_ERR_MALFORMED (-3) /* bad geometry / unknown variant */
#define NFC_ERR_OVERFLOW (-4)  /* checked integer add failed (never wraps) */
#define NFC_ERR_UNSORTED (-5)  /* V_SORTED variant on regressing keys */
/* CUDA-library specific (no counterpart in the reference): */
#define NFC_ERR_CUDA (-6)        /* a CUDA runtime call failed; see nfc_last_error() */
#define NFC_ERR_TIMEOUT (-7)     /* a bounded cross-CTA wait gave up */
#define NFC_ERR_NOMEM (-8)       /* device scratch allocation failed */
#define NFC_ERR_UNSUPPORTED (-9) /* argument combination not supported */

/* ====================================================================== */
/* 1. numfast-native ABI (host pointers)                                  */
/* ====================================================================== */

/* lib.rs:85 nf_group_sum_count — f64 sums + int64 counts over dense codes. */
int32_t nf_group_sum_count(const int32_t* keys, const double* values, size_t n,
                           double* sums, int64_t* counts, size_t g);

/* lib.rs:117 nf_group_multi_sum_count — SoA multi-column f64 sums, shared
 * counts; -2 on a key outside [0, g). */
int32_t nf_group_multi_sum_count(const int32_t* keys, const double* values,
                                 size_t n, size_t ncols, double* sums,
                                 int64_t* counts, size_t g);

/* lib.rs:150 nf_group_mixed_sum_only — int32 (checked, -4) + f64 sums, no
 * counts lane. */
int32_t nf_group_mixed_sum_only(const int32_t* keys, const int32_t* i32_vals,
                                const double* f64_vals, size_t n, size_t n_i32,
                                size_t n_f64, int32_t* i32_sums,
                                double* f64_sums, size_t g);

/* lib.rs:184 nf_group_count_only — keys-only count pass. */
int32_t nf_group_count_only(const int32_t* keys, size_t n, int64_t* counts,
                            size_t g);

/* lib.rs:213 nf_group_owner_2i32_1f64 — owner-range shard: only lanes
 * [lo, hi) of the outputs are written. */
int32_t nf_group_owner_2i32_1f64(const int32_t* keys, const int32_t* a,
                                 const int32_t* b, const double* c, size_t n,
                                 size_t lo, size_t hi, int32_t* s1, int32_t* s2,
                                 double* s3, int64_t* counts, size_t g);

/* lib.rs:262 nf_pack_i32_direct — out[i] = k1[i]*m2 + k2[i]; -2 on negative
 * input or int32 overflow.  Off the hot path but required by the loader. */
int32_t nf_pack_i32_direct(const int32_t* k1, const int32_t* k2, int32_t m2,
                           size_t n, int32_t* out);

/* lib.rs:287 nf_pack_sum_count_i32 — fused pack + int32 sum + int64 count:
 * code of row i = k1[i]*m2 + k2[i] (never materialised), sums/counts over
 * [0, g) overwritten; -2 on a failed pack or a code outside [0, g), -4 when a
 * group's running int32 sum in row order overflows (never wraps). */
int32_t nf_pack_sum_count_i32(const int32_t* k1, const int32_t* k2, int32_t m2,
                              const int32_t* vals, size_t n, int32_t* sums,
                              int64_t* counts, size_t g);

/* lib.rs:316 nf_pack_sum_count_f64 — same with float64 values and sums. */
int32_t nf_pack_sum_count_f64(const int32_t* k1, const int32_t* k2, int32_t m2,
                              const double* vals, size_t n, double* sums,
                              int64_t* counts, size_t g);

/* lib.rs:347 nf_pattern_encode — prefix + integer string encode.  Off the hot
 * path but required by the loader (native_cpu.py:131-132). */
int32_t nf_pattern_encode(const uint8_t* data, size_t total, const int32_t* offs,
                          size_t n, const uint8_t* prefix, size_t prefix_len,
                          int32_t* codes, uint8_t* valid, int32_t* width_out,
                          int32_t* err_row_out);

/* lib.rs:399 / :425 nf_sorted_run_{i64,f64} — run aggregate over
 * nondecreasing keys; returns ng, -1 unsorted, -2 null. */
int64_t nf_sorted_run_i64(const int32_t* keys, const int64_t* vals, size_t n,
                          int64_t* ukeys, int64_t* sums, int64_t* counts);
int64_t nf_sorted_run_f64(const int32_t* keys, const double* vals, size_t n,
                          int64_t* ukeys, double* sums, int64_t* counts);

/* lib.rs:462 / :492 nf_carry_build_{i64,f64} — compact dense M-state to
 * (ukeys, counts, sums) in ascending code order; returns ng. */
int64_t nf_carry_build_i64(const int64_t* counts_m, const int64_t* sums_m,
                           size_t m, int64_t* ukeys, int64_t* counts,
                           int64_t* sums);
int64_t nf_carry_build_f64(const int64_t* counts_m, const double* sums_m,
                           size_t m, int64_t* ukeys, int64_t* counts,
                           double* sums);

/* lib.rs:539 / :569 / :596 nf_group_variant_{f64,i64,i32} — variant 0 dense,
 * 1 checked (f64/i64), 2 sorted-dense; -3 unknown variant. */
int32_t nf_group_variant_f64(const int32_t* keys, const double* values, size_t n,
                             uint32_t variant, double* sums, int64_t* counts,
                             size_t g);
int32_t nf_group_variant_i64(const int32_t* keys, const int64_t* ticks, size_t n,
                             uint32_t variant, int64_t* sums, int64_t* counts,
                             size_t g);
int32_t nf_group_variant_i32(const int32_t* keys, const int32_t* ticks, size_t n,
                             uint32_t variant, int32_t* sums, int64_t* counts,
                             size_t g);

/* lib.rs:1326 / :1363 nf_sort_perm_{i32,i64} — stable radix argsort;
 * descending != 0 reverses key groups and keeps input order inside each. */
int32_t nf_sort_perm_i32(const int32_t* keys, size_t n, uint8_t descending,
                         int32_t* perm_out, uint32_t* tmp0, uint32_t* tmp1,
                         int32_t* tmp_p);
int32_t nf_sort_perm_i64(const int64_t* keys, size_t n, uint8_t descending,
                         int32_t* perm_out, uint64_t* tmp0, uint64_t* tmp1,
                         int32_t* tmp_p);

/* lib.rs:1420 / :1464 nf_unique_inverse_{i32,i64} — sorted unique + inverse
 * codes (np.unique(return_inverse=True) labelling); returns ng. */
int64_t nf_unique_inverse_i32(const int32_t* keys, size_t n, int32_t* uniq_out,
                              int32_t* inv_out, int32_t* perm, uint32_t* tmp0,
                              uint32_t* tmp1, int32_t* tmp_p);
int64_t nf_unique_inverse_i64(const int64_t* keys, size_t n, int64_t* uniq_out,
                              int32_t* inv_out, int32_t* perm, uint64_t* tmp0,
                              uint64_t* tmp1, int32_t* tmp_p);

/* ====================================================================== */
/* 2. nfc_* device-resident extension                                     */
/* ====================================================================== */

enum { NFC_I32 = 0, NFC_I64 = 1, NFC_F64 = 2 };
enum { NFC_AGG_SUM = 1, NFC_AGG_MIN = 2, NFC_AGG_MAX = 4 };

/* Grouping strategies.  All produce identical integer results and float64
 * sums within 1e-12 relative; they differ only in speed. */
enum {
  NFC_STRAT_AUTO = 0,
  NFC_STRAT_SORTED = 1,       /* nondecreasing keys: run aggregation        */
  NFC_STRAT_DENSE_SMEM = 2,   /* per-CTA shared-memory dense state          */
  NFC_STRAT_DENSE_GLOBAL = 3, /* L2-resident dense state, global atomics    */
  NFC_STRAT_PARTITION = 4,    /* key-range partition + on-chip aggregation  */
  NFC_STRAT_HASH = 5,         /* global open addressing + key sort          */
  NFC_STRAT_SHARED_HASH = 6,  /* per-CTA shared-memory hash tables in front
                                 of a global table sized from the distinct
                                 hint; overflow retries at full size        */
  NFC_STRAT_SORT = 7          /* stable radix sort of the valid rows by key,
                                 then run aggregation (the reference's
                                 "hash" plan executes as a sorted unique)   */
};

#define NFC_MAX_COLS 4

typedef struct nfc_value_col {
  int32_t dtype;           /* NFC_I32 / NFC_I64 / NFC_F64                   */
  int32_t aggs;            /* NFC_AGG_* bitmask (count is always produced)  */
  const void* data;        /* device, n values                              */
  const uint8_t* validity; /* device LSB bitmap (bit i = row i) or NULL     */
  void* sum_out;           /* device: int64 for integer columns, double    */
  void* min_out;           /* device, value dtype                           */
  void* max_out;           /* device, value dtype                           */
} nfc_value_col;

typedef struct nfc_groupby_args {
  int64_t n;
  const int32_t* keys;         /* device, n int32 keys                      */
  const uint8_t* key_validity; /* device LSB bitmap or NULL                 */
  int32_t ncols;               /* 0..NFC_MAX_COLS                           */
  const nfc_value_col* cols;   /* HOST array of ncols descriptors           */
  int64_t out_cap;             /* capacity of every output array            */
  int64_t* ukeys_out;          /* device, ascending distinct keys           */
  int64_t* counts_out;         /* device, rows per group                    */
  const uint8_t* row_filter;   /* device LSB bitmap or NULL: an upstream
                                  filter fused into the group-by (rows whose
                                  bit is 0 take no part, as if compacted out
                                  first; chain.py:945 filter -> group)       */
} nfc_groupby_args;

typedef struct nfc_probe {
  int64_t n_valid; /* rows whose key and every value are non-NULL */
  int64_t kmin;    /* over valid rows (0 when n_valid == 0)       */
  int64_t kmax;
  int32_t sorted;  /* valid keys nondecreasing in row order        */
  int32_t pad;
} nfc_probe;

#define NFC_MAX_STAGES 8

typedef struct nfc_groupby_stats {
  int32_t strategy; /* strategy that ran                          */
  int32_t status;   /* device status word (0 ok)                  */
  int64_t ng;       /* groups written                             */
  nfc_probe probe;
  int64_t buckets;  /* partition count (PARTITION) / table slots (HASH) */
  int32_t timing;   /* IN: nonzero records CUDA events between stages */
  int32_t launches; /* OUT: kernels launched by the call              */
  int32_t nstages;  /* OUT: stages timed (0 unless timing)            */
  int32_t pad;
  float stage_ms[NFC_MAX_STAGES]; /* OUT: device time per stage, in launch order */
  int64_t distinct_hint; /* IN: expected distinct keys (0 = unknown); sizes the
                            SHARED_HASH global table                        */
  int32_t overflowed;    /* OUT (SHARED_HASH): 0 the hinted table sufficed; 1 it
                            overflowed and a full-size retry ran; 2 that
                            overflowed too and HASH ran                      */
  int32_t planner_used;  /* OUT (nfc_groupby_planned): NFC_PLANNER_FIXED or
                            NFC_PLANNER_LEARNED, whichever decided           */
  int64_t predicted_distinct; /* OUT (learned planner): network's estimate */
  int32_t learned_pick;  /* OUT (learned planner): NFC_PICK_*, -1 if none   */
  int32_t fixed_pick;    /* OUT (planned): the fixed planner's strategy     */
} nfc_groupby_stats;

/* Group-by with validity: probe (one D2H of 32 bytes), plan, run, read back
 * ng.  Stages (stats->stage_ms when stats->timing is set):
 *   DENSE_*:   probe, state init, aggregate, compact
 *   PARTITION: probe, histogram+plan, scatter, merge-init+aggregate
 *   HASH:      probe, table init, aggregate, extract+sort+emit  Returns ng >= 0, or a negative NFC_ERR_* code.  out_cap must be >=
 * ng (n is always enough).  stream may be NULL (legacy default stream). */
int64_t nfc_groupby(const nfc_groupby_args* args, int32_t strategy,
                    void* stream, nfc_groupby_stats* stats);

/* The fixed heuristic planner's pick for a probe (no GPU work). */
int32_t nfc_plan_strategy(const nfc_groupby_args* args, const nfc_probe* probe);

/* Stable argsort of n keys (dtype NFC_I32 / NFC_I64 / NFC_F64).  Rows whose
 * validity bit is 0 go last in input order (cpu.py:1174-1225).  descending
 * follows _stable_desc_idx (cpu.py:1154): key groups reversed, input order
 * kept inside each group.  perm_out: device int32[n]. */
int32_t nfc_sort_perm(int32_t dtype, const void* keys, const uint8_t* validity,
                      int64_t n, int32_t descending, int32_t* perm_out,
                      void* stream);

/* The first k entries of nfc_sort_perm's permutation (same order, same ties,
 * NULL rows last; sort -> slice of cpu.py:3170-3200) without sorting every
 * row: radix selection of the k-th key (11-bit digit histograms, usually one
 * pass over the column), one pass that compacts the rows it keeps and the
 * rows that tie on the selected prefix, a sort of those ties and of the k
 * kept rows.  0 <= k <= n; perm_out: device int32[k].  For k > n / 8 the
 * full argsort is used.  Synchronises the stream (digit counts are read on
 * the host). */
int32_t nfc_sort_topk(int32_t dtype, const void* keys, const uint8_t* validity,
                      int64_t n, int32_t descending, int64_t k,
                      int32_t* perm_out, void* stream);

/* out[i] = values[idx[i]] for 4- or 8-byte elements (ir_gather). */
int32_t nfc_gather(int32_t elem_bytes, const void* values, int64_t nvalues,
                   const int32_t* idx, int64_t n, void* out, void* stream);

/* Sorted unique of int32 keys with first-occurrence row, per-key count and
 * (optional) inverse codes.  Returns ng or a negative code.  uniq/first/
 * counts need capacity n; inv may be NULL. */
int64_t nfc_unique(const int32_t* keys, int64_t n, int32_t* uniq_out,
                   int32_t* first_out, int64_t* counts_out, int32_t* inv_out,
                   void* stream);

/* Grouped COUNT DISTINCT (the executor's group_count_distinct,
 * src/Drivers/CPU/_lib/cpu.py:3705-3768): per int32 key, the number of
 * distinct int32 values among rows whose key and value are both valid.
 * ukeys ascending; both outputs int64 with capacity out_cap (n always
 * suffices).  Returns ng >= 0 or a negative NFC_ERR_* code. */
int64_t nfc_group_count_distinct(const int32_t* keys, const uint8_t* key_validity,
                                 const int32_t* values, const uint8_t* value_validity,
                                 int64_t n, int64_t out_cap, int64_t* ukeys_out,
                                 int64_t* nunique_out, void* stream);

/* Dense codes of (a, b) int32 key pairs, ranked in the order of the word
 * ((a ^ a_flip) << 32) | (b ^ b_flip) (flip 0x80000000 = signed order, 0 =
 * unsigned): the building block of composite (tuple) keys, whose orders in
 * the reference's composite_tuple_index (groupindex.py:520-639) are folds of
 * such pairs.  codes_out[n] gets each row's code, or -1 for a row whose bit
 * in `validity` (LSB bitmap, NULL = all rows) is 0; ua_out/ub_out (capacity
 * n) get the pair of each code.  Returns the number of codes or a negative
 * NFC_ERR_* code. */
int64_t nfc_composite_codes(const int32_t* a, uint32_t a_flip, const int32_t* b,
                            uint32_t b_flip, const uint8_t* validity, int64_t n,
                            int32_t* codes_out, int32_t* ua_out, int32_t* ub_out,
                            void* stream);

/* Bit-packed tuple keys: the narrow alternative to composite codes.  A tuple
 * of ncols (1..NFC_MAX_KEY_COLS) int32 columns, each ordered by its bits XOR
 * flips[c] (0x80000000 signed, 0 unsigned), column 0 most significant, packs
 * into ONE non-negative int32 when the columns' flipped ranges fit in 31 bits
 * together: code = concat over c of ((col_c ^ flip_c) - min_c) in widths[c]
 * bits.  The code's integer order is the tuple order, so a group-by of the
 * codes groups the tuples in the reference's composite order without a sort.
 *
 * nfc_key_ranges: min/max of (col_c ^ flip_c) as uint32 over the rows valid
 *   in `validity` (NULL = all); `cols` is a HOST array of device pointers.
 *   Returns the number of valid rows (0: the ranges are left min > max).
 * nfc_pack_key_bits: codes_out[n] for every row (rows not valid get
 *   arbitrary codes: the caller's validity masks them); NFC_ERR_RANGE when
 *   the widths sum above 31.
 * nfc_unpack_key_bits: the inverse over ng int64 codes (group-by ukeys):
 *   cols_out (a HOST array of device pointers) get the key columns. */
#define NFC_MAX_KEY_COLS 8
int64_t nfc_key_ranges(const int32_t* const* cols, const uint32_t* flips, int ncols,
                       const uint8_t* validity, int64_t n, uint32_t* min_out,
                       uint32_t* max_out, void* stream);
int nfc_pack_key_bits(const int32_t* const* cols, const uint32_t* flips,
                      const uint32_t* mins, const int32_t* widths, int ncols, int64_t n,
                      int32_t* codes_out, void* stream);
int nfc_unpack_key_bits(const int64_t* codes, int64_t ng, const uint32_t* flips,
                        const uint32_t* mins, const int32_t* widths, int ncols,
                        int32_t* const* cols_out, void* stream);

/* Philox4x32-10 fills, bit-exact with the reference's rng_fill_i32/f64
 * (src/Drivers/CPU/_lib/rng.py:111-141): lane i uses counter offset + i. */
int32_t nfc_rng_fill_i32(int64_t n, uint64_t seed, uint64_t stream_id,
                         uint64_t offset, int64_t lo, int64_t hi, int32_t* out,
                         void* stream);
int32_t nfc_rng_fill_f64(int64_t n, uint64_t seed, uint64_t stream_id,
                         uint64_t offset, double lo, double hi, double* out,
                         void* stream);

/* Synthetic workload generators built on the same Philox lanes. */
/* lognormal(mu, sigma) by Box-Muller over two f64 streams. */
int32_t nfc_gen_lognormal(int64_t n, uint64_t seed, uint64_t stream_a,
                          uint64_t stream_b, double mu, double sigma,
                          double* out, void* stream);
/* Zipf(s) ranks over [1, domain] by continuous inverse CDF, written as
 * rank - 1. */
int32_t nfc_gen_zipf(int64_t n, uint64_t seed, uint64_t stream_id, double s,
                     int64_t domain, int32_t* out, void* stream);
/* LSB validity bitmap: bit i = (u_i >= p_null), u from one f64 stream. */
int32_t nfc_gen_validity(int64_t n, uint64_t seed, uint64_t stream_id,
                         double p_null, uint8_t* bitmap_out, void* stream);

/* ---------------------------------------------------------------------
 * Planners.  No counterpart in the reference's ABI beyond the fixed rule:
 *
 * The FIXED planner restates the reference's plan_groupby_impl
 * (src/Runtime/Planner/_lib/planner.py:200-262) with the executor's byte
 * estimates (groupindex.py:72-83, cpu.py:381-421) and its CPU buffer budget
 * (2^31 - 1 bytes): sorted keys -> SORTED; dense_by_code or shift-dense ->
 * the dense family (DENSE_SMEM / DENSE_GLOBAL / PARTITION by span, the
 * library's own split); otherwise the reference's "hash" plan, which
 * executes as a sorted unique -> SORT.
 *
 * The LEARNED planner reads a device sketch of the first 65,536 keys
 * (nfc_sketch: 256 HyperLogLog registers + 24 run/range statistics), runs
 * the MLP (nfc_mlp_forward) and picks one of four strategies; the network's
 * distinct-count estimate sizes the SHARED_HASH table.  The fixed planner
 * stays its fallback and judge: a dense pick whose span the dense family
 * cannot hold, or a pick whose softmax probability is below the planner's
 * min_confidence, runs the fixed planner's choice instead.  Results are the
 * same whichever strategy runs.
 * --------------------------------------------------------------------- */
#define NFC_SKETCH_FEATURES 280
#define NFC_MLP_IN 280
#define NFC_MLP_H 128
#define NFC_MLP_OUT 5
#define NFC_MLP_NPARAMS 53125  /* W1 b1 W2 b2 W3 b3, float32 */
#define NFC_MLP_NWEIGHTS 52864 /* W1 W2 W3, bf16 */

#define NFC_PLANNER_AUTO 0    /* the library's own span heuristic (nfc_plan_strategy) */
#define NFC_PLANNER_FIXED 1
#define NFC_PLANNER_LEARNED 2

/* Strategy classes of the learned planner's output. */
#define NFC_PICK_DENSE 0
#define NFC_PICK_SHARED_HASH 1
#define NFC_PICK_GLOBAL_HASH 2
#define NFC_PICK_SORT 3

/* 280 float32 features of the first min(n, 65536) keys (one CTA). */
int32_t nfc_sketch(const int32_t* keys, const uint8_t* key_validity, int64_t n,
                   float* features_out, void* stream);

/* MLP kernels (all device pointers).  x: batch x 280 features; feat_mu /
 * feat_sd: per-feature standardisation (both NULL = none); weights_bf16:
 * NFC_MLP_NWEIGHTS bf16; params: NFC_MLP_NPARAMS float32 (biases read from
 * here); h1, h2: batch x 128 activations (kept for backward); out: batch x 5. */
int32_t nfc_mlp_forward(const float* x, int64_t batch, const float* feat_mu,
                        const float* feat_sd, const uint16_t* weights_bf16,
                        const float* params, float* h1, float* h2, float* out,
                        void* stream);
/* grad: NFC_MLP_NPARAMS float32 (overwritten); dh1, dh2: batch x 128 scratch. */
int32_t nfc_mlp_backward(const float* x, int64_t batch, const float* feat_mu,
                         const float* feat_sd, const uint16_t* weights_bf16,
                         const float* h1, const float* h2, const float* dout,
                         float* dh1, float* dh2, float* grad, void* stream);
/* card_weight * (out0 - y_card)^2 + class_weight * w * CE(out[1..4], label)
 * per row, w = sample_weight[row] (NULL = 1); label < 0 skips the class
 * term; dout = d(mean loss)/d(out); *loss_sum += mean loss. */
int32_t nfc_mlp_loss(const float* out, const float* y_card, const int32_t* label,
                     const float* sample_weight, int64_t batch, float card_weight,
                     float class_weight, float* dout, float* loss_sum, void* stream);
/* One Adam step on the float32 parameters, then refresh the bf16 weights. */
int32_t nfc_mlp_adam(float* params, const float* grad, float* m, float* v,
                     uint16_t* weights_bf16, int64_t step, float lr, float beta1,
                     float beta2, float eps, float weight_decay, void* stream);
/* bf16 weights from the float32 parameters (round to nearest even). */
int32_t nfc_mlp_to_bf16(const float* params, uint16_t* weights_bf16, void* stream);

typedef struct nfc_planner nfc_planner;
/* Host arrays: params NFC_MLP_NPARAMS floats, mu / sd NFC_MLP_IN floats
 * (NULL = no standardisation).  Allocates the device copy on the current
 * device; NULL on error. */
nfc_planner* nfc_planner_create(const float* params, const float* feat_mu,
                                const float* feat_sd, float min_confidence);
void nfc_planner_destroy(nfc_planner* planner);
/* The fixed planner's strategy for a probe (no GPU work; naggs = aggregate
 * count as the reference counts it). */
int32_t nfc_plan_fixed(const nfc_probe* probe, int32_t naggs);
/* Group-by whose strategy is chosen by `mode` (NFC_PLANNER_*); planner may be
 * NULL unless mode is NFC_PLANNER_LEARNED.  Same arguments and result as
 * nfc_groupby. */
int64_t nfc_groupby_planned(const nfc_groupby_args* args, int32_t mode,
                            nfc_planner* planner, void* stream,
                            nfc_groupby_stats* stats);

/* ---------------------------------------------------------------------
 * Batched group-by.  No counterpart in the reference's ABI: the reference
 * runs one groupby_multi node per query (src/Drivers/CPU/_lib/cpu.py:
 * 3435-3704).  Here nq independent queries `group(key, {v: (sum, count)})`
 * over one concatenated int32 key column and one int32 value column run in
 * ONE persistent kernel launch (optionally replayed from a CUDA graph).
 * Query q owns rows [row_offsets[q], row_offsets[q+1]); per query the
 * result equals that node's: rows with a NULL key or value dropped, groups
 * in ascending key order, int64 counts and sums.
 *
 * nfc_batch_create builds the static work list (probe, solo, aggregate and
 * emit items) for the row layout and tuning and allocates the plan's device
 * memory; the same object is reused for every batch with that layout.
 * nfc_batch_run writes query q's groups to ukeys/sums/counts[group_offsets[q]
 * .. + ngroups[q]); each query reserves min(valid rows, key span) entries of
 * out_cap, so out_cap = total rows always suffices.  A query the kernel
 * cannot finish (sparse key span, state arena or out_cap exhausted, or
 * |value| * rows too large for the packed 64-bit state) is deferred and
 * finished by nfc_groupby on the host side of the call.  Returns the number
 * of deferred queries (>= 0) or a negative NFC_ERR_* code.  Flags:
 *   NFC_BATCH_GRAPH    capture the launch once into a CUDA graph (re-captured
 *                      when any pointer or out_cap changes) and replay it;
 *   NFC_BATCH_NO_SYNC  return right after enqueueing; nfc_batch_finish then
 *                      reads the status and runs deferred queries.
 * key_validity / value_validity: LSB bitmaps over the concatenated rows, or
 * NULL.  Calls on one object are serialised by a mutex; keys/values must
 * stay unchanged until the call (or nfc_batch_finish) returns.
 * --------------------------------------------------------------------- */
typedef struct nfc_batch nfc_batch;

typedef struct nfc_batch_tuning {
  int32_t solo_rows;      /* queries with rows <= solo_rows run whole in one CTA */
  int32_t chunk_rows;     /* rows per aggregate item (multiple of 8192) */
  int32_t probe_rows;     /* rows per probe item (multiple of 8192) */
  int32_t emit_slice;     /* minimum key slots per emit item (multiple of 2048) */
  int32_t emit_max_items; /* emit items per query at most */
  int32_t smem_slots;     /* shared-memory table slots per CTA (multiple of 1024) */
  int32_t smem_span_div;  /* shared-memory plan iff span <= smem_slots and span * div <= chunk_rows */
  int32_t warp_agg;       /* global-plan reductions: 0 one per row; 1 equal keys of a warp
                             combined (match_any); 2 the warp's leading key combined (ballot +
                             reduce); 3 a per-CTA shared-memory hash cache in front of them */
  int32_t ctas_per_sm;    /* resident CTAs per SM: 1 or 2 */
  int32_t schedule;       /* item order: 0 phase-major, 1 emits interleaved two queries behind, 2 solo queries last */
  int32_t agg_split;      /* 0, or cut every query into at least this many aggregate items */
  int32_t pad;
  int64_t arena_bytes;    /* device state arena; 0 = 2 bytes per row (>= 256 MiB, <= 1/4 of free memory) */
} nfc_batch_tuning;

#define NFC_BATCH_GRAPH 1
#define NFC_BATCH_NO_SYNC 2

/* Per-query plan codes reported by nfc_batch_query_plans. */
#define NFC_BATCH_PLAN_NONE 0
#define NFC_BATCH_PLAN_EMPTY 1    /* no valid rows */
#define NFC_BATCH_PLAN_SMEM 2     /* shared-memory tables flushed to the global state */
#define NFC_BATCH_PLAN_GLOBAL 3   /* warp-aggregated reductions into the global state */
#define NFC_BATCH_PLAN_DEFERRED 4 /* finished by nfc_groupby */
#define NFC_BATCH_PLAN_SOLO 5     /* one CTA, shared memory only */

void nfc_batch_default_tuning(nfc_batch_tuning* tuning);
/* row_offsets: HOST int64[nq + 1], row_offsets[0] = 0; tuning may be NULL.
 * Returns NULL on error (nfc_last_error()). */
nfc_batch* nfc_batch_create(int64_t nq, const int64_t* row_offsets,
                            const nfc_batch_tuning* tuning);
int64_t nfc_batch_run(nfc_batch* batch, const int32_t* keys,
                      const uint8_t* key_validity, const int32_t* values,
                      const uint8_t* value_validity, int64_t out_cap,
                      int64_t* ukeys_out, int64_t* sums_out,
                      int64_t* counts_out, int64_t* group_offsets,
                      int64_t* ngroups, int32_t flags, void* stream);
int64_t nfc_batch_finish(nfc_batch* batch, void* stream);
/* Plan code of every query in the last run (host int32[nq]). */
int32_t nfc_batch_query_plans(nfc_batch* batch, int32_t* plans_out,
                              void* stream);
/* SM cycles (out[0..5]) and item counts (out[6..11]) of the last run per
 * item type: probe, solo, aggregate, emit, and the aggregate items of
 * shared-memory and of global plans (summed over CTAs). */
int32_t nfc_batch_profile(nfc_batch* batch, int64_t* out, void* stream);
/* out[0..7] = nq, total rows, items, probe items, solo items, aggregate
 * items, emit items, arena bytes. */
int32_t nfc_batch_info(const nfc_batch* batch, int64_t* out, int32_t nout);
void nfc_batch_destroy(nfc_batch* batch);

/* Group-by that allocates nothing.  No counterpart in the reference: it is
 * for callers that cannot call cudaMalloc -- plugins loaded into a host
 * process whose allocator forbids foreign device allocations (the host owns
 * every byte of device memory and accounts for it), and real-time loops that
 * must not touch the allocator because an allocation can block on a device
 * synchronisation.  Scratch is one static device array of
 * NFC_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds until
 * process exit; the caller still owns inputs and outputs (same
 * nfc_groupby_args as nfc_groupby).  The call synchronises `stream` twice:
 * once to read the probe (key range, valid rows) on the host, once to read
 * the group count.
 *
 * Limits: n <= NFC_NOALLOC_MAX_ROWS, and the valid keys' span
 * (kmax - kmin + 1) times the per-group state size must fit
 * NFC_NOALLOC_STATE_BYTES (about 545K groups for one int32 and one float64
 * column with sum/min/max); otherwise NFC_ERR_RANGE and nothing is written.
 * The first call on a device looks up the array's device address in the
 * device's primary context and keeps it for the life of the process, so a
 * process that resets the device (cudaDeviceReset) must not call it again.
 * All calls share the array and the call clears what must start at zero;
 * calls that overlap on the GPU (from different streams or threads) race
 * and must be serialised by the caller.
 * Returns ng >= 0 or a negative NFC_ERR_* code. */
#define NFC_NOALLOC_MAX_ROWS (1ll << 25)
#define NFC_NOALLOC_STATE_BYTES (24ll << 20)
#define NFC_NOALLOC_SCRATCH_BYTES (32ll << 20)
int64_t nfc_groupby_dense_noalloc(const nfc_groupby_args* args, void* stream);

/* Diagnostics. */
const char* nfc_last_error(void);
int32_t nfc_version(void);

/* Self-test of the bounded waits (no counterpart in the reference, whose CPU
 * path has no cross-thread waits): runs one CTA whose decoupled look-back
 * waits on a predecessor that never publishes and whose mbarrier waits on a
 * phase that never completes, each giving up after `spins` polls.  Writes the
 * two device status words to host status_out[0..1] (NFC_ERR_TIMEOUT each when
 * the waits gave up as designed).  The library's kernels use the same waits
 * with a limit of 2^24 polls. */
int32_t nfc_selftest_bounded_waits(uint32_t spins, int32_t* status_out, void* stream);

/* Host-side fault injection for tests (no counterpart in the reference): lets
 * `after` more device scratch allocations succeed and makes the next one fail
 * as if the device were out of memory (the call then returns NFC_ERR_NOMEM),
 * then disarms itself; a negative value disarms.  Process-wide. */
int32_t nfc_debug_fail_alloc(int64_t after);

#ifdef __cplusplus
}
#endif

#endif /* NUMFAST_CUDA_H */
