// Host-side entry points shared between the group-by translation units.
#pragma once

#include "groupby_core.cuh"

namespace nfc {

// Optional per-stage CUDA-event timing of one call (events on the call's
// stream, so each interval is the device time of the kernels between two
// marks) and a count of the kernels the call launched.
struct StageTimer {
  bool on = false;
  int n = 0;
  int launches = 0;
  cudaEvent_t ev[NFC_MAX_STAGES + 1] = {};
  void mark(cudaStream_t s) {
    if (!on || n > NFC_MAX_STAGES) return;
    if (!ev[n]) cudaEventCreate(&ev[n]);
    cudaEventRecord(ev[n], s);
    ++n;
  }
  void launched(int k = 1) { launches += k; }
  int finish(float* out) {
    int stages = 0;
    for (int i = 0; i + 1 < n; ++i) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) == cudaSuccess) out[stages++] = ms;
    }
    return stages;
  }
  ~StageTimer() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Strategy choice made after the probe (the learned and fixed planners).
struct PlanHook {
  virtual ~PlanHook() = default;
  // May replace *strategy and *distinct_hint; returns NFC_OK or an error.
  virtual int choose(const ColSet& cs, const nfc_probe& p, int* strategy, int64_t* distinct_hint) = 0;
};
int64_t groupby_run(const nfc_groupby_args* a, int32_t strategy, PlanHook* hook, void* stream,
                    nfc_groupby_stats* stats);

int build_colset(const nfc_groupby_args* a, ColSet* cs, OutSet* o);
bool inputs_aligned(const nfc_groupby_args* a);
// Probe records: k_probe writes one per block of kProbeBlockRows rows (in
// row order): the first and last valid key, the valid key range and count,
// and flags (bit 0: some row valid, bit 1: valid keys nondecreasing).
constexpr int kProbeChunks = 2;
constexpr int64_t kProbeSpan = 1024 * kProbeChunks;
constexpr int64_t kProbeBlockRows = 8 * kProbeSpan;
struct ProbeRec {
  int32_t first, last, kmin, kmax;
  uint32_t nvalid, flags;
};

// Probe of the call's rows: *host_probe (read back), the combined validity
// bitmap (*vmask_out, null when no input has a bitmap) and, when recs_out is
// given, the device array of ceil(n / kProbeBlockRows) probe records.
int run_probe(const nfc_groupby_args* a, cudaStream_t s, Scratch& sc, uint32_t** vmask_out,
              nfc_probe* host_probe, StageTimer* tm, const ProbeRec** recs_out = nullptr);
int plan_strategy(const ColSet& cs, const nfc_probe& p);

// PARTITION strategy (partition.cu).
int pick_partition_width(size_t slot_bytes, int64_t m, int* wb_out);
int run_partition(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
                  const uint32_t* vmask, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err,
                  int64_t* buckets_out, StageTimer* tm);

// HASH strategy (hash.cu): global open-addressing table keyed by the raw
// int32 key, then a radix sort of the occupied slots by key.
int run_hash(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
             const uint32_t* vmask, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err,
             int64_t* slots_out, StageTimer* tm);

// Shared tail of the hash strategies: compact the occupied slots of `table`
// (cap slots, at most `bound` occupied), sort them by key and emit.
int hash_finish(const ColSet& cs, const OutSet& o, const StateRef& st, const uint64_t* table, int64_t cap,
                int64_t bound, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err, StageTimer* tm);
// Zero a table of cap slots and set its state to the aggregate identities.
void hash_clear_init(const ColSet& cs, const StateRef& st, uint64_t* table, int64_t cap, cudaStream_t s);

// SHARED_HASH strategy (shash.cu): per-CTA shared-memory tables in front of a
// global table of about 2 * distinct_hint slots.  *overflow_level: 0 the
// hinted table held every key; 1 it overflowed and a retry with a table of
// 2 * min(span, valid rows) slots succeeded; 2 that retry overflowed too and
// nothing was emitted (the caller reruns the group-by as HASH).
int run_shared_hash(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
                    const uint32_t* vmask, int64_t distinct_hint, cudaStream_t s, Scratch& sc, int64_t* d_ng,
                    int32_t* d_err, int64_t* slots_out, int* overflow_level, StageTimer* tm);

// SORTED strategy (sorted.cu): valid keys nondecreasing in row order (the
// probe's sortedness flag); one pass reduces each run of equal keys, the
// probe records give every tile the last valid key before it.
int run_sorted(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
               const uint32_t* vmask, const ProbeRec* recs, cudaStream_t s, Scratch& sc, int64_t* d_ng,
               int32_t* d_err, StageTimer* tm);

// SORT strategy (sortgb.cu): stable radix sort of the valid rows by key,
// then run aggregation in key order.
int run_sort_groupby(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
                     const uint32_t* vmask, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err,
                     StageTimer* tm);
// Positions of the rows whose bit is set in an LSB bitmap, in row order;
// *nv_out (host) is their number.
int valid_positions(const uint8_t* bm, int64_t n, uint32_t* pos, int64_t* nv_out, cudaStream_t s, Scratch& sc,
                    int32_t* d_err);
// Positions of the valid rows (bit set in vmask, or all rows when vmask is
// null) sorted stably by int32 key; perm_out needs n_valid entries.
int sort_valid_rows_i32(const int32_t* keys, const uint32_t* vmask, int64_t n, int64_t n_valid, uint32_t* perm_out,
                        cudaStream_t s, Scratch& sc, int32_t* d_err);

// Key sketch (sketch.cu) into caller-provided scratch of sketch_scratch_bytes().
struct MlpRef;
// With mlp given, the sketch's last CTA also runs the network into mlp->out
// and leaves the scratch zeroed (it must be zero before the first such call).
int sketch_launch(const int32_t* keys, const uint8_t* key_validity, int64_t n, float* features_out, void* scratch,
                  cudaStream_t s, const MlpRef* mlp = nullptr);
size_t sketch_scratch_bytes();

// Radix sort (radix.cu).  Sorts (key, value) pairs ascending by the key's
// unsigned bit pattern over bits [0, key_bits); stable.  keys/vals are
// overwritten with the sorted sequence; alt buffers are scratch of n.
// vals may be null (keys only); if iota_vals is set, vals_in is ignored and
// the payload of element i is i.
int radix_sort_u32(uint32_t* keys, uint32_t* keys_alt, uint32_t* vals, uint32_t* vals_alt, int64_t n,
                   int key_bits, bool iota_vals, cudaStream_t s, Scratch& sc, int32_t* d_err,
                   uint32_t** keys_result, uint32_t** vals_result);
int radix_sort_u64(uint64_t* keys, uint64_t* keys_alt, uint32_t* vals, uint32_t* vals_alt, int64_t n,
                   int key_bits, bool iota_vals, cudaStream_t s, Scratch& sc, int32_t* d_err,
                   uint64_t** keys_result, uint32_t** vals_result);
// The same over the keys src[i] ^ in_xor of a read-only column (e.g. the
// sign flip that orders int32 as unsigned): no separate transform pass;
// keys / keys_alt are scratch of n and the result is in one of them.
int radix_sort_u32_from(const uint32_t* src, uint32_t in_xor, uint32_t* keys, uint32_t* keys_alt, uint32_t* vals,
                        uint32_t* vals_alt, int64_t n, int key_bits, bool iota_vals, cudaStream_t s, Scratch& sc,
                        int32_t* d_err, uint32_t** keys_result, uint32_t** vals_result);

}  // namespace nfc
