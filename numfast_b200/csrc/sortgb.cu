// SORT strategy: group-by through a stable sort of the valid rows by key.
//
// This is how the reference executes its "hash" plan for keys too sparse
// for a dense index: a sorted unique with inverse codes, then per-group
// bincounts (src/Drivers/CPU/_lib/groupindex.py:178-211; planner.py:254-262).
// Here:
//   1. positions of the valid rows, sorted stably by key (onesweep radix
//      sort of (key, row) pairs, radix.cu)
//   2. k_sort_runs: tiles of 1024 sorted positions; run heads by comparing
//      neighbouring keys, run ids by a block scan plus a decoupled look-back
//      across tiles; rows fold into a shared-memory state indexed by the
//      tile-local run, and each tile-local run is merged once into the
//      global state slot of its run id (so a long run costs one set of
//      global atomics per tile, not per row)
//   3. k_sort_emit: run r -> output r (runs are already in key order).
#include <algorithm>

#include "agg_smem.cuh"
#include "groupby_host.h"

namespace nfc {
namespace {

constexpr int kSrThreads = 256;
constexpr int kSrTile = kSrThreads * 4;

NFC_DEV uint64_t load_raw(const ColSet& cs, int c, int dt, int64_t row) {
  return dt == NFC_I32 ? (uint64_t)(int64_t) static_cast<const int32_t*>(cs.data[c])[row]
                       : static_cast<const uint64_t*>(cs.data[c])[row];
}

template <int NC, uint32_t SIG>
__global__ void __launch_bounds__(kSrThreads) k_sort_runs(const int32_t* __restrict__ keys,
                                                         const uint32_t* __restrict__ perm, int64_t nv, ColSet cs,
                                                         StateRef gst, int64_t* ukeys, uint64_t* lb,
                                                         uint32_t* ticket, int64_t* ng_out, int32_t* err) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  __shared__ int s_cont;
  const AggState<NC> st = carve_agg<NC, SIG>(cs, sm, kSrTile);
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  for (int g = threadIdx.x; g < kSrTile; g += kSrThreads) agg_init<NC, SIG>(cs, st, g);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t ntiles = (nv + kSrTile - 1) / kSrTile;
  if (tile >= ntiles) return;
  const int64_t i0 = tile * kSrTile + (int64_t)threadIdx.x * 4;
  uint32_t row[4];
  int32_t k[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    row[j] = i0 + j < nv ? perm[i0 + j] : 0u;
    k[j] = i0 + j < nv ? keys[row[j]] : 0;
  }
  const int32_t prev = (i0 > 0 && i0 < nv) ? keys[perm[i0 - 1]] : 0;
  uint32_t heads = 0, c = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t i = i0 + j;
    if (i < nv && (i == 0 || (j == 0 ? prev != k[0] : k[j - 1] != k[j]))) {
      heads |= 1u << j;
      ++c;
    }
  }
  // Tile-local run index of this thread's first element: heads before it
  // in the tile, minus one unless the tile itself starts a run there.
  uint32_t total;
  const uint32_t excl = block_excl_scan(c, s_scan, &total);
  if (threadIdx.x < 32) {
    // base = runs whose head lies in earlier tiles.  A tile whose first
    // element is not a head continues run base - 1 in its local slot 0.
    const int64_t lbx = lookback_exclusive(lb, tile, total, err);  // whole warp
    if (threadIdx.x == 0) {
      s_base = lbx;
      s_cont = (heads & 1u) ? 0 : 1;
      if (tile == ntiles - 1) *ng_out = s_base + total;
    }
  }
  __syncthreads();
  const int64_t base = s_base;
  // Local slot l holds run base + l - shift.
  const int shift = s_cont;
  int32_t l = (int32_t)excl - 1 + shift;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t i = i0 + j;
    if (i >= nv) break;
    if (heads & (1u << j)) {
      ++l;
      ukeys[base + l - shift] = k[j];
    }
    uint64_t raw[NC > 0 ? NC : 1];
#pragma unroll
    for (int cc = 0; cc < NC; ++cc) raw[cc] = load_raw(cs, cc, col_dt<SIG>(cs, cc), row[j]);
    agg_apply<NC, SIG>(cs, st, (uint32_t)l, raw);
  }
  __syncthreads();
  const int nloc = (int)total + shift;
  for (int g = threadIdx.x; g < nloc; g += kSrThreads) agg_merge<NC, SIG>(cs, gst, base + g - shift, st, g);
}

__global__ void k_sort_state_init(ColSet cs, StateRef st, int64_t slots) {
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < slots; d += (int64_t)gridDim.x * blockDim.x)
    state_init_slot(cs, st, d);
}

__global__ void k_sort_emit(ColSet cs, StateRef st, const int64_t* ng_ptr, OutSet o) {
  const int64_t ng = *ng_ptr;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < ng; r += (int64_t)gridDim.x * blockDim.x)
    state_emit(cs, st, r, o, r, o.ukeys[r]);
}

constexpr uint32_t kSigI32Sum = sig_col(0, NFC_I32, NFC_AGG_SUM);

template <int NC, uint32_t SIG>
int launch_runs(const int32_t* keys, const uint32_t* perm, int64_t nv, const ColSet& cs, const StateRef& gst,
                int64_t* ukeys, uint64_t* lb, uint32_t* ticket, int64_t* d_ng, int32_t* d_err, size_t slot_bytes,
                cudaStream_t s) {
  const size_t smem = slot_bytes * kSrTile + 64;
  NFC_CUDA(cudaFuncSetAttribute(k_sort_runs<NC, SIG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t ntiles = (nv + kSrTile - 1) / kSrTile;
  k_sort_runs<NC, SIG><<<(unsigned)ntiles, kSrThreads, smem, s>>>(keys, perm, nv, cs, gst, ukeys, lb, ticket, d_ng,
                                                                  d_err);
  NFC_CUDA(cudaGetLastError());
  return NFC_OK;
}

}  // namespace

int run_sort_groupby(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
                     const uint32_t* vmask, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err,
                     StageTimer* tm) {
  const int64_t nv = p.n_valid;
  if (nv == 0) return NFC_OK;
  const int64_t span = p.kmax - p.kmin + 1;
  const int64_t bound = std::max<int64_t>(1, std::min<int64_t>(span, nv));
  uint32_t* perm = nullptr;
  NFC_CUDA(sc.alloc(&perm, (size_t)std::max<int64_t>(nv, 1)));
  int rc = sort_valid_rows_i32(a->keys, vmask, a->n, nv, perm, s, sc, d_err);
  if (rc) return rc;
  tm->mark(s);
  const size_t slot_bytes = state_bytes_per_slot(cs);
  unsigned char* stb = nullptr;
  NFC_CUDA(sc.alloc(&stb, (size_t)bound * slot_bytes + 64));
  const StateRef gst = carve_state(cs, stb, bound);
  const unsigned gi = (unsigned)std::max<int64_t>(1, std::min<int64_t>((bound + 255) / 256, (int64_t)num_sms() * 8));
  k_sort_state_init<<<gi, 256, 0, s>>>(cs, gst, bound);
  NFC_CUDA(cudaGetLastError());
  const int64_t ntiles = (nv + kSrTile - 1) / kSrTile;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 1));
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles);
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 1), s));
  // The smem state of a 1024-row tile reuses the 16-bit split sums: exact.
  switch (cs.ncols) {
    case 0: rc = launch_runs<0, 0>(a->keys, perm, nv, cs, gst, o.ukeys, lb, ticket, d_ng, d_err, slot_bytes, s); break;
    case 1:
      rc = sig_of(cs) == kSigI32Sum
               ? launch_runs<1, kSigI32Sum>(a->keys, perm, nv, cs, gst, o.ukeys, lb, ticket, d_ng, d_err, slot_bytes, s)
               : launch_runs<1, 0>(a->keys, perm, nv, cs, gst, o.ukeys, lb, ticket, d_ng, d_err, slot_bytes, s);
      break;
    case 2: rc = launch_runs<2, 0>(a->keys, perm, nv, cs, gst, o.ukeys, lb, ticket, d_ng, d_err, slot_bytes, s); break;
    case 3: rc = launch_runs<3, 0>(a->keys, perm, nv, cs, gst, o.ukeys, lb, ticket, d_ng, d_err, slot_bytes, s); break;
    default: rc = launch_runs<4, 0>(a->keys, perm, nv, cs, gst, o.ukeys, lb, ticket, d_ng, d_err, slot_bytes, s); break;
  }
  if (rc) return rc;
  tm->launched(2);
  tm->mark(s);
  k_sort_emit<<<gi, 256, 0, s>>>(cs, gst, d_ng, o);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);
  return NFC_OK;
}

}  // namespace nfc
