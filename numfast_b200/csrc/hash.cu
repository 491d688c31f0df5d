// HASH strategy: keys whose span is too wide for a dense table.
//
// The reference routes this case to its "hash" plan, which executes as a
// sorted unique + inverse (groupindex.py:178-211, planner.py:254-262); the
// output contract is the same as every other strategy: ascending keys.
//
// Here: a global open-addressing table (linear probing, multiplicative
// hash on the raw 32-bit key; slot word = 1<<32 | key, 0 = empty) holds one
// aggregation state per distinct key.  Rows are folded in with atomics,
// the occupied slots are compacted, radix-sorted by key and emitted.
// A probe sequence longer than the table sets NFC_ERR_RANGE (cannot happen
// at the load factor used, <= 0.5), so a full table never spins.
#include <algorithm>

#include "groupby_host.h"
#include "hash_core.cuh"

namespace nfc {

__global__ void __launch_bounds__(256) k_hash_agg(const int32_t* __restrict__ keys,
                                                  const uint32_t* __restrict__ vmask, ColSet cs, int64_t n,
                                                  bool aligned, uint64_t* table, int lg, StateRef st,
                                                  int32_t* err) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (n + 127) >> 7;
  for (int64_t tile = gw; tile < ntiles; tile += nw) {
    const int64_t row0 = tile * 128 + 4 * lane;
    Tile4 t;
    if (aligned && row0 + 4 <= n) load_tile4_full<true>(keys, vmask, cs, row0, t);
    else load_tile4_tail<true>(keys, vmask, cs, row0, n, t);
    // Equal keys of a warp (hot keys, runs) are combined first; only the lane
    // that applies a row or a combined group probes the table.
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      uint64_t raw[NFC_MAX_COLS];
#pragma unroll
      for (int c = 0; c < NFC_MAX_COLS; ++c) raw[c] = t.raw[c][r];
      warp_agg_apply(cs, st, (t.valid >> r) & 1u, t.key[r], raw,
                     [&](int32_t key) { return hash_slot(table, lg, key, err); });
    }
  }
}

// Compact occupied slots -> (order-preserving key, slot).
__global__ void __launch_bounds__(256) k_hash_extract(const uint64_t* __restrict__ table, int64_t cap,
                                                      uint32_t* okeys, uint32_t* oslots, uint64_t* lb,
                                                      uint32_t* ticket, int64_t* ng_out, int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t ntiles = (cap + 1023) / 1024;
  if (tile >= ntiles) return;
  const int64_t s0 = tile * 1024 + threadIdx.x * 4;
  uint64_t w[4];
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    w[j] = s0 + j < cap ? table[s0 + j] : 0ull;
    c += w[j] ? 1u : 0u;
  }
  uint32_t total;
  const uint32_t excl = block_excl_scan(c, s_scan, &total);
  if (threadIdx.x < 32) {
    const int64_t lbx = lookback_exclusive(lb, tile, total, err);  // whole warp
    if (threadIdx.x == 0) {
      s_base = lbx;
      if (tile == ntiles - 1) *ng_out = s_base + total;
    }
  }
  __syncthreads();
  int64_t pos = s_base + excl;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (w[j]) {
      okeys[pos] = (uint32_t)w[j] ^ 0x80000000u;
      oslots[pos] = (uint32_t)(s0 + j);
      ++pos;
    }
}

__global__ void k_hash_emit(ColSet cs, StateRef st, const uint32_t* __restrict__ skeys,
                            const uint32_t* __restrict__ sslots, const int64_t* ng_ptr, OutSet o) {
  const int64_t ng = *ng_ptr;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ng; i += (int64_t)gridDim.x * blockDim.x)
    state_emit(cs, st, sslots[i], o, i, (int64_t)(int32_t)(skeys[i] ^ 0x80000000u));
}

__global__ void k_hash_clear(uint64_t* table, int64_t cap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cap; i += (int64_t)gridDim.x * blockDim.x)
    table[i] = 0ull;
}

__global__ void k_state_init_h(ColSet cs, StateRef st, int64_t slots) {
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < slots; d += (int64_t)gridDim.x * blockDim.x)
    state_init_slot(cs, st, d);
}

int run_hash(const nfc_groupby_args* a, const ColSet& cs, const OutSet& o, const nfc_probe& p,
             const uint32_t* vmask, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err,
             int64_t* slots_out, StageTimer* tm) {
  const int64_t span = p.kmax - p.kmin + 1;
  const int64_t bound = std::max<int64_t>(1, std::min<int64_t>(span, p.n_valid));
  int lg = 10;
  while ((1ll << lg) < 2 * bound) ++lg;
  const int64_t cap = 1ll << lg;
  *slots_out = cap;
  const size_t slot_bytes = state_bytes_per_slot(cs);
  uint64_t* table = nullptr;
  unsigned char* stb = nullptr;
  NFC_CUDA(sc.alloc(&table, (size_t)cap));
  NFC_CUDA(sc.alloc(&stb, (size_t)cap * slot_bytes + 64));
  const StateRef st = carve_state(cs, stb, cap);
  hash_clear_init(cs, st, table, cap, s);
  NFC_CUDA(cudaGetLastError());
  tm->launched(2);
  tm->mark(s);
  const int64_t ntiles128 = (a->n + 127) / 128;
  const unsigned ga = (unsigned)std::max<int64_t>(1, std::min<int64_t>((ntiles128 + 7) / 8, (int64_t)num_sms() * 8));
  k_hash_agg<<<ga, 256, 0, s>>>(a->keys, vmask, cs, a->n, inputs_aligned(a), table, lg, st, d_err);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  tm->mark(s);

  return hash_finish(cs, o, st, table, cap, bound, s, sc, d_ng, d_err, tm);
}

int hash_finish(const ColSet& cs, const OutSet& o, const StateRef& st, const uint64_t* table, int64_t cap,
                int64_t bound, cudaStream_t s, Scratch& sc, int64_t* d_ng, int32_t* d_err, StageTimer* tm) {
  const int64_t etiles = (cap + 1023) / 1024;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)etiles + 1));
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + etiles);
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (etiles + 1), s));
  uint32_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr;
  NFC_CUDA(sc.alloc(&k0, (size_t)bound));
  NFC_CUDA(sc.alloc(&k1, (size_t)bound));
  NFC_CUDA(sc.alloc(&v0, (size_t)bound));
  NFC_CUDA(sc.alloc(&v1, (size_t)bound));
  k_hash_extract<<<(unsigned)etiles, 256, 0, s>>>(table, cap, k0, v0, lb, ticket, d_ng, d_err);
  NFC_CUDA(cudaGetLastError());
  tm->launched();
  int64_t ng = 0;
  NFC_CUDA(cudaMemcpyAsync(&ng, d_ng, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if (ng > bound) {
    set_last_error("hash: %lld groups > bound %lld", (long long)ng, (long long)bound);
    return NFC_ERR_RANGE;
  }
  uint32_t *kr = nullptr, *vr = nullptr;
  int rc = radix_sort_u32(k0, k1, v0, v1, ng, 32, false, s, sc, d_err, &kr, &vr);
  if (rc) return rc;
  if (ng > 0) {
    k_hash_emit<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((ng + 255) / 256, (int64_t)num_sms() * 8)), 256, 0,
                  s>>>(cs, st, kr, vr, d_ng, o);
    NFC_CUDA(cudaGetLastError());
    tm->launched();
  }
  tm->mark(s);
  return NFC_OK;
}

void hash_clear_init(const ColSet& cs, const StateRef& st, uint64_t* table, int64_t cap, cudaStream_t s) {
  const unsigned g = (unsigned)std::min<int64_t>((cap + 255) / 256, (int64_t)num_sms() * 8);
  k_hash_clear<<<g, 256, 0, s>>>(table, cap);
  k_state_init_h<<<g, 256, 0, s>>>(cs, st, cap);
}

}  // namespace nfc
