// Shared device/host helpers for libnumfast_cuda (sm_100a).
//
// Return codes follow the numfast-native C ABI table
// (numfast-native/src/core/errors.rs:13-38): 0 ok, -1 null pointer /
// unsorted abort, -2 out-of-range key / null state, -3 malformed /
// bad variant, -4 integer overflow, -5 unsorted (V_SORTED).  Codes
// below -5 are specific to the CUDA library (device failures).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/numfast_cuda.h"

#define NFC_DEV __device__ __forceinline__
#define NFC_HD __host__ __device__ __forceinline__

namespace nfc {

constexpr int kWarp = 32;

// Bounded spin: every wait on a flag written by another CTA gives up after
// this many polls, records NFC_ERR_TIMEOUT in the call's status word and
// returns, so a scheduling surprise can never hang the GPU.
constexpr uint32_t kSpinLimit = 1u << 24;

// ---------------------------------------------------------------------
// Host-side error plumbing.
// ---------------------------------------------------------------------
void set_last_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

#define NFC_CUDA(call)                                      \
  do {                                                      \
    cudaError_t _e = (call);                                \
    if (_e != cudaSuccess) return nfc::cuda_fail(_e, #call); \
  } while (0)

int num_sms();
void keep_pool_memory();

// Per-thread pinned host buffer of kReadbackBytes for a call's small
// device-to-host read-backs (allocated on the thread's first use and kept
// until exit; null if that allocation failed).  The allocation-free entry
// point never uses it.
constexpr size_t kReadbackBytes = 16384;
unsigned char* pinned_readback();
// Copy `bytes` of device memory to host memory `dst` and wait for the
// stream: through the pinned buffer when there is one and it is large
// enough (one DMA), else straight into dst (a pageable copy, which the
// driver stages).
cudaError_t readback(void* dst, const void* src, size_t bytes, cudaStream_t s);
// Host-side fault injection for tests (nfc_debug_fail_alloc): true when the
// scratch allocation being made is the one armed to fail.
bool alloc_fault();

// Stream-ordered scratch allocation.  Scratch is freed on the same stream
// by the RAII holder, so concurrent calls on different streams never share
// memory (the numfast-native ABI is reentrant, cpu.py:521-636 calls it from
// a thread pool).
struct Scratch {
  cudaStream_t s = nullptr;
  void* p[32] = {};
  int n = 0;
  explicit Scratch(cudaStream_t st) : s(st) { keep_pool_memory(); }
  ~Scratch() {
    for (int i = 0; i < n; ++i)
      if (p[i]) cudaFreeAsync(p[i], s);
  }
  template <class T>
  cudaError_t alloc(T** out, size_t count) {
    *out = nullptr;
    if (n >= 32) return cudaErrorMemoryAllocation;
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 256;
    if (alloc_fault()) return cudaErrorMemoryAllocation;
    void* q = nullptr;
    cudaError_t e = cudaMallocAsync(&q, bytes, s);
    if (e != cudaSuccess) return e;
    p[n++] = q;
    *out = static_cast<T*>(q);
    return cudaSuccess;
  }
};


// ---------------------------------------------------------------------
// Ordered encodings for atomic min/max of float64.
// ord(x) is monotone in x over non-NaN doubles, with -0.0 < +0.0.
// The MIN lane maps every NaN to 0 and the MAX lane maps every NaN to
// UINT64_MAX, so a NaN anywhere in a group wins both reductions (NaN
// propagates, like np.minimum/np.maximum in the reference's
// _group_minmax, Drivers/CPU/_lib/cpu.py:2470-2601).
// ---------------------------------------------------------------------
NFC_HD uint64_t f64_ord(uint64_t bits) {
  return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ull);
}
NFC_HD uint64_t f64_unord(uint64_t o) {
  return (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
}
NFC_HD bool f64_bits_isnan(uint64_t bits) {
  return (bits & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull;
}
NFC_HD uint64_t f64_min_enc(uint64_t bits) {
  return f64_bits_isnan(bits) ? 0ull : f64_ord(bits);
}
NFC_HD uint64_t f64_max_enc(uint64_t bits) {
  return f64_bits_isnan(bits) ? ~0ull : f64_ord(bits);
}
constexpr uint64_t kCanonNaN = 0x7FF8000000000000ull;
NFC_HD uint64_t f64_min_dec(uint64_t e) { return e == 0ull ? kCanonNaN : f64_unord(e); }
NFC_HD uint64_t f64_max_dec(uint64_t e) { return e == ~0ull ? kCanonNaN : f64_unord(e); }

// ---------------------------------------------------------------------
// Warp helpers.
// ---------------------------------------------------------------------
NFC_DEV unsigned lane_id() { return threadIdx.x & 31u; }
NFC_DEV unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <class T>
NFC_DEV T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

NFC_DEV uint32_t ld_volatile_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
NFC_DEV uint64_t ld_volatile_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

// Bit i of an LSB-first validity bitmap (Arrow layout).
NFC_DEV bool bit_at(const uint8_t* bm, int64_t i) {
  return (bm[i >> 3] >> (i & 7)) & 1u;
}

}  // namespace nfc
