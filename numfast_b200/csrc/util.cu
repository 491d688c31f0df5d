// Error plumbing and device queries shared by every translation unit.
#include <stdarg.h>
#include <stdio.h>

#include <atomic>
#include <cstring>

#include "nfc_common.cuh"

namespace nfc {

static thread_local char g_last_error[512] = "";

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int cuda_fail(cudaError_t e, const char* what) {
  set_last_error("%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
  return e == cudaErrorMemoryAllocation ? NFC_ERR_NOMEM : NFC_ERR_CUDA;
}

int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached[dev] = v;
  }
  return cached[dev];
}

// Stream-ordered scratch comes from the device's default memory pool.  By
// default the pool returns memory to the OS at every synchronisation, which
// would re-map gigabytes of scratch on every call; keep it instead (once per
// device).
void keep_pool_memory() {
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done[dev] = true;
}

unsigned char* pinned_readback() {
  thread_local unsigned char* p = nullptr;
  thread_local bool tried = false;
  if (!tried) {
    tried = true;
    if (cudaMallocHost(reinterpret_cast<void**>(&p), kReadbackBytes) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();  // clear the failure: the pageable copies still work
    }
  }
  return p;
}

cudaError_t readback(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  unsigned char* pin = bytes <= kReadbackBytes ? pinned_readback() : nullptr;
  cudaError_t e = cudaMemcpyAsync(pin ? static_cast<void*>(pin) : dst, src, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && pin) std::memcpy(dst, pin, bytes);
  return e;
}

// Armed count for nfc_debug_fail_alloc: k >= 0 lets k more scratch
// allocations succeed and fails the next one (then disarms); -1 is off.
static std::atomic<int64_t> g_alloc_fault{-1};

bool alloc_fault() {
  int64_t v = g_alloc_fault.load(std::memory_order_relaxed);
  while (v >= 0)
    if (g_alloc_fault.compare_exchange_weak(v, v - 1)) return v == 0;
  return false;
}

}  // namespace nfc

extern "C" int32_t nfc_debug_fail_alloc(int64_t after) {
  nfc::g_alloc_fault.store(after < 0 ? -1 : after);
  return NFC_OK;
}

extern "C" const char* nfc_last_error(void) { return nfc::g_last_error; }
extern "C" int32_t nfc_version(void) { return 1; }
