// Self-test of the bounded waits every cross-CTA wait in the library uses.
//
// Kernels never spin forever: a decoupled look-back whose predecessor tile
// never publishes, or a bulk-copy mbarrier phase that never completes, gives
// up after a poll limit, records NFC_ERR_TIMEOUT in the call's status word
// and returns, so the host reads an error instead of the GPU hanging.  This
// entry point makes both waits run out on purpose (a predecessor status and
// an mbarrier that nothing ever sets) with a small poll limit and reports the
// two status words; the context stays usable afterwards.
#include "bulk.cuh"
#include "groupby_core.cuh"
#include "groupby_host.h"

namespace nfc {

__global__ void k_selftest_waits(uint64_t* status, int32_t* err, uint32_t spins) {
  __shared__ __align__(8) uint64_t bar;
  // Tile 1 of a look-back whose tile 0 never publishes (status[0] stays 0).
  if (threadIdx.x < 32) lookback_exclusive(status, 1, 5, err, spins);
  // A phase of an mbarrier that expects one arrival that never comes.
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, spins)) atomicExch(err + 1, NFC_ERR_TIMEOUT);
}

}  // namespace nfc

extern "C" int32_t nfc_selftest_bounded_waits(uint32_t spins, int32_t* status_out, void* stream) {
  using namespace nfc;
  if (!status_out) return NFC_ERR_NULL;
  if (spins == 0) return NFC_ERR_MALFORMED;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch sc(s);
  uint64_t* buf = nullptr;
  NFC_CUDA(sc.alloc(&buf, 4));  // status[2], err[2]
  NFC_CUDA(cudaMemsetAsync(buf, 0, 4 * sizeof(uint64_t), s));
  int32_t* err = reinterpret_cast<int32_t*>(buf + 2);
  k_selftest_waits<<<1, 64, 0, s>>>(buf, err, spins);
  NFC_CUDA(cudaGetLastError());
  NFC_CUDA(cudaMemcpyAsync(status_out, err, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  return NFC_OK;
}
