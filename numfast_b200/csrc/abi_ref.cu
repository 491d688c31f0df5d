// numfast-native C ABI on the GPU: host buffers in, host buffers out.
//
// Each nf_* entry point keeps the reference's name, argument meaning and
// return codes (numfast-native/src/lib.rs, errors.rs:13-38), so the
// reference's ctypes loader (native_cpu.py:93-143) binds this library
// unchanged through NUMFAST_NATIVE_DLL.  Inputs are staged to the GPU on a
// per-thread stream with stream-ordered scratch, so the entry points are
// reentrant (native_cpu's thread pool calls them concurrently with disjoint
// outputs, cpu.py:521-636).
//
// Integer results are exact.  Checked int32/int64 sums reproduce the
// reference's "a running per-group sum in row order left the type" rule
// (add_i32_checked / add_i64_checked, series/reduce.rs): a cheap bound
// (per-group sum of |v|) proves most inputs safe; otherwise rows are
// stably sorted by key on the GPU and every group's prefix sums are
// checked in row order.  float64 sums use atomics (order differs from the
// reference's sequential loop; within 1e-12 relative for well-conditioned
// sums, the reference's own tolerance).
#include <string.h>

#include <algorithm>
#include <vector>

#include "groupby_host.h"

namespace nfc {

static cudaStream_t thread_stream() {
  thread_local cudaStream_t s = nullptr;
  if (!s) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  return s;
}

static unsigned grid_n(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8));
}

// Flags word layout (device int32[4]): [0] first out-of-range row + 1 (min),
// [1] status, [2] definite overflow, [3] needs ordered overflow check.
struct CodeScatter {
  const int32_t* keys;
  int64_t n;
  int64_t g;
  unsigned long long* counts;  // may be null
  // f64 lanes
  int nf;
  const double* fv;            // nf*n SoA
  double* fs;                  // nf*g
  // integer lanes (accumulated exactly in int64, checked on the host side)
  int ni;
  int ibytes;                  // 4 or 8
  const void* iv;              // ni*n SoA
  unsigned long long* is;      // ni*g (int64 two's complement)
  double* iabs;                // ni*g sum of |v| (bound)
  int64_t lo, hi;              // only groups in [lo, hi) are accumulated
  int32_t* flags;
};

__global__ void k_code_scatter(CodeScatter a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = a.keys[i];
    if (k < 0 || (int64_t)k >= a.g) {
      atomicMin(&a.flags[0], (int32_t)std::min<int64_t>(i, INT32_MAX - 1));
      continue;
    }
    if (k < a.lo || k >= a.hi) continue;
    if (a.counts) atomicAdd(&a.counts[k], 1ull);
    for (int c = 0; c < a.nf; ++c) atomicAdd(&a.fs[(int64_t)c * a.g + k], a.fv[(int64_t)c * a.n + i]);
    for (int c = 0; c < a.ni; ++c) {
      const int64_t v = a.ibytes == 4 ? (int64_t) static_cast<const int32_t*>(a.iv)[(int64_t)c * a.n + i]
                                      : static_cast<const int64_t*>(a.iv)[(int64_t)c * a.n + i];
      atomicAdd(&a.is[(int64_t)c * a.g + k], (unsigned long long)v);
      atomicAdd(&a.iabs[(int64_t)c * a.g + k], fabs((double)v));
    }
  }
}

// Rows sorted by key (stable): one thread per run walks it in row order
// with checked adds; sets flags[2] on the first overflow.
__global__ void k_ordered_check(const int32_t* skeys, const uint32_t* perm, int64_t n, int ni, int ibytes,
                                const void* iv, int64_t nrows_total, int32_t* flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (i > 0 && skeys[i - 1] == skeys[i]) continue;  // not a run head
    for (int c = 0; c < ni; ++c) {
      int64_t acc = 0;
      for (int64_t j = i; j < n && skeys[j] == skeys[i]; ++j) {
        const int64_t row = perm[j];
        const int64_t v = ibytes == 4 ? (int64_t) static_cast<const int32_t*>(iv)[(int64_t)c * nrows_total + row]
                                      : static_cast<const int64_t*>(iv)[(int64_t)c * nrows_total + row];
        if (ibytes == 4) {
          acc += v;
          if (acc > INT32_MAX || acc < INT32_MIN) { atomicExch(&flags[2], 1); break; }
        } else {
          const long long r = (long long)((unsigned long long)acc + (unsigned long long)v);
          if (((acc ^ r) & (v ^ r)) < 0) { atomicExch(&flags[2], 1); break; }
          acc = r;
        }
      }
    }
  }
}

// RAII device copy of a host buffer.
struct Dev {
  Scratch& sc;
  explicit Dev(Scratch& s) : sc(s) {}
  template <class T>
  int up(const T* h, size_t count, T** d) {
    NFC_CUDA(sc.alloc(d, count));
    if (count) NFC_CUDA(cudaMemcpyAsync(*d, h, count * sizeof(T), cudaMemcpyHostToDevice, sc.s));
    return NFC_OK;
  }
  template <class T>
  int zeros(size_t count, T** d) {
    NFC_CUDA(sc.alloc(d, count));
    NFC_CUDA(cudaMemsetAsync(*d, 0, std::max<size_t>(count, 1) * sizeof(T), sc.s));
    return NFC_OK;
  }
};

template <class T>
static int down(cudaStream_t s, T* h, const T* d, size_t count) {
  if (count) NFC_CUDA(cudaMemcpyAsync(h, d, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  return NFC_OK;
}

int argsort_i32_device(const int32_t* keys, int64_t n, uint32_t* perm, cudaStream_t s, Scratch& sc, int32_t* d_err);

struct ScatterSpec {
  const int32_t* keys;
  size_t n, g;
  bool counts;
  int nf;
  const double* fv;
  int ni, ibytes;
  const void* iv;
  size_t lo, hi;
  bool int_checked;  // apply the running-sum overflow rule
  int64_t int_min, int_max;
  // Fused pack (nf_pack_sum_count_*): when set, the group code of row i is
  // keys[i] * m2 + keys2[i], formed on the device.
  const int32_t* keys2 = nullptr;
  int32_t m2 = 0;
};

struct ScatterOut {
  std::vector<int64_t> counts;
  std::vector<double> fs;
  std::vector<int64_t> is;
};

// Composite code k1 * m2 + k2 of every row (pack_elem, core/numeric.rs:24):
// a negative component or a code above INT32_MAX marks the row out of range
// (first such row in flags[0]) and leaves code -1, which the scatter skips.
__global__ void k_pack_codes(const int32_t* k1, const int32_t* k2, int32_t m2, int64_t n, int32_t* out,
                             int32_t* flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = k1[i], b = k2[i];
    const int64_t v = (int64_t)a * (int64_t)m2 + (int64_t)b;
    const bool ok = a >= 0 && b >= 0 && v <= INT32_MAX;
    if (!ok) atomicMin(&flags[0], (int32_t)std::min<int64_t>(i, INT32_MAX - 1));
    out[i] = ok ? (int32_t)v : -1;
  }
}

// Returns 0, -2 (range), -4 (overflow) or a CUDA error.
static int scatter_codes(const ScatterSpec& sp, ScatterOut& out) {
  cudaStream_t s = thread_stream();
  Scratch sc(s);
  Dev dv(sc);
  int32_t* dkeys = nullptr;
  int rc = dv.up(sp.keys, sp.n, &dkeys);
  if (rc) return rc;
  int32_t* dkeys2 = nullptr;
  if (sp.keys2 && (rc = dv.up(sp.keys2, sp.n, &dkeys2))) return rc;
  CodeScatter a{};
  a.keys = dkeys;
  a.n = (int64_t)sp.n;
  a.g = (int64_t)sp.g;
  a.lo = (int64_t)sp.lo;
  a.hi = (int64_t)sp.hi;
  int32_t* flags = nullptr;
  NFC_CUDA(sc.alloc(&flags, 4));
  const int32_t init[4] = {INT32_MAX, 0, 0, 0};
  NFC_CUDA(cudaMemcpyAsync(flags, init, sizeof(init), cudaMemcpyHostToDevice, s));
  a.flags = flags;
  if (dkeys2 && sp.n > 0) {
    // Codes overwrite the staged first key column in place.
    k_pack_codes<<<grid_n((int64_t)sp.n), 256, 0, s>>>(dkeys, dkeys2, sp.m2, (int64_t)sp.n, dkeys, flags);
    NFC_CUDA(cudaGetLastError());
  }
  if (sp.counts && (rc = dv.zeros(sp.g, &a.counts))) return rc;
  a.nf = sp.nf;
  if (sp.nf > 0) {
    double* d = nullptr;
    if ((rc = dv.up(sp.fv, (size_t)sp.nf * sp.n, &d))) return rc;
    a.fv = d;
    if ((rc = dv.zeros((size_t)sp.nf * sp.g, &a.fs))) return rc;
  }
  a.ni = sp.ni;
  a.ibytes = sp.ibytes;
  if (sp.ni > 0) {
    unsigned char* d = nullptr;
    if ((rc = dv.up(static_cast<const unsigned char*>(sp.iv), (size_t)sp.ni * sp.n * sp.ibytes, &d))) return rc;
    a.iv = d;
    if ((rc = dv.zeros((size_t)sp.ni * sp.g, &a.is))) return rc;
    if ((rc = dv.zeros((size_t)sp.ni * sp.g, &a.iabs))) return rc;
  }
  if (sp.n > 0) {
    k_code_scatter<<<grid_n((int64_t)sp.n), 256, 0, s>>>(a);
    NFC_CUDA(cudaGetLastError());
  }
  int32_t hflags[4];
  NFC_CUDA(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, s));
  out.counts.assign(sp.counts ? sp.g : 0, 0);
  out.fs.assign((size_t)sp.nf * sp.g, 0.0);
  out.is.assign((size_t)sp.ni * sp.g, 0);
  std::vector<double> iabs((size_t)sp.ni * sp.g, 0.0);
  if (sp.counts && (rc = down(s, reinterpret_cast<unsigned long long*>(out.counts.data()), a.counts, sp.g))) return rc;
  if (sp.nf && (rc = down(s, out.fs.data(), a.fs, (size_t)sp.nf * sp.g))) return rc;
  if (sp.ni && (rc = down(s, reinterpret_cast<unsigned long long*>(out.is.data()), a.is, (size_t)sp.ni * sp.g))) return rc;
  if (sp.ni && (rc = down(s, iabs.data(), a.iabs, (size_t)sp.ni * sp.g))) return rc;
  NFC_CUDA(cudaStreamSynchronize(s));
  if (hflags[0] != INT32_MAX) return NFC_ERR_RANGE;
  if (!sp.int_checked || sp.ni == 0) return NFC_OK;
  // Running-sum overflow rule.
  bool ambiguous = false;
  for (size_t i = 0; i < out.is.size(); ++i) {
    if (sp.ibytes == 4 && (out.is[i] > sp.int_max || out.is[i] < sp.int_min)) return NFC_ERR_OVERFLOW;
    if (iabs[i] > (double)sp.int_max * (sp.ibytes == 4 ? 1.0 : 0.5)) ambiguous = true;
  }
  if (!ambiguous) return NFC_OK;
  uint32_t* perm = nullptr;
  NFC_CUDA(sc.alloc(&perm, sp.n));
  if ((rc = argsort_i32_device(dkeys, (int64_t)sp.n, perm, s, sc, flags + 1))) return rc;
  int32_t* skeys = nullptr;
  NFC_CUDA(sc.alloc(&skeys, sp.n));
  rc = nfc_gather(4, dkeys, (int64_t)sp.n, reinterpret_cast<const int32_t*>(perm), (int64_t)sp.n, skeys, s);
  if (rc) return rc;
  k_ordered_check<<<grid_n((int64_t)sp.n), 256, 0, s>>>(skeys, perm, (int64_t)sp.n, sp.ni, sp.ibytes, a.iv,
                                                        (int64_t)sp.n, flags);
  NFC_CUDA(cudaGetLastError());
  NFC_CUDA(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if (hflags[1]) return hflags[1];
  return hflags[2] ? NFC_ERR_OVERFLOW : NFC_OK;
}

// Sortedness check: flag stays 1 if keys nondecreasing.  One store per CTA
// that saw a descent (a store per descending row would pile every row of an
// unsorted column onto one address).
__global__ void k_is_sorted(const int32_t* k, int64_t n, int32_t* flag) {
  bool desc = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x + 1; i < n; i += (int64_t)gridDim.x * blockDim.x)
    desc |= k[i] < k[i - 1];
  if (__syncthreads_or(desc) && threadIdx.x == 0) atomicExch(flag, 0);
}

static int keys_sorted(const int32_t* hkeys, size_t n, bool* sorted) {
  *sorted = true;
  if (n < 2) return NFC_OK;
  cudaStream_t s = thread_stream();
  Scratch sc(s);
  Dev dv(sc);
  int32_t* dk = nullptr;
  int rc = dv.up(hkeys, n, &dk);
  if (rc) return rc;
  int32_t* flag = nullptr;
  NFC_CUDA(sc.alloc(&flag, 1));
  const int32_t one = 1;
  NFC_CUDA(cudaMemcpyAsync(flag, &one, sizeof(one), cudaMemcpyHostToDevice, s));
  k_is_sorted<<<grid_n((int64_t)n), 256, 0, s>>>(dk, (int64_t)n, flag);
  NFC_CUDA(cudaGetLastError());
  int32_t h = 1;
  NFC_CUDA(cudaMemcpyAsync(&h, flag, sizeof(h), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  *sorted = h != 0;
  return NFC_OK;
}

// Dense compaction of (counts_m, sums_m) -> (ukeys, counts, sums), 8-byte sums.
__global__ void __launch_bounds__(256) k_carry(const int64_t* cm, const uint64_t* sm, int64_t m, int64_t* uk,
                                               int64_t* cnt, uint64_t* sums, uint64_t* lb, uint32_t* ticket,
                                               int64_t* ng_out, int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile, ntiles = (m + 1023) / 1024;
  if (tile >= ntiles) return;
  const int64_t j0 = tile * 1024 + threadIdx.x * 4;
  uint32_t c = 0, pres = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (j0 + j < m && cm[j0 + j] != 0) { pres |= 1u << j; ++c; }
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
  int64_t p = s_base + excl;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (pres & (1u << j)) {
      uk[p] = j0 + j;
      cnt[p] = cm[j0 + j];
      sums[p] = sm[j0 + j];
      ++p;
    }
}

static int64_t carry_build(const int64_t* counts_m, const uint64_t* sums_m, size_t m, int64_t* ukeys, int64_t* counts,
                           uint64_t* sums) {
  cudaStream_t s = thread_stream();
  Scratch sc(s);
  Dev dv(sc);
  int64_t* dcm = nullptr;
  uint64_t* dsm = nullptr;
  int rc;
  if ((rc = dv.up(counts_m, m, &dcm)) || (rc = dv.up(sums_m, m, &dsm))) return rc;
  int64_t *duk = nullptr, *dcn = nullptr;
  uint64_t* dsu = nullptr;
  NFC_CUDA(sc.alloc(&duk, m));
  NFC_CUDA(sc.alloc(&dcn, m));
  NFC_CUDA(sc.alloc(&dsu, m));
  const int64_t ntiles = ((int64_t)m + 1023) / 1024;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 3));
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 3), s));
  int64_t* dng = reinterpret_cast<int64_t*>(lb + ntiles);
  int32_t* derr = reinterpret_cast<int32_t*>(lb + ntiles + 1);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles + 2);
  k_carry<<<(unsigned)ntiles, 256, 0, s>>>(dcm, dsm, (int64_t)m, duk, dcn, dsu, lb, ticket, dng, derr);
  NFC_CUDA(cudaGetLastError());
  int64_t h[2] = {0, 0};
  NFC_CUDA(cudaMemcpyAsync(h, dng, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  const int64_t ng = h[0];
  if ((int32_t)h[1]) return (int32_t)h[1];
  if ((rc = down(s, ukeys, duk, (size_t)ng)) || (rc = down(s, counts, dcn, (size_t)ng)) ||
      (rc = down(s, sums, dsu, (size_t)ng)))
    return rc;
  NFC_CUDA(cudaStreamSynchronize(s));
  return ng;
}

// Sorted runs over nondecreasing keys (sorted.rs:24-56): heads, run sums.
__global__ void __launch_bounds__(256) k_sorted_runs(const int32_t* k, const uint64_t* v, bool is_f64, int64_t n,
                                                     int64_t* uk, uint64_t* sums, int64_t* cnt, uint64_t* lb,
                                                     uint32_t* ticket, int64_t* ng_out, int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile, ntiles = (n + 1023) / 1024;
  if (tile >= ntiles) return;
  const int64_t i0 = tile * 1024 + threadIdx.x * 4;
  uint32_t c = 0, heads = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t i = i0 + j;
    if (i < n && (i == 0 || k[i] != k[i - 1])) { heads |= 1u << j; ++c; }
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
  int64_t r = s_base + excl - 1;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t i = i0 + j;
    if (i >= n) break;
    if (heads & (1u << j)) {
      ++r;
      uk[r] = k[i];
      // Sequential run sum in row order, like the reference loop.
      int64_t e = i + 1;
      uint64_t acc = v[i];
      int64_t ct = 1;
      while (e < n && k[e] == k[i]) {
        if (is_f64) acc = __double_as_longlong(__longlong_as_double((long long)acc) + __longlong_as_double((long long)v[e]));
        else acc += v[e];
        ++e;
        ++ct;
      }
      sums[r] = acc;
      cnt[r] = ct;
    }
  }
}

static int64_t sorted_run(const int32_t* keys, const uint64_t* vals, bool is_f64, size_t n, int64_t* ukeys,
                          uint64_t* sums, int64_t* counts) {
  bool sorted = true;
  int rc = keys_sorted(keys, n, &sorted);
  if (rc) return rc;
  if (!sorted) return -1;
  cudaStream_t s = thread_stream();
  Scratch sc(s);
  Dev dv(sc);
  int32_t* dk = nullptr;
  uint64_t* dv_ = nullptr;
  if ((rc = dv.up(keys, n, &dk)) || (rc = dv.up(vals, n, &dv_))) return rc;
  int64_t *duk = nullptr, *dcn = nullptr;
  uint64_t* dsu = nullptr;
  NFC_CUDA(sc.alloc(&duk, n));
  NFC_CUDA(sc.alloc(&dcn, n));
  NFC_CUDA(sc.alloc(&dsu, n));
  const int64_t ntiles = ((int64_t)n + 1023) / 1024;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 3));
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 3), s));
  int64_t* dng = reinterpret_cast<int64_t*>(lb + ntiles);
  int32_t* derr = reinterpret_cast<int32_t*>(lb + ntiles + 1);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles + 2);
  k_sorted_runs<<<(unsigned)ntiles, 256, 0, s>>>(dk, dv_, is_f64, (int64_t)n, duk, dsu, dcn, lb, ticket, dng, derr);
  NFC_CUDA(cudaGetLastError());
  int64_t h[2] = {0, 0};
  NFC_CUDA(cudaMemcpyAsync(h, dng, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if ((int32_t)h[1]) return (int32_t)h[1];
  const int64_t ng = h[0];
  if ((rc = down(s, ukeys, duk, (size_t)ng)) || (rc = down(s, counts, dcn, (size_t)ng)) ||
      (rc = down(s, sums, dsu, (size_t)ng)))
    return rc;
  NFC_CUDA(cudaStreamSynchronize(s));
  return ng;
}

}  // namespace nfc

using namespace nfc;

// ---------------------------------------------------------------------
// Group-by family.
// ---------------------------------------------------------------------
extern "C" int32_t nf_group_sum_count(const int32_t* keys, const double* values, size_t n, double* sums,
                                      int64_t* counts, size_t g) {
  if (!keys || !values || !sums || !counts) return NFC_ERR_NULL;
  ScatterSpec sp{keys, n, g, true, 1, values, 0, 4, nullptr, 0, g, false, 0, 0};
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  memcpy(sums, o.fs.data(), g * sizeof(double));
  memcpy(counts, o.counts.data(), g * sizeof(int64_t));
  return NFC_OK;
}

extern "C" int32_t nf_group_multi_sum_count(const int32_t* keys, const double* values, size_t n, size_t ncols,
                                            double* sums, int64_t* counts, size_t g) {
  if (!keys || !values || !sums || !counts) return NFC_ERR_NULL;
  ScatterSpec sp{keys, n, g, true, (int)ncols, values, 0, 4, nullptr, 0, g, false, 0, 0};
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  memcpy(sums, o.fs.data(), ncols * g * sizeof(double));
  memcpy(counts, o.counts.data(), g * sizeof(int64_t));
  return NFC_OK;
}

extern "C" int32_t nf_group_mixed_sum_only(const int32_t* keys, const int32_t* i32_vals, const double* f64_vals,
                                           size_t n, size_t n_i32, size_t n_f64, int32_t* i32_sums,
                                           double* f64_sums, size_t g) {
  if (!keys) return NFC_ERR_NULL;
  if ((n_i32 > 0 && (!i32_vals || !i32_sums)) || (n_f64 > 0 && (!f64_vals || !f64_sums))) return NFC_ERR_NULL;
  ScatterSpec sp{keys, n, g, false, (int)n_f64, f64_vals, (int)n_i32, 4, i32_vals, 0, g, true, INT32_MIN, INT32_MAX};
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  for (size_t i = 0; i < n_i32 * g; ++i) i32_sums[i] = (int32_t)o.is[i];
  if (n_f64) memcpy(f64_sums, o.fs.data(), n_f64 * g * sizeof(double));
  return NFC_OK;
}

extern "C" int32_t nf_group_count_only(const int32_t* keys, size_t n, int64_t* counts, size_t g) {
  if (!keys || !counts) return NFC_ERR_NULL;
  ScatterSpec sp{keys, n, g, true, 0, nullptr, 0, 4, nullptr, 0, g, false, 0, 0};
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  memcpy(counts, o.counts.data(), g * sizeof(int64_t));
  return NFC_OK;
}

extern "C" int32_t nf_group_owner_2i32_1f64(const int32_t* keys, const int32_t* a, const int32_t* b, const double* c,
                                            size_t n, size_t lo, size_t hi, int32_t* s1, int32_t* s2, double* s3,
                                            int64_t* counts, size_t g) {
  if (!keys || !a || !b || !c || !s1 || !s2 || !s3 || !counts || lo > hi || hi > g) return NFC_ERR_NULL;
  std::vector<int32_t> ab(2 * n);
  if (n) {
    memcpy(ab.data(), a, n * sizeof(int32_t));
    memcpy(ab.data() + n, b, n * sizeof(int32_t));
  }
  ScatterSpec sp{keys, n, g, true, 1, c, 2, 4, ab.data(), lo, hi, true, INT32_MIN, INT32_MAX};
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  for (size_t k = lo; k < hi; ++k) {
    s1[k] = (int32_t)o.is[k];
    s2[k] = (int32_t)o.is[g + k];
    s3[k] = o.fs[k];
    counts[k] = o.counts[k];
  }
  return NFC_OK;
}

extern "C" int32_t nf_group_variant_f64(const int32_t* keys, const double* values, size_t n, uint32_t variant,
                                        double* sums, int64_t* counts, size_t g) {
  if (!keys || !values || !sums || !counts) return NFC_ERR_NULL;
  if (variant > 2) return NFC_ERR_MALFORMED;
  if (variant == 2) {
    bool sorted = true;
    const int rc = keys_sorted(keys, n, &sorted);
    if (rc) return rc;
    if (!sorted) return NFC_ERR_UNSORTED;
  }
  return nf_group_sum_count(keys, values, n, sums, counts, g);
}

extern "C" int32_t nf_group_variant_i64(const int32_t* keys, const int64_t* ticks, size_t n, uint32_t variant,
                                        int64_t* sums, int64_t* counts, size_t g) {
  if (!keys || !ticks || !sums || !counts) return NFC_ERR_NULL;
  if (variant > 2) return NFC_ERR_MALFORMED;
  if (variant == 2) {
    bool sorted = true;
    const int rc = keys_sorted(keys, n, &sorted);
    if (rc) return rc;
    if (!sorted) return NFC_ERR_UNSORTED;
  }
  ScatterSpec sp{keys, n, g, true, 0, nullptr, 1, 8, ticks, 0, g, true, INT64_MIN, INT64_MAX};
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  memcpy(sums, o.is.data(), g * sizeof(int64_t));
  memcpy(counts, o.counts.data(), g * sizeof(int64_t));
  return NFC_OK;
}

extern "C" int32_t nf_group_variant_i32(const int32_t* keys, const int32_t* ticks, size_t n, uint32_t variant,
                                        int32_t* sums, int64_t* counts, size_t g) {
  if (!keys || !ticks || !sums || !counts) return NFC_ERR_NULL;
  if (variant != 0 && variant != 2) return NFC_ERR_MALFORMED;
  if (variant == 2) {
    bool sorted = true;
    const int rc = keys_sorted(keys, n, &sorted);
    if (rc) return rc;
    if (!sorted) return NFC_ERR_UNSORTED;
  }
  ScatterSpec sp{keys, n, g, true, 0, nullptr, 1, 4, ticks, 0, g, true, INT32_MIN, INT32_MAX};
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  for (size_t i = 0; i < g; ++i) sums[i] = (int32_t)o.is[i];
  memcpy(counts, o.counts.data(), g * sizeof(int64_t));
  return NFC_OK;
}

extern "C" int64_t nf_sorted_run_i64(const int32_t* keys, const int64_t* vals, size_t n, int64_t* ukeys,
                                     int64_t* sums, int64_t* counts) {
  if (n == 0) return 0;
  if (!keys || !vals || !ukeys || !sums || !counts) return NFC_ERR_RANGE;
  return sorted_run(keys, reinterpret_cast<const uint64_t*>(vals), false, n, ukeys, reinterpret_cast<uint64_t*>(sums),
                    counts);
}

extern "C" int64_t nf_sorted_run_f64(const int32_t* keys, const double* vals, size_t n, int64_t* ukeys, double* sums,
                                     int64_t* counts) {
  if (n == 0) return 0;
  if (!keys || !vals || !ukeys || !sums || !counts) return NFC_ERR_RANGE;
  return sorted_run(keys, reinterpret_cast<const uint64_t*>(vals), true, n, ukeys, reinterpret_cast<uint64_t*>(sums),
                    counts);
}

extern "C" int64_t nf_carry_build_i64(const int64_t* counts_m, const int64_t* sums_m, size_t m, int64_t* ukeys,
                                      int64_t* counts, int64_t* sums) {
  if (m == 0) return 0;
  if (!counts_m || !sums_m || !ukeys || !counts || !sums) return NFC_ERR_RANGE;
  return carry_build(counts_m, reinterpret_cast<const uint64_t*>(sums_m), m, ukeys, counts,
                     reinterpret_cast<uint64_t*>(sums));
}

extern "C" int64_t nf_carry_build_f64(const int64_t* counts_m, const double* sums_m, size_t m, int64_t* ukeys,
                                      int64_t* counts, double* sums) {
  if (m == 0) return 0;
  if (!counts_m || !sums_m || !ukeys || !counts || !sums) return NFC_ERR_RANGE;
  return carry_build(counts_m, reinterpret_cast<const uint64_t*>(sums_m), m, ukeys, counts,
                     reinterpret_cast<uint64_t*>(sums));
}

// ---------------------------------------------------------------------
// Sort / unique family.
// ---------------------------------------------------------------------
template <class T>
static int32_t sort_perm_host(int32_t dtype, const T* keys, size_t n, uint8_t descending, int32_t* perm_out) {
  cudaStream_t s = thread_stream();
  Scratch sc(s);
  Dev dv(sc);
  T* dk = nullptr;
  int rc = dv.up(keys, n, &dk);
  if (rc) return rc;
  int32_t* dp = nullptr;
  NFC_CUDA(sc.alloc(&dp, n));
  rc = nfc_sort_perm(dtype, dk, nullptr, (int64_t)n, descending != 0, dp, s);
  if (rc) return rc;
  if ((rc = down(s, perm_out, dp, n))) return rc;
  NFC_CUDA(cudaStreamSynchronize(s));
  return NFC_OK;
}

extern "C" int32_t nf_sort_perm_i32(const int32_t* keys, size_t n, uint8_t descending, int32_t* perm_out,
                                    uint32_t* tmp0, uint32_t* tmp1, int32_t* tmp_p) {
  if (n == 0) return NFC_OK;
  if (!keys || !perm_out || !tmp0 || !tmp1 || !tmp_p) return NFC_ERR_NULL;
  if (n > (size_t)INT32_MAX) return NFC_ERR_MALFORMED;
  return sort_perm_host<int32_t>(NFC_I32, keys, n, descending, perm_out);
}

extern "C" int32_t nf_sort_perm_i64(const int64_t* keys, size_t n, uint8_t descending, int32_t* perm_out,
                                    uint64_t* tmp0, uint64_t* tmp1, int32_t* tmp_p) {
  if (n == 0) return NFC_OK;
  if (!keys || !perm_out || !tmp0 || !tmp1 || !tmp_p) return NFC_ERR_NULL;
  if (n > (size_t)INT32_MAX) return NFC_ERR_MALFORMED;
  return sort_perm_host<int64_t>(NFC_I64, keys, n, descending, perm_out);
}

template <class T>
__global__ void k_unique_runs(const T* keys, const int32_t* perm, int64_t n, T* uniq, int32_t* inv, uint64_t* lb,
                              uint32_t* ticket, int64_t* ng_out, int32_t* err) {
  __shared__ uint32_t s_scan[33];
  __shared__ int64_t s_tile, s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int64_t tile = s_tile, ntiles = (n + 1023) / 1024;
  if (tile >= ntiles) return;
  const int64_t i0 = tile * 1024 + threadIdx.x * 4;
  uint32_t c = 0, heads = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t i = i0 + j;
    if (i < n && (i == 0 || keys[perm[i]] != keys[perm[i - 1]])) { heads |= 1u << j; ++c; }
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
  int64_t r = s_base + excl - 1;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t i = i0 + j;
    if (i >= n) break;
    if (heads & (1u << j)) uniq[++r] = keys[perm[i]];
    inv[perm[i]] = (int32_t)r;
  }
}

template <class T>
static int64_t unique_inverse_host(int32_t dtype, const T* keys, size_t n, T* uniq_out, int32_t* inv_out) {
  cudaStream_t s = thread_stream();
  Scratch sc(s);
  Dev dv(sc);
  T* dk = nullptr;
  int rc = dv.up(keys, n, &dk);
  if (rc) return rc;
  int32_t* dp = nullptr;
  NFC_CUDA(sc.alloc(&dp, n));
  rc = nfc_sort_perm(dtype, dk, nullptr, (int64_t)n, 0, dp, s);
  if (rc) return rc;
  T* du = nullptr;
  int32_t* di = nullptr;
  NFC_CUDA(sc.alloc(&du, n));
  NFC_CUDA(sc.alloc(&di, n));
  const int64_t ntiles = ((int64_t)n + 1023) / 1024;
  uint64_t* lb = nullptr;
  NFC_CUDA(sc.alloc(&lb, (size_t)ntiles + 3));
  NFC_CUDA(cudaMemsetAsync(lb, 0, sizeof(uint64_t) * (ntiles + 3), s));
  int64_t* dng = reinterpret_cast<int64_t*>(lb + ntiles);
  int32_t* derr = reinterpret_cast<int32_t*>(lb + ntiles + 1);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(lb + ntiles + 2);
  k_unique_runs<T><<<(unsigned)ntiles, 256, 0, s>>>(dk, dp, (int64_t)n, du, di, lb, ticket, dng, derr);
  NFC_CUDA(cudaGetLastError());
  int64_t h[2] = {0, 0};
  NFC_CUDA(cudaMemcpyAsync(h, dng, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NFC_CUDA(cudaStreamSynchronize(s));
  if ((int32_t)h[1]) return (int32_t)h[1];
  const int64_t ng = h[0];
  if ((rc = down(s, uniq_out, du, (size_t)ng)) || (rc = down(s, inv_out, di, n))) return rc;
  NFC_CUDA(cudaStreamSynchronize(s));
  return ng;
}

extern "C" int64_t nf_unique_inverse_i32(const int32_t* keys, size_t n, int32_t* uniq_out, int32_t* inv_out,
                                         int32_t* perm, uint32_t* tmp0, uint32_t* tmp1, int32_t* tmp_p) {
  if (n == 0) return 0;
  if (!keys || !uniq_out || !inv_out || !perm || !tmp0 || !tmp1 || !tmp_p) return NFC_ERR_RANGE;
  if (n > (size_t)INT32_MAX) return NFC_ERR_MALFORMED;
  return unique_inverse_host<int32_t>(NFC_I32, keys, n, uniq_out, inv_out);
}

extern "C" int64_t nf_unique_inverse_i64(const int64_t* keys, size_t n, int64_t* uniq_out, int32_t* inv_out,
                                         int32_t* perm, uint64_t* tmp0, uint64_t* tmp1, int32_t* tmp_p) {
  if (n == 0) return 0;
  if (!keys || !uniq_out || !inv_out || !perm || !tmp0 || !tmp1 || !tmp_p) return NFC_ERR_RANGE;
  if (n > (size_t)INT32_MAX) return NFC_ERR_MALFORMED;
  return unique_inverse_host<int64_t>(NFC_I64, keys, n, uniq_out, inv_out);
}

// ---------------------------------------------------------------------
// Loader-required symbols off the group-by path (native_cpu.py:125-132):
// plain host code, same contracts as transform/pack.rs and
// transform/pattern.rs.
// ---------------------------------------------------------------------
extern "C" int32_t nf_pack_i32_direct(const int32_t* k1, const int32_t* k2, int32_t m2, size_t n, int32_t* out) {
  if (!k1 || !k2 || !out) return NFC_ERR_NULL;
  for (size_t i = 0; i < n; ++i) {
    if (k1[i] < 0 || k2[i] < 0) return NFC_ERR_RANGE;
    const int64_t v = (int64_t)k1[i] * (int64_t)m2 + (int64_t)k2[i];
    if (v > INT32_MAX) return NFC_ERR_RANGE;
    out[i] = (int32_t)v;
  }
  return NFC_OK;
}

// Fused pack + aggregate (lib.rs:287 / :316, groupby/pack_fused.rs:26-90):
// the code of row i is k1[i] * m2 + k2[i] (formed on the device, never
// written back), then sum + count per code in [0, g).  -2 on a row whose
// pack fails or whose code is outside [0, g); the int32 form returns -4 when
// a group's running sum in row order leaves int32 (add_i32_checked).
extern "C" int32_t nf_pack_sum_count_i32(const int32_t* k1, const int32_t* k2, int32_t m2, const int32_t* vals,
                                         size_t n, int32_t* sums, int64_t* counts, size_t g) {
  if (!k1 || !k2 || !vals || !sums || !counts) return NFC_ERR_NULL;
  ScatterSpec sp{k1, n, g, true, 0, nullptr, 1, 4, vals, 0, g, true, INT32_MIN, INT32_MAX};
  sp.keys2 = k2;
  sp.m2 = m2;
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  for (size_t i = 0; i < g; ++i) sums[i] = (int32_t)o.is[i];
  memcpy(counts, o.counts.data(), g * sizeof(int64_t));
  return NFC_OK;
}

extern "C" int32_t nf_pack_sum_count_f64(const int32_t* k1, const int32_t* k2, int32_t m2, const double* vals,
                                         size_t n, double* sums, int64_t* counts, size_t g) {
  if (!k1 || !k2 || !vals || !sums || !counts) return NFC_ERR_NULL;
  ScatterSpec sp{k1, n, g, true, 1, vals, 0, 4, nullptr, 0, g, false, 0, 0};
  sp.keys2 = k2;
  sp.m2 = m2;
  ScatterOut o;
  const int rc = scatter_codes(sp, o);
  if (rc) return rc;
  memcpy(sums, o.fs.data(), g * sizeof(double));
  memcpy(counts, o.counts.data(), g * sizeof(int64_t));
  return NFC_OK;
}

extern "C" int32_t nf_pattern_encode(const uint8_t* data, size_t total, const int32_t* offs, size_t n,
                                     const uint8_t* prefix, size_t prefix_len, int32_t* codes, uint8_t* valid,
                                     int32_t* width_out, int32_t* err_row_out) {
  if (!data || !offs || !prefix || !codes || !valid || !width_out || !err_row_out) return NFC_ERR_NULL;
  *width_out = -1;
  *err_row_out = -1;
  int32_t prev = offs[0];
  if (prev < 0 || (size_t)prev > total) return NFC_ERR_MALFORMED;
  for (size_t i = 0; i < n; ++i) {
    codes[i] = 0;
    valid[i] = 0;
    const int32_t end = offs[i + 1];
    if (end < prev || end < 0 || (size_t)end > total) return NFC_ERR_MALFORMED;
    const uint8_t* row = data + prev;
    const size_t len = (size_t)(end - prev);
    prev = end;
    if (len < prefix_len || memcmp(row, prefix, prefix_len) != 0) continue;
    const uint8_t* body = row + prefix_len;
    size_t blen = len - prefix_len;
    const bool neg = blen > 0 && body[0] == '-';
    if (neg) { ++body; --blen; }
    if (blen == 0) continue;
    // Magnitude with saturation; a non-digit anywhere makes the row invalid.
    bool ok = true, big = false;
    int64_t mag = 0;
    for (size_t j = 0; j < blen; ++j) {
      const uint8_t ch = body[j];
      if (ch < '0' || ch > '9') { ok = false; break; }
      if (!big) {
        mag = mag * 10 + (ch - '0');
        if (mag > ((int64_t)1 << 40)) big = true;
      }
    }
    if (!ok) continue;
    const int64_t lim = neg ? ((int64_t)1 << 31) : (int64_t)INT32_MAX;
    if (big || mag > lim) {
      *err_row_out = (int32_t)i;
      return NFC_ERR_RANGE;
    }
    codes[i] = neg ? (int32_t)(-mag) : (int32_t)mag;
    valid[i] = 1;
    if ((int32_t)blen > *width_out) *width_out = (int32_t)blen;
  }
  return NFC_OK;
}

namespace nfc {
int argsort_i32_device(const int32_t* keys, int64_t n, uint32_t* perm, cudaStream_t s, Scratch& sc, int32_t* d_err) {
  (void)sc;
  (void)d_err;
  return nfc_sort_perm(NFC_I32, keys, nullptr, n, 0, reinterpret_cast<int32_t*>(perm), s);
}
}  // namespace nfc
