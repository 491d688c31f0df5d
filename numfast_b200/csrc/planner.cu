// Strategy planners around the group-by body: the reference's fixed rule,
// restated, and the learned planner (device sketch + MLP) that it judges.
#include <math.h>

#include <mutex>
#include <new>

#include "groupby_host.h"
#include "mlp_core.cuh"

namespace nfc {

// plan_groupby_impl (src/Runtime/Planner/_lib/planner.py:200-262) with the
// executor's byte estimates (groupindex.py:72-83: shift-dense 16R + 8N,
// by-code 16M + 8N for int32 keys) and the CPU buffer budget 2^31 - 1
// (Planner.py:54-65 fills it from max_buffer_bytes).  Python-int arithmetic
// there; int64 here (every term is far below 2^63 for n < 2^31).
int plan_fixed(const nfc_probe& p, int naggs, const ColSet* cs) {
  if (p.n_valid == 0) return NFC_STRAT_DENSE_GLOBAL;  // "empty": nothing to group
  if (p.sorted) return NFC_STRAT_SORTED;
  const int64_t n = p.n_valid;
  const int64_t r = p.kmax - p.kmin + 1;
  const int64_t r_max = 64000000, budget = (1ll << 31) - 1;
  const int64_t cap = std::min<int64_t>(r_max, 4 * n);
  naggs = std::max(1, naggs);
  const int64_t est = 16 * r + 8 * n;
  const int64_t per_col = 8 * std::min(r, n) + 8 * n;
  const int64_t total_shift = est + naggs * per_col;
  bool dense = false;
  if (p.kmin >= 0) {
    const int64_t m_code = p.kmin + r;
    const int64_t total_code = 16 * m_code + 8 * n + naggs * 8 * std::min(m_code, n);
    if (m_code <= cap && total_code <= budget && total_code <= total_shift) dense = true;  // dense_by_code
  }
  if (!dense && r <= cap && total_shift <= budget) dense = true;  // shift-based dense
  if (!dense) return NFC_STRAT_SORT;  // "hash" -> hash_dynamic_index == sorted unique
  if (cs) {
    const int s = plan_strategy(*cs, p);
    return s == NFC_STRAT_HASH ? NFC_STRAT_SORT : s;
  }
  return NFC_STRAT_DENSE_GLOBAL;
}

static int naggs_of(const ColSet& cs) {
  int k = 0;
  for (int c = 0; c < cs.ncols; ++c) k += __builtin_popcount((unsigned)cs.aggs[c]);
  return std::max(1, k);
}

}  // namespace nfc

using namespace nfc;

struct nfc_planner {
  int device = 0;
  float* d_params = nullptr;
  uint16_t* d_w = nullptr;
  float* d_block = nullptr;  // mu | sd | feat
  float* d_mu = nullptr;
  float* d_sd = nullptr;
  float* d_feat = nullptr;
  float* h_out = nullptr;  // mapped pinned memory, NFC_MLP_OUT floats
  float* d_hout = nullptr;  // its device address (the network writes there)
  void* d_sketch = nullptr;  // sketch scratch
  float min_conf = 0.f;
  // Sketch + inference run on their own stream, forked from the caller's
  // stream, so that they overlap the probe instead of preceding it.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::mutex mu;
};

namespace {

struct FixedHook final : PlanHook {
  nfc_groupby_stats* stats;
  explicit FixedHook(nfc_groupby_stats* st) : stats(st) {}
  int choose(const ColSet& cs, const nfc_probe& p, int* strategy, int64_t*) override {
    *strategy = plan_fixed(p, naggs_of(cs), &cs);
    if (stats) {
      stats->planner_used = NFC_PLANNER_FIXED;
      stats->fixed_pick = *strategy;
      stats->learned_pick = -1;
    }
    return NFC_OK;
  }
};

struct LearnedHook final : PlanHook {
  nfc_planner* pl;
  nfc_groupby_stats* stats;
  LearnedHook(nfc_planner* p, nfc_groupby_stats* st) : pl(p), stats(st) {}
  int choose(const ColSet& cs, const nfc_probe& p, int* strategy, int64_t* hint) override {
    // The sketch and the MLP ran on the planner's side stream next to the
    // probe; their output is in mapped host memory once ev_join completes.
    NFC_CUDA(cudaEventSynchronize(pl->ev_join));
    float o[NFC_MLP_OUT];
    for (int k = 0; k < NFC_MLP_OUT; ++k) o[k] = static_cast<volatile float*>(pl->h_out)[k];
    int pick = 0;
    float mx = o[1];
    for (int k = 1; k < NFC_MLP_OUT - 1; ++k)
      if (o[1 + k] > mx) {
        mx = o[1 + k];
        pick = k;
      }
    float se = 0.f;
    for (int k = 0; k < NFC_MLP_OUT - 1; ++k) se += expf(o[1 + k] - mx);
    const float conf = 1.f / se;
    const double pred = exp2(fmin(fmax((double)o[0], 0.0), 1.0) * 32.0) - 1.0;
    const int fixed = plan_fixed(p, naggs_of(cs), &cs);
    int strat = fixed;
    bool learned = conf >= pl->min_conf;
    if (learned) {
      switch (pick) {
        case NFC_PICK_DENSE: {
          const int d = plan_strategy(cs, p);
          if (d == NFC_STRAT_HASH) learned = false;  // span too wide for the dense family
          else strat = d;
          break;
        }
        case NFC_PICK_SHARED_HASH:
          strat = NFC_STRAT_SHARED_HASH;
          *hint = (int64_t)fmin(fmax(pred * 2.0, 4096.0), 4.0e9);
          break;
        case NFC_PICK_GLOBAL_HASH: strat = NFC_STRAT_HASH; break;
        default: strat = NFC_STRAT_SORT; break;
      }
    }
    if (!learned) strat = fixed;
    *strategy = strat;
    if (stats) {
      stats->planner_used = learned ? NFC_PLANNER_LEARNED : NFC_PLANNER_FIXED;
      stats->predicted_distinct = (int64_t)pred;
      stats->learned_pick = pick;
      stats->fixed_pick = fixed;
    }
    return NFC_OK;
  }
};

void planner_free(nfc_planner* p) {
  if (!p) return;
  cudaFree(p->d_params);
  cudaFree(p->d_w);
  cudaFree(p->d_block);
  cudaFree(p->d_sketch);
  if (p->h_out) cudaFreeHost(p->h_out);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  if (p->side) cudaStreamDestroy(p->side);
  delete p;
}

}  // namespace

extern "C" int32_t nfc_plan_fixed(const nfc_probe* probe, int32_t naggs) {
  if (!probe) return NFC_ERR_NULL;
  return plan_fixed(*probe, naggs, nullptr);
}

extern "C" nfc_planner* nfc_planner_create(const float* params, const float* feat_mu, const float* feat_sd,
                                           float min_confidence) {
  if (!params || ((feat_mu == nullptr) != (feat_sd == nullptr))) {
    set_last_error("nfc_planner_create: params required; feat_mu and feat_sd both or neither");
    return nullptr;
  }
  nfc_planner* p = new (std::nothrow) nfc_planner();
  if (!p) return nullptr;
  cudaGetDevice(&p->device);
  p->min_conf = min_confidence;
  cudaError_t e = cudaMalloc(&p->d_params, sizeof(float) * NFC_MLP_NPARAMS);
  if (e == cudaSuccess) e = cudaMalloc(&p->d_w, sizeof(uint16_t) * NFC_MLP_NWEIGHTS);
  // mu | sd | feat in one allocation.
  const size_t nf = 3 * NFC_MLP_IN;
  if (e == cudaSuccess) e = cudaMalloc(&p->d_block, sizeof(float) * nf);
  if (e == cudaSuccess) e = cudaHostAlloc(&p->h_out, sizeof(float) * 8, cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer(&p->d_hout, p->h_out, 0);
  if (e == cudaSuccess) e = cudaMalloc(&p->d_sketch, sketch_scratch_bytes());
  // The fused sketch expects zeroed scratch and leaves it zeroed.
  if (e == cudaSuccess) e = cudaMemset(p->d_sketch, 0, sketch_scratch_bytes());
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) {
    p->d_mu = p->d_block;
    p->d_sd = p->d_mu + NFC_MLP_IN;
    p->d_feat = p->d_sd + NFC_MLP_IN;
    e = cudaMemcpy(p->d_params, params, sizeof(float) * NFC_MLP_NPARAMS, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && feat_mu) e = cudaMemcpy(p->d_mu, feat_mu, sizeof(float) * NFC_MLP_IN, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && feat_sd) e = cudaMemcpy(p->d_sd, feat_sd, sizeof(float) * NFC_MLP_IN, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !feat_mu) p->d_mu = nullptr;  // no standardisation
  if (e == cudaSuccess && nfc_mlp_to_bf16(p->d_params, p->d_w, nullptr) != NFC_OK) e = cudaErrorUnknown;
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cuda_fail(e, "nfc_planner_create");
    planner_free(p);
    return nullptr;
  }
  return p;
}

extern "C" void nfc_planner_destroy(nfc_planner* p) { planner_free(p); }

extern "C" int64_t nfc_groupby_planned(const nfc_groupby_args* a, int32_t mode, nfc_planner* planner, void* stream,
                                       nfc_groupby_stats* stats) {
  if (!a) return NFC_ERR_NULL;
  if (stats) {
    stats->planner_used = mode == NFC_PLANNER_AUTO ? NFC_PLANNER_AUTO : NFC_PLANNER_FIXED;
    stats->predicted_distinct = 0;
    stats->learned_pick = -1;
    stats->fixed_pick = -1;
  }
  if (mode == NFC_PLANNER_AUTO) return groupby_run(a, NFC_STRAT_AUTO, nullptr, stream, stats);
  if (mode == NFC_PLANNER_FIXED) {
    FixedHook h(stats);
    return groupby_run(a, NFC_STRAT_AUTO, &h, stream, stats);
  }
  if (mode != NFC_PLANNER_LEARNED) return NFC_ERR_MALFORMED;
  if (!planner) return NFC_ERR_NULL;
  if (a->n < 0 || a->n > INT32_MAX) return NFC_ERR_MALFORMED;
  std::lock_guard<std::mutex> lock(planner->mu);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Fork: the side stream starts after the caller's prior work (the keys are
  // ready) and its kernels go in before the probe's, so they share the SMs.
  // Two launches: the sketch's last CTA runs the network and writes the
  // outputs straight into mapped host memory.
  cudaStream_t ps = planner->side;
  NFC_CUDA(cudaEventRecord(planner->ev_fork, s));
  NFC_CUDA(cudaStreamWaitEvent(ps, planner->ev_fork, 0));
  const MlpRef mref{planner->d_mu, planner->d_mu ? planner->d_sd : nullptr,
                    reinterpret_cast<const __nv_bfloat16*>(planner->d_w), planner->d_params, planner->d_hout};
  const int rc = sketch_launch(a->keys, a->key_validity, a->n, planner->d_feat, planner->d_sketch, ps, &mref);
  const cudaError_t ej = cudaEventRecord(planner->ev_join, ps);
  int64_t ng = rc;
  if (rc == NFC_OK && ej != cudaSuccess) ng = cuda_fail(ej, "cudaEventRecord(planner join)");
  if (ng == NFC_OK) {
    LearnedHook h(planner, stats);
    ng = groupby_run(a, NFC_STRAT_AUTO, &h, stream, stats);
  }
  // Join after the group-by (also on failure): later work on the caller's
  // stream, and whatever frees the keys after this call, come after the side
  // stream's reads.
  if (ej == cudaSuccess) cudaStreamWaitEvent(s, planner->ev_join, 0);
  return ng;
}
