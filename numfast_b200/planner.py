"""Learned strategy planner: workload generator, sample collection, training, inference.

The network (280 -> 128 -> 128 -> 5, bf16 weights, fp32 accumulation) reads a device
sketch of the first 65,536 keys (nfc_sketch) and predicts log2(1 + distinct) / 32 and
which of four grouping strategies is fastest: dense index, per-CTA shared-memory hash,
global hash, or sort.  Training data come from the engine itself: for each generated
input the exact distinct count is the group-by's own group count, and the label is the
strategy with the lowest measured end-to-end group-by time (CUDA events around
nfc_groupby).  Training runs on the GPU through the library's own forward, loss,
backward and Adam kernels.  At planning time nfc_groupby_planned runs sketch + MLP on
the device; the reference's fixed rule (restated as nfc_plan_fixed) remains the fallback
for infeasible or low-confidence picks.

Key distributions of the mixed stream (`draw_specs`): uniform, Zipf(s in [0.5, 2]),
sorted runs (runs of one key, run lengths uniform in [1, 2 * mean]) and clustered
blocks (blocks of 64K rows drawing from one narrow key window each), with cardinality
log-uniform in [1, min(rows, 50M)] and the key values either a dense range at a random
base or scattered over the int32 range by a bijective mix.
"""

import ctypes
import math
import os

import numpy as np
import torch

from . import _lib
from . import device as dev

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "planner_weights.npz")
KINDS = ("uniform", "zipf", "runs", "clustered")
# Strategy classes -> nfc_groupby strategies used when timing them.
PICK_STRATEGIES = ("dense", "shared_hash", "hash", "sort")


# ------------------------------------------------------------------ workload

def draw_specs(count, seed, min_rows=100_000, max_rows=50_000_000, max_card=50_000_000):
    """Input descriptions of a mixed stream (host RNG only; keys are made on the device)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        rows = int(math.exp(rng.uniform(math.log(min_rows), math.log(max_rows))))
        card = int(max(1, math.exp(rng.uniform(0.0, math.log(min(rows, max_card))))))
        kind = KINDS[int(rng.integers(0, len(KINDS)))]
        s = float(rng.uniform(0.5, 2.0))
        if abs(s - 1.0) < 1e-3:
            s = 1.002
        specs.append({"id": i, "seed": int(seed), "rows": rows, "card": card, "kind": kind, "s": s,
                      "sparse": bool(rng.integers(0, 2)), "base": int(rng.integers(-(1 << 30), 1 << 30)),
                      "mean_run": int(rng.integers(2, 2000)), "salt": int(rng.integers(0, 1 << 31))})
    return specs


def _mix32(x, salt):
    """Bijective 32-bit scramble of int64 tensor values (returned as int32)."""
    x = (x + salt) & 0xFFFFFFFF
    x = (x ^ (x >> 16)) * 0x45D9F3B & 0xFFFFFFFF
    x = (x ^ (x >> 16)) * 0x45D9F3B & 0xFFFFFFFF
    x = x ^ (x >> 16)
    return (x - ((x >> 31) << 32)).to(torch.int32)


def make_input(spec, device="cuda"):
    """(keys, values) int32 device tensors of one stream input.  Ranks in [0, card) are
    drawn per kind on the device (Philox stream = input id), then mapped to key values."""
    n, c, q, seed = spec["rows"], spec["card"], spec["id"], spec["seed"]
    kind = spec["kind"]
    if kind == "uniform":
        r = dev.rng_fill_i32(n, seed, 2 * q, 0, c, device=device).long()
    elif kind == "zipf":
        r = dev.gen_zipf(n, seed, 2 * q, spec["s"], c, device=device).long()
    elif kind == "runs":
        mean = spec["mean_run"]
        nruns = n // mean + 2
        lens = dev.rng_fill_i32(nruns, seed, 2 * q, 1, 2 * mean, device=device).long()
        while int(lens.sum()) < n:
            lens = torch.cat([lens, lens])
        vals = dev.rng_fill_i32(lens.numel(), seed, (1 << 24) + q, 0, c, device=device).long()
        r = torch.repeat_interleave(vals, lens)[:n]
    else:  # clustered: blocks of 64K rows, each from a window of w ranks
        w = max(1, min(c, 1024))
        nwin = max(1, c // w)
        nb = (n + 65535) // 65536
        win = dev.rng_fill_i32(nb, seed, (1 << 24) + q, 0, nwin, device=device).long()
        off = dev.rng_fill_i32(n, seed, 2 * q, 0, w, device=device).long()
        r = torch.repeat_interleave(win, 65536)[:n] * w + off
    if spec["sparse"]:
        keys = _mix32(r, spec["salt"])
    else:
        keys = (r + spec["base"]).to(torch.int32)
    vals = dev.rng_fill_i32(n, seed, 2 * q + 1, -1000, 1001, device=device)
    return keys.contiguous(), vals


# ------------------------------------------------------------------ device calls

def sketch(keys, key_validity=None, out=None):
    lib = _lib.load()
    if out is None:
        out = torch.empty(_lib.MLP_IN, dtype=torch.float32, device=keys.device)
    _lib.check("nfc_sketch", lib.nfc_sketch(keys.data_ptr(), key_validity.data_ptr() if key_validity is not None
                                            else None, keys.numel(), out.data_ptr(),
                                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return out


def _groupby_args(keys, vals, buffers, vcol):
    vcol.dtype = _lib.I32
    vcol.aggs = _lib.AGG_SUM
    vcol.data = vals.data_ptr()
    vcol.validity = None
    vcol.sum_out = buffers["sum"].data_ptr()
    vcol.min_out = None
    vcol.max_out = None
    a = _lib.GroupbyArgs()
    a.n = keys.numel()
    a.keys = keys.data_ptr()
    a.key_validity = None
    a.ncols = 1
    a.cols = ctypes.pointer(vcol)
    a.out_cap = buffers["cap"]
    a.ukeys_out = buffers["ukeys"].data_ptr()
    a.counts_out = buffers["counts"].data_ptr()
    return a


def sum_count_buffers(cap, device="cuda"):
    return {"cap": cap, "ukeys": torch.empty(cap, dtype=torch.int64, device=device),
            "sum": torch.empty(cap, dtype=torch.int64, device=device),
            "counts": torch.empty(cap, dtype=torch.int64, device=device)}


def groupby_sum_count(keys, vals, mode="learned", planner=None, strategy=None, distinct_hint=0, buffers=None):
    """group(key, {v: (sum, count)}) through nfc_groupby_planned (mode auto / fixed /
    learned) or, with `strategy`, through nfc_groupby with that strategy.  Returns
    (ng, stats, buffers)."""
    lib = _lib.load()
    n = keys.numel()
    if buffers is None or buffers["cap"] < max(n, 1):
        buffers = sum_count_buffers(max(n, 1), keys.device)
    vcol = _lib.ValueCol()
    a = _groupby_args(keys, vals, buffers, vcol)
    st = _lib.GroupbyStats()
    st.distinct_hint = int(distinct_hint)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if strategy is not None:
        code = _lib.STRAT_AUTO if strategy == "dense" else dict((v, k) for k, v in
                                                                _lib.STRATEGY_NAMES.items())[strategy]
        ng = lib.nfc_groupby(ctypes.byref(a), code, stream, ctypes.byref(st))
    else:
        m = {"auto": _lib.PLANNER_AUTO, "fixed": _lib.PLANNER_FIXED, "learned": _lib.PLANNER_LEARNED}[mode]
        ng = lib.nfc_groupby_planned(ctypes.byref(a), m, planner.handle if planner is not None else None, stream,
                                     ctypes.byref(st))
    _lib.check("nfc_groupby", ng)
    return int(ng), st, buffers


class LearnedPlanner:
    """Device copy of the trained network (nfc_planner)."""

    def __init__(self, params, mu=None, sd=None, min_confidence=0.0):
        self.lib = _lib.load()
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == _lib.MLP_NPARAMS
        mu_a = None if mu is None else np.ascontiguousarray(mu, dtype=np.float32)
        sd_a = None if sd is None else np.ascontiguousarray(sd, dtype=np.float32)
        self.params, self.mu, self.sd = p, mu_a, sd_a
        h = self.lib.nfc_planner_create(p.ctypes.data, mu_a.ctypes.data if mu_a is not None else None,
                                        sd_a.ctypes.data if sd_a is not None else None, float(min_confidence))
        if not h:
            raise _lib.NativeError("nfc_planner_create", _lib.ERR_MALFORMED, _lib.last_error())
        self.handle = h

    @classmethod
    def load(cls, path=WEIGHTS, min_confidence=None):
        z = np.load(path)
        mc = float(z["min_confidence"]) if min_confidence is None else min_confidence
        return cls(z["params"], z["mu"], z["sd"], mc)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.nfc_planner_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ training data

def time_strategy(keys, vals, strategy, distinct_hint=0, reps=2, buffers=None):
    """Median device milliseconds of one group-by call with the given strategy
    (inf when the strategy cannot run on this input)."""
    if strategy == "dense":
        # The dense family applies only when the library's span rule keeps it.
        pass
    times = []
    st_used = None
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        try:
            ng, st, buffers = groupby_sum_count(keys, vals, strategy=strategy, distinct_hint=distinct_hint,
                                                buffers=buffers)
        except _lib.NativeError:
            return math.inf, buffers, None
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        st_used = st.strategy
    if strategy == "dense" and st_used == _lib.STRAT_HASH:
        return math.inf, buffers, st_used
    return float(np.median(times[1:])), buffers, st_used


def collect(specs, timed_every=1, reps=2, log=None):
    """Samples for the given input specs: features (N x 280), exact distinct counts,
    per-strategy times (N x 4, NaN where not timed) and fixed-planner times."""
    feats = np.zeros((len(specs), _lib.MLP_IN), dtype=np.float32)
    distinct = np.zeros(len(specs), dtype=np.int64)
    times = np.full((len(specs), 4), np.nan)
    fbuf = torch.empty(_lib.MLP_IN, dtype=torch.float32, device="cuda")
    buffers = None
    for i, sp in enumerate(specs):
        keys, vals = make_input(sp)
        feats[i] = sketch(keys, out=fbuf).cpu().numpy()
        ng, _, buffers = groupby_sum_count(keys, vals, mode="auto", buffers=buffers)
        distinct[i] = ng
        if timed_every and i % timed_every == 0:
            for j, s in enumerate(PICK_STRATEGIES):
                t, buffers, _ = time_strategy(keys, vals, s, distinct_hint=ng, reps=reps, buffers=buffers)
                times[i, j] = t
        if log and (i + 1) % 200 == 0:
            log("collected %d / %d" % (i + 1, len(specs)))
        del keys, vals
    return {"features": feats, "distinct": distinct, "times": times}


# ------------------------------------------------------------------ training on the GPU

def init_params(seed=0):
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((_lib.MLP_IN, _lib.MLP_H), (_lib.MLP_H, _lib.MLP_H), (_lib.MLP_H, _lib.MLP_OUT)):
        lim = math.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-lim, lim, fan_in * fan_out).astype(np.float32))
        parts.append(np.zeros(fan_out, dtype=np.float32))
    return np.concatenate(parts)


def targets(data):
    """Regression target log2(1 + distinct) / 32; class = fastest strategy (-1 when the
    sample was not timed); class weight = the sample's best time over the mean best time
    (clipped to [0.05, 20]), so the loss follows total stream time."""
    y = (np.log2(1.0 + data["distinct"].astype(np.float64)) / 32.0).astype(np.float32)
    t = data["times"]
    timed = ~np.isnan(t).any(axis=1)
    tt = np.where(np.isnan(t), np.inf, t)
    lab = np.where(timed, np.argmin(tt, axis=1), -1).astype(np.int32)
    best = np.where(timed, tt.min(axis=1), 0.0)
    mean_best = best[timed].mean() if timed.any() else 1.0
    w = np.where(timed, np.clip(best / mean_best, 0.05, 20.0), 0.0).astype(np.float32)
    return y, lab, w


def train(data, epochs=60, batch=1024, lr=2e-3, card_weight=4.0, class_weight=1.0, seed=0, log=None):
    """Adam on the library's MLP kernels.  Returns (params, mu, sd, history)."""
    lib = _lib.load()
    x_np = data["features"].astype(np.float32)
    mu = x_np.mean(axis=0).astype(np.float32)
    sd = np.maximum(x_np.std(axis=0), 1e-3).astype(np.float32)
    y_np, lab_np, w_np = targets(data)
    n = x_np.shape[0]
    d = "cuda"
    X = torch.from_numpy(x_np).to(d)
    Y = torch.from_numpy(y_np).to(d)
    L = torch.from_numpy(lab_np).to(d)
    W = torch.from_numpy(w_np).to(d)
    MU = torch.from_numpy(mu).to(d)
    SD = torch.from_numpy(sd).to(d)
    params = torch.from_numpy(init_params(seed)).to(d)
    grad = torch.zeros_like(params)
    m = torch.zeros_like(params)
    v = torch.zeros_like(params)
    w = torch.empty(_lib.MLP_NWEIGHTS, dtype=torch.int16, device=d)
    h1 = torch.empty(batch, _lib.MLP_H, device=d)
    h2 = torch.empty_like(h1)
    dh1 = torch.empty_like(h1)
    dh2 = torch.empty_like(h1)
    out = torch.empty(batch, _lib.MLP_OUT, device=d)
    dout = torch.empty_like(out)
    loss = torch.zeros(1, device=d)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check("nfc_mlp_to_bf16", lib.nfc_mlp_to_bf16(params.data_ptr(), w.data_ptr(), st))
    g = torch.Generator(device="cpu").manual_seed(seed)
    step = 0
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(d)
        loss.zero_()
        nb = 0
        for b0 in range(0, n - batch + 1 if n >= batch else 1, batch):
            idx = perm[b0:b0 + batch]
            xb, yb, lb, wb = X[idx].contiguous(), Y[idx].contiguous(), L[idx].contiguous(), W[idx].contiguous()
            B = xb.shape[0]
            _lib.check("fwd", lib.nfc_mlp_forward(xb.data_ptr(), B, MU.data_ptr(), SD.data_ptr(), w.data_ptr(),
                                                  params.data_ptr(), h1.data_ptr(), h2.data_ptr(), out.data_ptr(),
                                                  st))
            _lib.check("loss", lib.nfc_mlp_loss(out.data_ptr(), yb.data_ptr(), lb.data_ptr(), wb.data_ptr(), B,
                                                card_weight, class_weight, dout.data_ptr(), loss.data_ptr(), st))
            _lib.check("bwd", lib.nfc_mlp_backward(xb.data_ptr(), B, MU.data_ptr(), SD.data_ptr(), w.data_ptr(),
                                                   h1.data_ptr(), h2.data_ptr(), dout.data_ptr(), dh1.data_ptr(),
                                                   dh2.data_ptr(), grad.data_ptr(), st))
            step += 1
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * ep / max(epochs, 1)))
            _lib.check("adam", lib.nfc_mlp_adam(params.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(),
                                                w.data_ptr(), step, lr_t, 0.9, 0.999, 1e-8, 1e-5, st))
            nb += 1
        hist.append(float(loss.item()) / max(nb, 1))
        if log and (ep % 10 == 0 or ep == epochs - 1):
            log("epoch %d loss %.5f" % (ep, hist[-1]))
    return params.cpu().numpy(), mu, sd, hist


def predict(params, mu, sd, features):
    """Network outputs (N x 5) for host features through the CUDA forward pass."""
    lib = _lib.load()
    d = "cuda"
    X = torch.from_numpy(np.ascontiguousarray(features, dtype=np.float32)).to(d)
    B = X.shape[0]
    P = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).to(d)
    w = torch.empty(_lib.MLP_NWEIGHTS, dtype=torch.int16, device=d)
    h1 = torch.empty(B, _lib.MLP_H, device=d)
    h2 = torch.empty_like(h1)
    out = torch.empty(B, _lib.MLP_OUT, device=d)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    MU = torch.from_numpy(mu).to(d)
    SD = torch.from_numpy(sd).to(d)
    _lib.check("to_bf16", lib.nfc_mlp_to_bf16(P.data_ptr(), w.data_ptr(), st))
    _lib.check("fwd", lib.nfc_mlp_forward(X.data_ptr(), B, MU.data_ptr(), SD.data_ptr(), w.data_ptr(), P.data_ptr(),
                                          h1.data_ptr(), h2.data_ptr(), out.data_ptr(), st))
    return out.cpu().numpy()


def save(path, params, mu, sd, min_confidence=0.0, meta=None):
    np.savez_compressed(path, params=params.astype(np.float32), mu=mu.astype(np.float32), sd=sd.astype(np.float32),
                        min_confidence=np.float32(min_confidence), meta=np.array(repr(meta or {})))
