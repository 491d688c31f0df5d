"""Batched group-by: many independent sum+count group-bys in one persistent launch.

Each query is ``group(key, {v: ("sum", "count")})`` over its own row range of one
concatenated int32 key column and one int32 value column -- per query the same result
as the executor's ``groupby_multi`` node (src/Drivers/CPU/_lib/cpu.py:3435-3704): NULL
key or value rows dropped, groups in ascending key order, int64 counts and sums.

``BatchGroupby`` owns the device-side plan (work items, state arena) for one row layout
and runs it through ``nfc_batch_run`` (optionally as a replayed CUDA graph).
``autotune`` picks the tile sizes and the item schedule by timing candidate tunings on
the caller's own batch.  ``config4_layout`` / ``make_config4`` generate the synthetic
batched workload: 4,096 queries, rows log-uniform in [1K, 4M], cardinality log-uniform
in [1, rows], keys uniform or Zipf(s in [0.5, 2]), values uniform in [-1000, 1000].
"""

import ctypes
import json
import math
import os
import statistics

import numpy as np
import torch

from . import _lib

VALUE_STREAM_BASE = 1 << 20


def default_tuning():
    t = _lib.BatchTuning()
    _lib.load().nfc_batch_default_tuning(ctypes.byref(t))
    return t


def tuning_from_dict(d):
    t = default_tuning()
    for k, v in d.items():
        setattr(t, k, int(v))
    return t


class BatchResult:
    """Outputs of one batched run (device tensors) plus the number of deferred queries."""

    def __init__(self, ukeys, sums, counts, group_offsets, ngroups, deferred):
        self.ukeys = ukeys
        self.sums = sums
        self.counts = counts
        self.group_offsets = group_offsets
        self.ngroups = ngroups
        self.deferred = deferred

    def query(self, q):
        """(ukeys, sums, counts) of query q as host numpy arrays."""
        off = int(self.group_offsets[q])
        ng = int(self.ngroups[q])
        sl = slice(off, off + ng)
        return (self.ukeys[sl].cpu().numpy(), self.sums[sl].cpu().numpy(), self.counts[sl].cpu().numpy())


class BatchGroupby:
    """Plan of a batched group-by for a fixed row layout (row_offsets, host int64[nq+1])."""

    def __init__(self, row_offsets, tuning=None):
        self.lib = _lib.load()
        ro = np.ascontiguousarray(np.asarray(row_offsets, dtype=np.int64))
        if ro.ndim != 1 or ro.size < 2:
            raise ValueError("row_offsets must be int64[nq + 1]")
        self.row_offsets = ro
        self.nq = ro.size - 1
        self.total_rows = int(ro[-1])
        self.tuning = tuning if tuning is not None else default_tuning()
        h = self.lib.nfc_batch_create(self.nq, ro.ctypes.data, ctypes.byref(self.tuning))
        if not h:
            raise _lib.NativeError("nfc_batch_create", _lib.ERR_MALFORMED, _lib.last_error())
        self.handle = h
        self._out = None

    def close(self):
        if getattr(self, "handle", None):
            self.lib.nfc_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        out = (ctypes.c_int64 * 8)()
        _lib.check("nfc_batch_info", self.lib.nfc_batch_info(self.handle, out, 8))
        names = ["nq", "rows", "items", "probe_items", "solo_items", "agg_items", "emit_items", "arena_bytes"]
        return dict(zip(names, [int(x) for x in out]))

    def outputs(self, out_cap=None, device="cuda"):
        cap = self.total_rows if out_cap is None else int(out_cap)
        o = self._out
        if o is None or o["cap"] != cap or o["ukeys"].device != torch.device(device):
            o = {"cap": cap,
                 "ukeys": torch.empty(max(cap, 1), dtype=torch.int64, device=device),
                 "sums": torch.empty(max(cap, 1), dtype=torch.int64, device=device),
                 "counts": torch.empty(max(cap, 1), dtype=torch.int64, device=device),
                 "group_offsets": torch.empty(self.nq, dtype=torch.int64, device=device),
                 "ngroups": torch.empty(self.nq, dtype=torch.int64, device=device)}
            self._out = o
        return o

    def run(self, keys, values, key_validity=None, value_validity=None, out_cap=None, graph=True,
            sync=True, stream=None):
        """Run the batch; returns a BatchResult (deferred = None when sync is False)."""
        if keys.dtype != torch.int32 or values.dtype != torch.int32:
            raise TypeError("keys and values must be int32")
        if keys.numel() != self.total_rows or values.numel() != self.total_rows:
            raise ValueError("keys/values must hold row_offsets[-1] = %d rows" % self.total_rows)
        o = self.outputs(out_cap, keys.device)
        flags = (_lib.BATCH_GRAPH if graph else 0) | (0 if sync else _lib.BATCH_NO_SYNC)
        st = stream if stream is not None else torch.cuda.current_stream(keys.device)
        rc = self.lib.nfc_batch_run(
            self.handle, keys.data_ptr(), key_validity.data_ptr() if key_validity is not None else None,
            values.data_ptr(), value_validity.data_ptr() if value_validity is not None else None,
            o["cap"], o["ukeys"].data_ptr(), o["sums"].data_ptr(), o["counts"].data_ptr(),
            o["group_offsets"].data_ptr(), o["ngroups"].data_ptr(), flags, ctypes.c_void_p(st.cuda_stream))
        _lib.check("nfc_batch_run", rc)
        return BatchResult(o["ukeys"], o["sums"], o["counts"], o["group_offsets"], o["ngroups"],
                           int(rc) if sync else None)

    def finish(self, stream=None):
        st = stream if stream is not None else torch.cuda.current_stream()
        return int(_lib.check("nfc_batch_finish", self.lib.nfc_batch_finish(self.handle,
                                                                            ctypes.c_void_p(st.cuda_stream))))

    def profile(self, stream=None):
        """Per item type of the last run: SM cycles summed over CTAs and item counts."""
        st = stream if stream is not None else torch.cuda.current_stream()
        out = (ctypes.c_int64 * 12)()
        _lib.check("nfc_batch_profile", self.lib.nfc_batch_profile(self.handle, out, ctypes.c_void_p(st.cuda_stream)))
        names = ("probe", "solo", "agg", "emit", "agg_smem_plan", "agg_global_plan")
        return {n: {"cycles": int(out[i]), "items": int(out[6 + i])} for i, n in enumerate(names)}

    def plans(self, stream=None):
        """Plan name of every query in the last run."""
        st = stream if stream is not None else torch.cuda.current_stream()
        buf = np.zeros(self.nq, dtype=np.int32)
        _lib.check("nfc_batch_query_plans", self.lib.nfc_batch_query_plans(self.handle, buf.ctypes.data,
                                                                           ctypes.c_void_p(st.cuda_stream)))
        return [_lib.BATCH_PLAN_NAMES.get(int(p), "?") for p in buf]


# ------------------------------------------------------------------ autotuner

# Knobs in the order the coordinate search visits them.  A knob can set several
# tuning fields at once (shared-memory slots and CTAs per SM go together).
SEARCH_SPACE = [
    ("chunk_rows", [{"chunk_rows": v} for v in (32768, 65536, 131072, 262144)]),
    ("agg_split", [{"agg_split": v} for v in (0, 32, 64, 128, 256)]),
    ("solo_rows", [{"solo_rows": v} for v in (8192, 16384, 32768, 65536, 131072)]),
    ("smem", [{"smem_slots": 16384, "ctas_per_sm": 1}, {"smem_slots": 24576, "ctas_per_sm": 1},
              {"smem_slots": 12288, "ctas_per_sm": 2}, {"smem_slots": 8192, "ctas_per_sm": 2}]),
    ("smem_span_div", [{"smem_span_div": v} for v in (1, 2, 4, 8)]),
    ("warp_agg", [{"warp_agg": 0}, {"warp_agg": 1}, {"warp_agg": 2}, {"warp_agg": 3}]),
    ("schedule", [{"schedule": v} for v in (0, 1, 2)]),
    ("probe_rows", [{"probe_rows": v} for v in (131072, 262144, 524288, 1048576)]),
    ("emit", [{"emit_slice": 65536, "emit_max_items": 8}, {"emit_slice": 32768, "emit_max_items": 16},
              {"emit_slice": 131072, "emit_max_items": 4}]),
]


def layout_signature(row_offsets):
    """Key of a row layout for the tuning cache: query count and log2 row-count histogram."""
    rows = np.diff(np.asarray(row_offsets, dtype=np.int64))
    hist = np.bincount(np.log2(np.maximum(rows, 1)).astype(np.int64), minlength=32)
    return "nq%d-rows%d-h%s" % (rows.size, int(rows.sum()), ".".join(str(int(x)) for x in hist))


def time_tuning(row_offsets, tuning, keys, values, key_validity=None, value_validity=None, reps=3,
                out_cap=None):
    """Device milliseconds of one graph replay (median of reps) plus host time spent on
    deferred queries, for one candidate tuning."""
    import time
    b = BatchGroupby(row_offsets, tuning)
    try:
        cap = out_cap
        r = b.run(keys, values, key_validity, value_validity, out_cap=cap, graph=True, sync=True)
        extra = 0.0
        if r.deferred:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.run(keys, values, key_validity, value_validity, out_cap=cap, graph=True, sync=True)
            extra = (time.perf_counter() - t0) * 1e3
        st = torch.cuda.current_stream()
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            b.run(keys, values, key_validity, value_validity, out_cap=cap, graph=True, sync=False)
            e1.record(st)
            e1.synchronize()
            b.finish()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times) + extra, r.deferred
    finally:
        b.close()


def autotune(row_offsets, keys, values, key_validity=None, value_validity=None, reps=3, passes=1,
             out_cap=None, cache_path=None, log=None):
    """Coordinate search over SEARCH_SPACE starting from the library defaults.

    Returns (tuning, report).  With cache_path, results are stored per (device, layout
    signature) in a JSON file and reused on the next call."""
    dev_name = torch.cuda.get_device_name(keys.device)
    key = dev_name + "|" + layout_signature(row_offsets)
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            return tuning_from_dict(cache[key]["tuning"]), dict(cache[key], cached=True)
    best = default_tuning().as_dict()
    best_ms, _ = time_tuning(row_offsets, tuning_from_dict(best), keys, values, key_validity, value_validity, reps,
                             out_cap)
    trials = [{"tuning": dict(best), "ms": best_ms}]
    for _ in range(passes):
        for name, options in SEARCH_SPACE:
            for opt in options:
                cand = dict(best, **opt)
                if cand == best:
                    continue
                ms, deferred = time_tuning(row_offsets, tuning_from_dict(cand), keys, values, key_validity,
                                           value_validity, reps, out_cap)
                trials.append({"tuning": cand, "ms": ms, "deferred": deferred})
                if log:
                    log("autotune %s=%s: %.3f ms (best %.3f)" % (name, opt, ms, best_ms))
                if ms < best_ms:
                    best, best_ms = cand, ms
    report = {"tuning": best, "ms": best_ms, "trials": len(trials),
              "default_ms": trials[0]["ms"], "cached": False}
    if cache_path:
        cache = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        cache[key] = {"tuning": best, "ms": best_ms, "default_ms": trials[0]["ms"], "trials": len(trials)}
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return tuning_from_dict(best), report


# ------------------------------------------------------------------ synthetic workload

def config4_layout(nq=4096, seed=42, min_rows=1000, max_rows=4_000_000):
    """Per-query sizes and key distributions of the batched workload (host RNG, seeded).

    rows log-uniform in [min_rows, max_rows]; cardinality log-uniform in [1, rows];
    half the queries uniform keys over the cardinality, half Zipf(s) ranks with s
    uniform in [0.5, 2]; each query's keys are shifted by a random base."""
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(math.log(min_rows), math.log(max_rows), nq)).astype(np.int64)
    card = np.maximum(1, np.exp(rng.uniform(0.0, np.log(rows.astype(np.float64)))).astype(np.int64))
    card = np.minimum(card, rows)
    zipf = rng.integers(0, 2, nq).astype(bool)
    s = rng.uniform(0.5, 2.0, nq)
    s[np.abs(s - 1.0) < 1e-3] = 1.002  # the continuous inverse CDF needs s != 1
    base = rng.integers(-(1 << 30), 1 << 30, nq).astype(np.int64)
    row_offsets = np.zeros(nq + 1, dtype=np.int64)
    row_offsets[1:] = np.cumsum(rows)
    return {"rows": rows, "card": card, "zipf": zipf, "s": s, "base": base, "row_offsets": row_offsets,
            "seed": seed}


def make_config4(layout, device="cuda"):
    """Device keys/values of a layout: query q draws its keys from Philox stream q and its
    values from stream 2^20 + q (seed = layout seed)."""
    lib = _lib.load()
    ro = layout["row_offsets"]
    n = int(ro[-1])
    keys = torch.empty(n, dtype=torch.int32, device=device)
    vals = torch.empty(n, dtype=torch.int32, device=device)
    st = ctypes.c_void_p(torch.cuda.current_stream(keys.device).cuda_stream)
    seed = int(layout["seed"])
    for q in range(ro.size - 1):
        a, r = int(ro[q]), int(ro[q + 1] - ro[q])
        if r == 0:
            continue
        kp = keys.data_ptr() + 4 * a
        c, b = int(layout["card"][q]), int(layout["base"][q])
        if layout["zipf"][q]:
            _lib.check("nfc_gen_zipf", lib.nfc_gen_zipf(r, seed, q, float(layout["s"][q]), c, kp, st))
            keys[a:a + r] += b
        else:
            _lib.check("nfc_rng_fill_i32", lib.nfc_rng_fill_i32(r, seed, q, 0, b, b + c, kp, st))
        _lib.check("nfc_rng_fill_i32", lib.nfc_rng_fill_i32(r, seed, VALUE_STREAM_BASE + q, 0, -1000, 1001,
                                                            vals.data_ptr() + 4 * a, st))
    return keys, vals
