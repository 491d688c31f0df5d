#!/usr/bin/env python
"""Group-by throughput on B200: 100M int32 rows, 10M-key domain, 5% NULLs per column.

Workload (one step): group-by of 100,000,000 rows; key int32 uniform over [0, 10M);
v int32 uniform in [-1000, 1000]; f float64 lognormal(3, 1); an LSB validity bitmap per
column with 5% NULLs; aggregates count + sum/min/max of v and f.  Inputs are synthetic
(Philox lanes seeded like the reference RNG), generated on the device, 1.64 GB resident
in HBM -- larger than L2, so no flush is needed between steps.

  value : Mrows/s over all ranks, inputs resident in HBM, device time (CUDA events)
  e2e   : same metric through the public API with HOST (pinned) inputs: H2D of keys,
          values and bitmaps + group-by + D2H of the grouped result, every step
  roofline : algorithmic bytes (16.375 B/row in + 56 B/group out) / device time of one
          group-by call, against the measured HBM copy bandwidth
  cpu_baseline : the reference's CPU algorithm (NumPy restatement) on a bounded sample
  workloads : (default run, one GPU) the other configurations measured in the same run --
          sorted keys, radix unique over 200M keys (full range; runs), the batched
          persistent launch, and the learned-vs-fixed planner stream of 20,000 inputs

--impl reference runs that CPU algorithm instead (rank 0 only under torchrun), on the
same full workload and config as the CUDA arm, over every host core.
Multi-GPU: replicas only (each rank groups its own 100M rows; no collective on the
data path); value = total rows / max-over-ranks time.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ROWS = 100_000_000
SPAN = 10_000_000
P_NULL = 0.05
SEED = 42
METRIC = "group-by Mrows/s & % HBM peak @100M rows; learned vs fixed planner speedup"
CONFIG = {"workload": "groupby_100M_rows_10M_keys_5pct_nulls_sum_count_min_max_i32_f64",
          "rows": N_ROWS, "key_domain": SPAN, "null_fraction_per_column": P_NULL,
          "columns": "key int32, v int32 U[-1000,1000], f float64 lognormal(3,1)",
          "aggregates": "count, v.sum/min/max, f.sum/min/max",
          "l2": "inputs 1.64 GB > L2 (126 MB): no flush needed",
          "parallelism": "replicas"}
COMPOSITE_METRIC = "composite-key group-by Mrows/s @100M rows (2 int32 key columns, ~10M tuples)"
DISTINCT_METRIC = "grouped count-distinct Mrows/s @100M rows (1M keys x 100K values, 5% NULL keys)"
FILTER_METRIC = "fused filter -> group-by Mrows/s (input rows) @100M rows, 50% kept"
PLANNER_METRIC = "learned vs fixed planner speedup (end-to-end group-by time over a mixed stream)"
PLANNER_SEED = 2024  # held out: training uses 1234, the tests 777
SORTED_METRIC = "sorted-key group-by Mrows/s @100M rows (10M-key domain, 5% NULLs, count + sum/min/max)"
TOPK_METRIC = "top-k (k=1,000) Mkeys/s of a stable descending argsort @100M float64 keys (5% NULLs)"
TOPK_K = 1000
BATCH_METRIC = "batched group-by Mrows/s (4,096 sum+count queries, one persistent graph-replayed launch)"
BATCH_CONFIG = {"workload": "batch_4096_queries_rows_1K_4M_loguniform_sum_count_i32",
                "queries": 4096, "rows_per_query": "log-uniform [1K, 4M]",
                "cardinality": "log-uniform [1, rows]", "keys": "uniform or Zipf(s in [0.5, 2]), random base",
                "values": "int32 U[-1000, 1000]", "aggregates": "sum, count",
                "l2": "inputs ~15 GB > L2 (126 MB): no flush needed", "parallelism": "replicas"}
# DRAM bytes (read + write) of one headline group-by call: dram__bytes_read.sum +
# dram__bytes_write.sum of each kernel, captured one kernel at a time on a 40M-row case of the
# same key domain and scaled to 100M rows (reads and record writes by rows, the aggregate's
# output writes by groups); keyed by (rows, key domain).
MEASURED_DRAM_BYTES = {(100_000_000, 10_000_000): 8197100000.0}
ALG_IN_BYTES_PER_ROW = 4 + 4 + 8 + 3 / 8.0      # key + v + f + three validity bits
ALG_OUT_BYTES_PER_GROUP = 8 + 8 + 8 + 4 + 4 + 8 + 8 + 8  # key, count, v.sum/min/max, f.sum/min/max


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rows", type=int, default=N_ROWS)
    ap.add_argument("--span", type=int, default=SPAN)
    ap.add_argument("--workload", default="groupby",
                    choices=["groupby", "unique_full", "unique_runs", "batch", "planner", "filter",
                             "count_distinct", "composite", "sorted", "topk"])
    ap.add_argument("--inputs", type=int, default=20000, help="planner workload: inputs of the mixed stream")
    ap.add_argument("--batch-queries", type=int, default=4096, help="batch workload: queries (smaller = profiling case)")
    ap.add_argument("--no-autotune", action="store_true", help="batch workload: library default tuning")
    ap.add_argument("--tune-cache", default=None, help="batch workload: JSON cache of autotuned tunings")
    ap.add_argument("--no-workloads", action="store_true",
                    help="groupby workload: skip the other configurations measured in the same run")
    ap.add_argument("--ref-procs", type=int, default=0, help="reference arm: worker processes (default: host cores)")
    ap.add_argument("--dump", default=None, help="planner workload: write one JSON line per input to this path")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU side

def cpu_sample(rows, seed=SEED):
    from oracle import nf_oracle as O
    import numpy as np
    k = O.fill_i32(rows, seed, 0, 0, 0, SPAN)
    v = O.fill_i32(rows, seed, 1, 0, -1000, 1001)
    u1 = 1.0 - O.fill_f64(rows, seed, 2)
    u2 = O.fill_f64(rows, seed, 3)
    f = np.exp(3.0 + np.sqrt(-2.0 * np.log(u1)) * np.cos(2 * np.pi * u2))
    val = {"__key__": O.fill_f64(rows, seed, 4) >= P_NULL, "v": O.fill_f64(rows, seed, 5) >= P_NULL,
           "f": O.fill_f64(rows, seed, 6) >= P_NULL}
    return k, {"v": v, "f": f}, val


def cpu_groupby_rate(rows, reps):
    """Mrows/s of the reference's CPU algorithm (oracle port), median of reps."""
    from oracle import nf_oracle as O
    k, cols, val = cpu_sample(rows)
    ops = {"v": ("sum", "count", "min", "max"), "f": ("sum", "min", "max")}
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        O.groupby_multi(k, cols, ops, val)
        times.append(time.perf_counter() - t0)
    return rows / statistics.median(times) / 1e6, times


# ------------------------------------------------------------------ reference arm, all host cores
# The reference's NumPy executor runs on one thread; the reference arm spreads the same
# algorithm over every host core by key range: worker w groups the rows whose key lies in
# its range (one mask pass over the keys, then the oracle's groupby_multi on the kept rows),
# so the per-range results are the single-threaded result cut at key boundaries.  The
# inputs are the full workload (the same rows, distributions and seeds as the CUDA arm),
# filled in shared memory by the same workers in row slices before the timed steps.

_REF = {}


def _ref_attach(names, rows):
    import numpy as np
    from multiprocessing import shared_memory
    shm = [shared_memory.SharedMemory(name=nm) for nm in names]
    dts = [np.int32, np.int32, np.float64, np.bool_, np.bool_, np.bool_]
    arrs = [np.ndarray((rows,), dtype=dt, buffer=m.buf) for dt, m in zip(dts, shm)]
    _REF.update(shm=shm, k=arrs[0], v=arrs[1], f=arrs[2], kv=arrs[3], vv=arrs[4], fv=arrs[5], rows=rows)


def _ref_fill(lo, hi):
    """Rows [lo, hi) of the workload: the oracle's Philox lanes at offset lo."""
    import numpy as np
    from oracle import nf_oracle as O
    n = hi - lo
    _REF["k"][lo:hi] = O.fill_i32(n, SEED, 0, lo, 0, SPAN)
    _REF["v"][lo:hi] = O.fill_i32(n, SEED, 1, lo, -1000, 1001)
    u1 = 1.0 - O.fill_f64(n, SEED, 2, lo)
    u2 = O.fill_f64(n, SEED, 3, lo)
    _REF["f"][lo:hi] = np.exp(3.0 + np.sqrt(-2.0 * np.log(u1)) * np.cos(2 * np.pi * u2))
    _REF["kv"][lo:hi] = O.fill_f64(n, SEED, 4, lo) >= P_NULL
    _REF["vv"][lo:hi] = O.fill_f64(n, SEED, 5, lo) >= P_NULL
    _REF["fv"][lo:hi] = O.fill_f64(n, SEED, 6, lo) >= P_NULL
    return n


def _ref_range(lo, hi):
    from oracle import nf_oracle as O
    k = _REF["k"]
    m = (k >= lo) & (k < hi)
    ops = {"v": ("sum", "count", "min", "max"), "f": ("sum", "min", "max")}
    r = O.groupby_multi(k[m], {"v": _REF["v"][m], "f": _REF["f"][m]}, ops,
                        {"__key__": _REF["kv"][m], "v": _REF["vv"][m], "f": _REF["fv"][m]})
    return int(r["ukeys"].size)


class RefPool:
    """Process pool (spawn) over the workload in shared memory, one key range per worker."""

    def __init__(self, rows, workers):
        import multiprocessing as mp
        import numpy as np
        from multiprocessing import shared_memory
        self.shm = [shared_memory.SharedMemory(create=True, size=max(1, rows * sz)) for sz in (4, 4, 8, 1, 1, 1)]
        self.rows = rows
        self.workers = workers
        self.pool = mp.get_context("spawn").Pool(workers, initializer=_ref_attach,
                                                 initargs=([m.name for m in self.shm], rows))
        cuts = np.linspace(0, rows, 4 * workers + 1).astype(np.int64)
        assert sum(self.pool.starmap(_ref_fill, list(zip(cuts[:-1].tolist(), cuts[1:].tolist())))) == rows
        edges = np.linspace(0, SPAN, workers + 1).astype(np.int64)
        self.ranges = list(zip(edges[:-1].tolist(), edges[1:].tolist()))

    def step(self):
        return sum(self.pool.starmap(_ref_range, self.ranges, chunksize=1))

    def close(self):
        self.pool.close()
        self.pool.join()
        for m in self.shm:
            m.close()
            m.unlink()


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload == "batch":
        return run_reference_batch(args, world)
    if args.workload == "filter":
        return run_reference_filter(args, world)
    if args.workload == "count_distinct":
        return run_reference_count_distinct(args, world)
    if args.workload == "composite":
        return run_reference_composite(args, world)
    if args.workload == "planner":
        print(json.dumps({"impl": "reference", "metric": PLANNER_METRIC,
                          "unavailable": "the reference has no learned planner; its fixed rule is the "
                                         "denominator of this metric (the cuda arm times both)"}), flush=True)
        return
    if args.workload == "sorted":
        print(json.dumps({"impl": "reference", "metric": SORTED_METRIC,
                          "unavailable": "measured in the cuda arm only (the headline's reference arm covers "
                                         "the group-by)"}), flush=True)
        return
    if args.workload != "groupby":
        return run_reference_unique(args, world)
    rows = args.rows
    cores = args.ref_procs or host_cores()
    t_fill = time.perf_counter()
    pool = RefPool(rows, cores)
    t_fill = time.perf_counter() - t_fill
    try:
        for _ in range(max(1, args.warmup)):
            groups = pool.step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            groups = pool.step()
        dt = time.perf_counter() - t0
    finally:
        pool.close()
    value = rows * args.steps / dt / 1e6
    sample = ("the full workload (%d rows, same distributions and seeds as the cuda arm; %d groups) every "
              "step, grouped by %d processes over key ranges; inputs filled in %.1f s before timing"
              % (rows, groups, cores, t_fill))
    config = CONFIG if rows == N_ROWS and args.span == SPAN else dict(CONFIG, rows=rows, key_domain=args.span)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mrows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64+f64",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": value, "unit": "Mrows/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "Mrows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _reference_line(args, world, metric, value, unit, ms, config, sample, dtype):
    return {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": config,
            "cpu_baseline": {"value": value, "unit": unit, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_filter(args, world):
    """The reference's order of work on a 10M-row sample: filter node (compaction), then
    groupby_multi (oracle port)."""
    from oracle import nf_oracle as O
    rows = 10_000_000
    k, cols, val = cpu_sample(rows)
    keep = O.fill_f64(rows, SEED, 8, 0, 0.0, 1.0) >= 0.5
    ops = {"v": ("sum", "count", "min", "max"), "f": ("sum", "min", "max")}

    def step():
        kk = k[keep]
        cc = {c: v[keep] for c, v in cols.items()}
        vv = {c: m[keep] for c, m in val.items()}
        O.groupby_multi(kk, cc, ops, vv)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = rows * args.steps / dt / 1e6
    line = _reference_line(args, world, FILTER_METRIC, value, "Mrows/s", dt / args.steps * 1e3,
                           dict(CONFIG, workload="filter_then_groupby_100M_rows_10M_keys"),
                           "%d-row sample of the workload, filter then group, per step" % rows, "int64+f64")
    print(json.dumps(line), flush=True)


def run_reference_unique(args, world):
    import numpy as np
    from oracle import nf_oracle as O
    rows = 10_000_000
    if args.workload == "unique_full":
        keys = O.fill_i32(rows, SEED, 10, 0, -2 ** 31, 2 ** 31)
    else:
        vals = O.fill_i32(1000, SEED, 11, 0, -2 ** 31, 2 ** 31)
        nruns = rows // 5000 + 1000
        lens = O.fill_i32(nruns, SEED, 12, 0, 1, 10001).astype(np.int64)
        pick = O.fill_i32(nruns, SEED, 13, 0, 0, 1000).astype(np.int64)
        keys = np.repeat(vals[pick], lens)[:rows]
    for _ in range(args.warmup):
        O.unique_first_count(keys)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.unique_first_count(keys)
    dt = time.perf_counter() - t0
    value = rows * args.steps / dt / 1e6
    line = _reference_line(args, world, UNIQUE_METRIC, value, "Mkeys/s", dt / args.steps * 1e3,
                           {"workload": args.workload, "rows": rows},
                           "first %d keys of the workload, per step" % rows, "int32")
    print(json.dumps(line), flush=True)


def batch_cpu_sample(lay, target_rows=20_000_000):
    """Host keys/values of the batch workload's first queries totalling about target_rows
    (same Philox lanes as the device generator)."""
    import numpy as np
    from oracle import nf_oracle as O
    from numfast_b200 import batch as B
    ro = lay["row_offsets"]
    nq = int(np.searchsorted(ro, target_rows)) or 1
    nq = min(nq, ro.size - 1)
    ks, vs = [], []
    for q in range(nq):
        r = int(ro[q + 1] - ro[q])
        c, b = int(lay["card"][q]), int(lay["base"][q])
        if lay["zipf"][q]:
            u = O.fill_f64(r, SEED, q, 0, 0.0, 1.0)
            oms = 1.0 - float(lay["s"][q])
            x = (1.0 + u * ((c + 1.0) ** oms - 1.0)) ** (1.0 / oms)
            k = np.clip(np.floor(x).astype(np.int64), 1, c) - 1 + b
        else:
            k = O.fill_i32(r, SEED, q, 0, b, b + c)
        ks.append(np.asarray(k, dtype=np.int32))
        vs.append(O.fill_i32(r, SEED, B.VALUE_STREAM_BASE + q, 0, -1000, 1001))
    return np.concatenate(ks), np.concatenate(vs), ro[:nq + 1].copy()


def run_reference_batch(args, world):
    from oracle import nf_oracle as O
    from numfast_b200 import batch as B
    lay = B.config4_layout()
    k, v, ro = batch_cpu_sample(lay)
    rows = int(ro[-1])
    for _ in range(args.warmup):
        O.batch_sum_count(k, v, ro)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.batch_sum_count(k, v, ro)
    dt = time.perf_counter() - t0
    value = rows * args.steps / dt / 1e6
    line = _reference_line(args, world, BATCH_METRIC, value, "Mrows/s", dt / args.steps * 1e3, BATCH_CONFIG,
                           "first %d queries (%d rows) of the batch, per step" % (ro.size - 1, rows), "int64")
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU side

class Clocks:
    """nvidia-smi sampler over the timed region."""

    def __init__(self, index):
        self.index = index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs(rows, device, span=SPAN):
    from numfast_b200 import device as dev
    k = dev.rng_fill_i32(rows, SEED, 0, 0, span, device=device)
    v = dev.rng_fill_i32(rows, SEED, 1, -1000, 1001, device=device)
    f = dev.gen_lognormal(rows, SEED, 2, 3, 3.0, 1.0, device=device)
    bms = [dev.gen_validity(rows, SEED, s, P_NULL, device=device) for s in (4, 5, 6)]
    return k, v, f, bms


def max_over_ranks(ms, device, world):
    """A step's device time as the slowest rank's: every rank calls it with its own CUDA-event
    time (the replicas share no data; this reduction is the only collective)."""
    if world == 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(rows_per_rank, world, ms_per_step):
    """Whole-job Mrows/s of N replicas: every rank's rows over the slowest rank's step time."""
    return rows_per_rank * world / (ms_per_step / 1e3) / 1e6


def run_cuda(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from numfast_b200 import device as dev

    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    rows = args.rows
    k, v, f, bms = make_inputs(rows, device, args.span)
    cols = [dev.DeviceColumn("v", v, ("sum", "min", "max"), bms[1]),
            dev.DeviceColumn("f", f, ("sum", "min", "max"), bms[2])]
    bufs = dev.GroupbyBuffers(rows, cols, device)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()

    def step(timing=False):
        return dev.groupby(k, cols, bms[0], buffers=bufs, timing=timing)

    for _ in range(max(args.warmup, 3)):
        r = step()
    torch.cuda.synchronize()
    # Per-stage device times (CUDA events on the launching stream) over timed-like calls.
    stage_runs = [step(timing=True).probe["stage_ms"] for _ in range(5)]
    ng = r.ngroups
    strategy = r.strategy
    launches_per_step = r.probe["launches"]

    clocks = Clocks(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_ms = max_over_ranks(e0.elapsed_time(e1), device, world)
    if world > 1:
        dist.barrier()
    ms_per_step = dev_ms / args.steps
    value = replica_rate(rows, world, ms_per_step)

    # ---- e2e: host (pinned) inputs -> H2D -> group-by -> D2H of the result ----
    # Every step copies its inputs in from pinned host memory and its grouped
    # result back out.  Steps are pipelined over three streams (copy-in,
    # group-by, copy-out) with double-buffered device inputs and outputs, so
    # the copy-in of step i+1 and the copy-out of step i-1 overlap step i.
    hk = k.cpu().pin_memory()
    hv = v.cpu().pin_memory()
    hf = f.cpu().pin_memory()
    hb = [b.cpu().pin_memory() for b in bms]
    del k, v, f, bms, cols
    torch.cuda.empty_cache()
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    slots = []
    for _ in range(2):
        dk, dv, df = torch.empty_like(hk, device=device), torch.empty_like(hv, device=device), \
            torch.empty_like(hf, device=device)
        db = [torch.empty_like(h, device=device) for h in hb]
        ecols = [dev.DeviceColumn("v", dv, ("sum", "min", "max"), db[1]),
                 dev.DeviceColumn("f", df, ("sum", "min", "max"), db[2])]
        slots.append({"k": dk, "v": dv, "f": df, "b": db, "cols": ecols,
                      "bufs": bufs if not slots else dev.GroupbyBuffers(rows, ecols, device),
                      "in_done": torch.cuda.Event(), "comp_done": torch.cuda.Event(), "out_done": torch.cuda.Event()})
    out_host = [{name: torch.empty(rows, dtype=t.dtype).pin_memory()
                 for name, t in [("ukeys", sl["bufs"].ukeys), ("counts", sl["bufs"].counts)] +
                 [("sum_" + c, t) for c, t in sl["bufs"].sum.items()] +
                 [("min_" + c, t) for c, t in sl["bufs"].min.items()] +
                 [("max_" + c, t) for c, t in sl["bufs"].max.items()]} for sl in slots]

    def copy_in(i):
        sl = slots[i % 2]
        with torch.cuda.stream(s_in):
            s_in.wait_event(sl["comp_done"])  # the group-by two steps back has finished reading
            sl["k"].copy_(hk, non_blocking=True)
            sl["v"].copy_(hv, non_blocking=True)
            sl["f"].copy_(hf, non_blocking=True)
            for d, h in zip(sl["b"], hb):
                d.copy_(h, non_blocking=True)
            sl["in_done"].record(s_in)

    def compute_and_copy_out(i):
        sl = slots[i % 2]
        s_comp.wait_event(sl["in_done"])
        s_comp.wait_event(sl["out_done"])  # the copy-out two steps back has drained the outputs
        res = dev.groupby(sl["k"], sl["cols"], sl["b"][0], stream=s_comp, buffers=sl["bufs"])
        sl["comp_done"].record(s_comp)
        n_out = res.ngroups
        srcs = {"ukeys": res.ukeys, "counts": res.counts}
        srcs.update({"sum_" + c: t for c, t in res.sums.items()})
        srcs.update({"min_" + c: t for c, t in res.mins.items()})
        srcs.update({"max_" + c: t for c, t in res.maxs.items()})
        d2h = 0
        with torch.cuda.stream(s_out):
            s_out.wait_event(sl["comp_done"])
            for name, t in srcs.items():
                out_host[i % 2][name][:n_out].copy_(t, non_blocking=True)
                d2h += n_out * t.element_size()
            sl["out_done"].record(s_out)
        return d2h

    def e2e_run(nsteps):
        d2h = 0
        copy_in(0)
        for i in range(nsteps):
            if i + 1 < nsteps:
                copy_in(i + 1)
            d2h = compute_and_copy_out(i)
        return d2h

    e2e_run(2)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(s_in)
    d2h = e2e_run(args.e2e_steps)
    s_in.wait_stream(s_out)
    s_in.wait_stream(s_comp)
    t1.record(s_in)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(t0.elapsed_time(t1), device, world)
    h2d = sum(x.numel() * x.element_size() for x in [hk, hv, hf] + hb)
    e2e_value = replica_rate(rows, world, e2e_ms / args.e2e_steps)

    if rank != 0:
        return
    peak, peak_kind = peaks()
    alg_bytes = ALG_IN_BYTES_PER_ROW * rows + ALG_OUT_BYTES_PER_GROUP * ng
    stage_avg = [statistics.mean(s[i] for s in stage_runs) for i in range(len(stage_runs[0]))]
    stage_names = {"partition": ["probe", "histogram+plan", "merge_init+scatter", "aggregate"],
                   "dense_global": ["probe", "state_init", "aggregate", "compact"],
                   "dense_smem": ["probe", "state_init", "aggregate", "compact"],
                   "hash": ["probe", "table_init", "aggregate", "extract+sort+emit"]}.get(strategy, [])
    stages = [{"stage": nm, "ms": ms, "share": ms / sum(stage_avg)} for nm, ms in zip(stage_names, stage_avg)]
    achieved = alg_bytes / (ms_per_step / 1e3) / 1e9
    traffic = MEASURED_DRAM_BYTES.get((rows, args.span))
    config = CONFIG if rows == N_ROWS and args.span == SPAN else dict(CONFIG, rows=rows, key_domain=args.span)
    line = {
        "metric": METRIC, "value": value, "unit": "Mrows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32/int64 exact + f64", "data": "synthetic (device Philox, seed 42)",
        "config": config,
        "groupby": {"strategy": strategy, "groups": ng},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "group-by call (all stages of one nfc_groupby)",
                     "algorithmic_bytes": alg_bytes, "stages": stages,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per kernel on a 40M-row case, scaled to the rows",
                     "dominant_stage": max(stages, key=lambda x: x["ms"])["stage"] if stages else None},
        "e2e": {"value": e2e_value, "unit": "Mrows/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": args.e2e_steps},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and world == 1:
        rows_cpu = 10_000_000
        rate, times = cpu_groupby_rate(rows_cpu, 3)
        line["cpu_baseline"] = {"value": rate, "unit": "Mrows/s", "cores": 1, "kind": "port",
                                "sample": "%d-row sample of the workload, median of 3 (%.1f s each)"
                                          % (rows_cpu, statistics.median(times))}
    return line


# ------------------------------------------------------------------ unique (200M keys)

UNIQUE_ROWS = 200_000_000
UNIQUE_METRIC = "radix unique + first-occurrence row + count, Mkeys/s @200M int32 keys"


def make_unique_keys(kind, rows, device):
    """unique_full: keys uniform over the whole int32 range.  unique_runs: 1,000 distinct
    values (uniform int32) laid out in runs of length uniform in [1, 10000]."""
    import torch
    from numfast_b200 import device as dev
    if kind == "unique_full":
        return dev.rng_fill_i32(rows, SEED, 10, -2 ** 31, 2 ** 31, device=device)
    vals = dev.rng_fill_i32(1000, SEED, 11, -2 ** 31, 2 ** 31, device=device)
    nruns = rows // 5000 + 1000
    lens = dev.rng_fill_i32(nruns, SEED, 12, 1, 10001, device=device).long()
    pick = dev.rng_fill_i32(nruns, SEED, 13, 0, 1000, device=device).long()
    keys = torch.repeat_interleave(vals[pick], lens)
    assert keys.numel() >= rows
    return keys[:rows].contiguous()


def run_unique(args, rank, world, local_rank):
    import torch
    from numfast_b200 import device as dev
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    rows = args.rows if args.rows != N_ROWS else UNIQUE_ROWS
    keys = make_unique_keys(args.workload, rows, device)
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        r = dev.unique(keys)
    torch.cuda.synchronize()
    ng = r["ng"]
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0.record(stream)
    for _ in range(args.steps):
        dev.unique(keys)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    value = rows / (ms / 1e3) / 1e6
    peak, peak_kind = peaks()
    alg = 4.0 * rows + 16.0 * ng
    achieved = alg / (ms / 1e3) / 1e9
    line = {"metric": UNIQUE_METRIC, "value": value, "unit": "Mkeys/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (device Philox, seed 42)",
            "config": {"workload": args.workload, "rows": rows, "distinct": ng,
                       "l2": "inputs 0.8 GB > L2 (126 MB): no flush needed"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg, "kernel": "unique call (all kernels of one nfc_unique)"},
            "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import nf_oracle as O
        sample = 10_000_000
        hk = keys[:sample].cpu().numpy()
        t0 = time.perf_counter()
        O.unique_first_count(hk)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": sample / dt / 1e6, "unit": "Mkeys/s", "cores": 1, "kind": "port",
                                "sample": "first %d keys of the workload, one run (%.1f s)" % (sample, dt)}
    return line if rank == 0 else None


def run_batch(args, rank, world, local_rank):
    import numpy as np
    import torch
    from numfast_b200 import batch as B
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    lay = B.config4_layout(nq=args.batch_queries)
    keys, vals = B.make_config4(lay, device)
    ro = lay["row_offsets"]
    n = int(ro[-1])
    cap = n // 4
    torch.cuda.synchronize()
    report = None
    if args.no_autotune:
        tuning = B.default_tuning()
    else:
        tuning, report = B.autotune(ro, keys, vals, reps=3, out_cap=cap, cache_path=args.tune_cache,
                                    log=lambda m: print(m, file=sys.stderr, flush=True))
    b = B.BatchGroupby(ro, tuning)
    res = b.run(keys, vals, out_cap=cap, graph=True)
    deferred = res.deferred
    ng_total = int(res.ngroups.sum())
    plans = b.plans()
    plan_counts = {p: plans.count(p) for p in sorted(set(plans))}
    prof = b.profile()
    # A step is complete only once deferred queries (if any) are finished on the
    # single-query path, so such a batch is timed with the synchronous call.
    sync = deferred > 0
    for _ in range(max(args.warmup, 3)):
        b.run(keys, vals, out_cap=cap, graph=True, sync=sync)
    b.finish()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0.record(stream)
    for _ in range(args.steps):
        b.run(keys, vals, out_cap=cap, graph=True, sync=sync)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    assert b.finish() == (0 if sync else deferred)
    ms = e0.elapsed_time(e1) / args.steps
    value = n / (ms / 1e3) / 1e6
    peak, peak_kind = peaks()
    alg = 8.0 * n + 24.0 * ng_total
    achieved = alg / (ms / 1e3) / 1e9
    cfg = dict(BATCH_CONFIG, queries=args.batch_queries, rows=n, groups=ng_total, out_cap=cap,
               deferred_queries=deferred, plans=plan_counts,
               item_profile=prof,
               tuning=tuning.as_dict(), autotune=report and {k: report[k] for k in ("ms", "default_ms", "trials",
                                                                                   "cached")})
    # End to end through the public API: pinned host inputs copied in, grouped result
    # (ukeys, sums, counts, offsets, group counts) copied out, every step.
    hk = torch.empty(n, dtype=torch.int32, pin_memory=True)
    hv = torch.empty(n, dtype=torch.int32, pin_memory=True)
    hk.copy_(keys)
    hv.copy_(vals)
    dk, dv = torch.empty_like(keys), torch.empty_like(vals)
    out_h = [torch.empty(ng_total + 1, dtype=torch.int64, pin_memory=True) for _ in range(3)]
    meta_h = torch.empty(2 * len(ro), dtype=torch.int64, pin_memory=True)
    e2e_steps = max(1, min(args.e2e_steps, 3))
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    d2h = 0
    t0.record(stream)
    for _ in range(e2e_steps):
        dk.copy_(hk, non_blocking=True)
        dv.copy_(hv, non_blocking=True)
        r = b.run(dk, dv, out_cap=cap, graph=True)
        used = int(torch.max(r.group_offsets + r.ngroups))
        for src, dst in zip((r.ukeys, r.sums, r.counts), out_h):
            dst[:min(used, dst.numel())].copy_(src[:min(used, dst.numel())], non_blocking=True)
        meta_h[:len(ro) - 1].copy_(r.group_offsets, non_blocking=True)
        meta_h[len(ro):2 * len(ro) - 1].copy_(r.ngroups, non_blocking=True)
        d2h = 3 * 8 * min(used, ng_total + 1) + 2 * 8 * (len(ro) - 1)
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = t0.elapsed_time(t1) / e2e_steps
    line = {"metric": BATCH_METRIC, "value": value, "unit": "Mrows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32 in, int64 exact sums/counts",
            "data": "synthetic (device Philox, seed 42 / stream per query)", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg,
                         "kernel": "k_batch (one persistent launch per step; 8 B/row in + 24 B/group out)"},
            "e2e": {"value": n / (e2e_ms / 1e3) / 1e6, "unit": "Mrows/s", "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "gpu_launches": args.steps, "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import nf_oracle as O
        k, v, sro = batch_cpu_sample(lay)
        t0 = time.perf_counter()
        O.batch_sum_count(k, v, sro)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": int(sro[-1]) / dt / 1e6, "unit": "Mrows/s", "cores": 1, "kind": "port",
                                "sample": "first %d queries (%d rows) of the batch, one run (%.1f s)"
                                % (sro.size - 1, int(sro[-1]), dt)}
    b.close()
    return line if rank == 0 else None


def run_planner(args, rank, world, local_rank):
    """A stream of inputs (100K..50M rows; uniform / Zipf / runs / clustered keys, dense or
    scattered key values; sum+count of an int32 value), each grouped once by the fixed
    planner and once by the learned planner; value = fixed time / learned time."""
    import numpy as np
    import torch
    from numfast_b200 import _lib
    from numfast_b200 import planner as PL
    torch.cuda.set_device(local_rank)
    planner = PL.LearnedPlanner.load()
    specs = PL.draw_specs(args.inputs, PLANNER_SEED)
    modes = ("fixed", "learned", "auto")
    tot = {m: 0.0 for m in modes}
    rows = 0
    groups = 0
    launches = 0
    picks = {m: {} for m in modes}
    fallbacks = 0
    mismatches = 0
    # Output buffers sized for the largest input up front: no allocation while timing.
    bufs = PL.sum_count_buffers(max(sp["rows"] for sp in specs))
    for sp in specs[:3]:  # warm every code path once
        keys, vals = PL.make_input(sp)
        for m in modes:
            _, _, bufs = PL.groupby_sum_count(keys, vals, mode=m, planner=planner, buffers=bufs)
    torch.cuda.synchronize()
    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    dump = open(args.dump, "w") if getattr(args, "dump", None) else None
    for sp in specs:
        keys, vals = PL.make_input(sp)
        ref = None
        rec = {k: sp[k] for k in ("id", "rows", "card", "kind", "s", "sparse", "mean_run")}
        for m in modes:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ng, st, bufs = PL.groupby_sum_count(keys, vals, mode=m, planner=planner, buffers=bufs)
            e1.record()
            e1.synchronize()
            tot[m] += e0.elapsed_time(e1)
            name = _lib.STRATEGY_NAMES.get(st.strategy, str(st.strategy))
            rec[m] = (name, round(e0.elapsed_time(e1), 4))
            picks[m][name] = picks[m].get(name, 0) + 1
            launches += st.launches + (2 if m == "learned" else 0)  # + sketch pass 1, pass 2 with the network
            if m == "learned" and st.planner_used != _lib.PLANNER_LEARNED:
                fallbacks += 1
            out = (ng, bufs["ukeys"][:ng].clone(), bufs["sum"][:ng].clone(), bufs["counts"][:ng].clone())
            if ref is None:
                ref = out
            elif ref[0] != out[0] or not all(torch.equal(a, b) for a, b in zip(ref[1:], out[1:])):
                mismatches += 1
        rows += sp["rows"]
        groups += ref[0]
        if dump:
            rec["ng"] = ref[0]
            dump.write(json.dumps(rec) + "\n")
        del keys, vals
    clk = clocks.stop()
    if dump:
        dump.close()
    speedup = tot["fixed"] / tot["learned"]
    peak, peak_kind = peaks()
    alg = 8.0 * rows + 24.0 * groups
    achieved = alg / (tot["learned"] / 1e3) / 1e9
    # End to end through host buffers on the first inputs (pinned copies in and out).
    n_e2e = min(len(specs), 100)
    e2e_ms = 0.0
    e2e_rows = 0
    h2d = d2h = 0
    for sp in specs[:n_e2e]:
        keys, vals = PL.make_input(sp)
        hk = torch.empty(keys.numel(), dtype=torch.int32, pin_memory=True)
        hv = torch.empty_like(hk, pin_memory=True)
        hk.copy_(keys)
        hv.copy_(vals)
        dk, dv = torch.empty_like(keys), torch.empty_like(vals)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dk.copy_(hk, non_blocking=True)
        dv.copy_(hv, non_blocking=True)
        ng, st, bufs = PL.groupby_sum_count(dk, dv, mode="learned", planner=planner, buffers=bufs)
        ho = torch.empty(3 * max(ng, 1), dtype=torch.int64, pin_memory=True)
        ho[:ng].copy_(bufs["ukeys"][:ng], non_blocking=True)
        ho[ng:2 * ng].copy_(bufs["sum"][:ng], non_blocking=True)
        ho[2 * ng:3 * ng].copy_(bufs["counts"][:ng], non_blocking=True)
        e1.record()
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        e2e_rows += sp["rows"]
        h2d += 8 * sp["rows"]
        d2h += 24 * ng
        del keys, vals, dk, dv
    line = {"metric": PLANNER_METRIC, "value": speedup, "unit": "x", "n_gpus": world, "steps": len(specs),
            "warmup": 3, "ms_per_step": tot["learned"] / len(specs), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32 in, int64 exact sums/counts",
            "data": "synthetic (device Philox, seed %d, one stream per input)" % PLANNER_SEED,
            "config": {"workload": "planner_stream_%d_inputs_rows_100K_50M" % len(specs), "inputs": len(specs),
                       "rows": rows, "groups": groups, "mrows_per_s": {m: rows / tot[m] / 1e3 for m in modes},
                       "learned_speedup_vs_fixed": speedup, "learned_speedup_vs_auto": tot["auto"] / tot["learned"],
                       "total_ms": tot, "strategy_counts": picks, "learned_fallbacks": fallbacks,
                       "result_mismatches": mismatches,
                       "l2": "every input is regenerated before its timed calls; inputs above 16M rows exceed L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": peak_kind, "algorithmic_bytes": alg,
                         "kernel": "whole stream under the learned planner (8 B/row in + 24 B/group out)"},
            "e2e": {"value": e2e_rows / e2e_ms / 1e3, "unit": "Mrows/s", "h2d_bytes_per_step": h2d // n_e2e,
                    "d2h_bytes_per_step": d2h // n_e2e, "steps": n_e2e,
                    "note": "learned planner, first %d inputs, pinned host buffers" % n_e2e},
            "gpu_launches": launches, "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import nf_oracle as O
        sample_rows = 0
        dt = 0.0
        for sp in specs:
            if sample_rows > 20_000_000:
                break
            keys, vals = PL.make_input(sp)
            hk, hv = keys.cpu().numpy(), vals.cpu().numpy()
            t0 = time.perf_counter()
            O.groupby_multi(hk, {"v": hv}, {"v": ("sum", "count")})
            dt += time.perf_counter() - t0
            sample_rows += sp["rows"]
        line["cpu_baseline"] = {"value": sample_rows / dt / 1e6, "unit": "Mrows/s", "cores": 1, "kind": "port",
                                "sample": "first inputs of the stream (%d rows), one run each" % sample_rows}
    return line if rank == 0 else None


def run_filter(args, rank, world, local_rank):
    """The headline group-by behind a filter keeping about half the rows: fused (the filter
    is one more bitmap in the probe) against compacting every column on the device first
    (torch boolean indexing, bitmaps unpacked and repacked) and grouping the survivors."""
    import torch
    from numfast_b200 import device as dev
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    rows = args.rows
    k, v, f, bms = make_inputs(rows, device, args.span)
    keep = dev.rng_fill_f64(rows, SEED, 8, device=device) >= 0.5
    weights = (2 ** torch.arange(8, device=device, dtype=torch.int32)).view(1, 8)

    def pack(b):
        pad = (-b.numel()) % 8
        bb = torch.cat([b, b.new_zeros(pad)]) if pad else b
        return (bb.view(-1, 8).to(torch.int32) * weights).sum(1).to(torch.uint8)

    def unpack(bm, n):
        bits = (bm.view(-1, 1).to(torch.int32) >> torch.arange(8, device=device, dtype=torch.int32)) & 1
        return bits.view(-1)[:n].bool()

    fbm = pack(keep)
    bufs = dev.GroupbyBuffers(rows, [dev.DeviceColumn("v", v, ("sum", "min", "max")),
                                     dev.DeviceColumn("f", f, ("sum", "min", "max"))], device)

    def fused():
        return dev.groupby(k, [dev.DeviceColumn("v", v, ("sum", "min", "max"), bms[1]),
                               dev.DeviceColumn("f", f, ("sum", "min", "max"), bms[2])], bms[0],
                           buffers=bufs, row_filter=fbm)

    def unfused():
        kk, vv, ff = k[keep], v[keep], f[keep]
        vb = [pack(unpack(b, rows)[keep]) for b in bms]
        return dev.groupby(kk, [dev.DeviceColumn("v", vv, ("sum", "min", "max"), vb[1]),
                                dev.DeviceColumn("f", ff, ("sum", "min", "max"), vb[2])], vb[0], buffers=bufs)

    def timed(fn, steps):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, r

    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    ms_f, rf = timed(fused, args.steps)
    clk = clocks.stop()
    ng = rf.ngroups
    uk = rf.ukeys.clone()
    ms_u, ru = timed(unfused, max(3, args.steps // 4))
    assert ru.ngroups == ng and torch.equal(ru.ukeys, uk)
    peak, peak_kind = peaks()
    alg = ALG_IN_BYTES_PER_ROW * rows + rows / 8.0 + ALG_OUT_BYTES_PER_GROUP * ng
    line = {"metric": FILTER_METRIC, "value": rows / (ms_f / 1e3) / 1e6, "unit": "Mrows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_f, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64 exact + f64",
            "data": "synthetic (device Philox, seed 42; filter u >= 0.5 on stream 8)",
            "config": dict(CONFIG, workload="filter_then_groupby_100M_rows_10M_keys", rows=rows,
                           kept=int(keep.sum()), groups=ng, fused_ms=ms_f, compact_then_group_ms=ms_u,
                           fused_speedup=ms_u / ms_f),
            "roofline": {"bound": "hbm", "achieved": alg / (ms_f / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms_f / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg, "kernel": "fused group-by call (filter bitmap in the probe)"},
            "clocks": clk}
    return line if rank == 0 else None


def cd_inputs_host(rows):
    from oracle import nf_oracle as O
    k = O.fill_i32(rows, SEED, 20, 0, 0, 1_000_000)
    v = O.fill_i32(rows, SEED, 21, 0, 0, 100_000)
    kv = O.fill_f64(rows, SEED, 22) >= P_NULL
    return k, v, kv


def run_count_distinct(args, rank, world, local_rank):
    """group_count_distinct over 100M rows: keys uniform over 1M values, values over 100K,
    5% NULL keys; value = input rows per second of the whole call."""
    import torch
    from numfast_b200 import device as dev
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    rows = args.rows
    k = dev.rng_fill_i32(rows, SEED, 20, 0, 1_000_000, device=device)
    v = dev.rng_fill_i32(rows, SEED, 21, 0, 100_000, device=device)
    kv = dev.gen_validity(rows, SEED, 22, P_NULL, device=device)
    for _ in range(max(args.warmup, 3)):
        uk, nu = dev.group_count_distinct(k, v, kv)
    torch.cuda.synchronize()
    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        uk, nu = dev.group_count_distinct(k, v, kv)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ng = int(uk.numel())
    peak, peak_kind = peaks()
    alg = 8.0 * rows + rows / 8.0 + 16.0 * ng
    line = {"metric": DISTINCT_METRIC, "value": rows / (ms / 1e3) / 1e6, "unit": "Mrows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 in, int64 out",
            "data": "synthetic (device Philox, seed 42, streams 20-22)",
            "config": {"workload": "count_distinct_100M_rows_1M_keys_100K_values", "rows": rows, "groups": ng,
                       "pairs": int(nu.sum()), "l2": "inputs 0.8 GB > L2: no flush needed"},
            "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg, "kernel": "group_count_distinct call (pack, 8 sort passes max, runs)"},
            "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import nf_oracle as O
        sample = 10_000_000
        hk, hv, hkv = cd_inputs_host(sample)
        t0 = time.perf_counter()
        O.group_count_distinct(hk, hv, hkv)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": sample / dt / 1e6, "unit": "Mrows/s", "cores": 1, "kind": "port",
                                "sample": "%d-row sample of the workload, one run (%.1f s)" % (sample, dt)}
    return line if rank == 0 else None


def run_reference_count_distinct(args, world):
    from oracle import nf_oracle as O
    rows = 10_000_000
    k, v, kv = cd_inputs_host(rows)
    for _ in range(args.warmup):
        O.group_count_distinct(k, v, kv)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.group_count_distinct(k, v, kv)
    dt = time.perf_counter() - t0
    value = rows * args.steps / dt / 1e6
    line = _reference_line(args, world, DISTINCT_METRIC, value, "Mrows/s", dt / args.steps * 1e3,
                           {"workload": "count_distinct_100M_rows_1M_keys_100K_values"},
                           "%d-row sample of the workload, per step" % rows, "int64")
    print(json.dumps(line), flush=True)


def comp_inputs_host(rows):
    from oracle import nf_oracle as O
    return (O.fill_i32(rows, SEED, 30, 0, -500, 500), O.fill_i32(rows, SEED, 31, 0, 0, 10_000),
            O.fill_i32(rows, SEED, 32, 0, -1000, 1001))


def run_composite(args, rank, world, local_rank):
    """group(key=(a, b), {v: (sum, count)}) over 100M rows: a uniform over 1,000 values, b
    over 10,000 (about 10M distinct tuples); value = input rows per second of the call
    (composite codes + group-by of the codes + key columns of the groups)."""
    import torch
    from numfast_b200 import device as dev
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    rows = args.rows
    a = dev.rng_fill_i32(rows, SEED, 30, -500, 500, device=device)
    b = dev.rng_fill_i32(rows, SEED, 31, 0, 10_000, device=device)
    v = dev.rng_fill_i32(rows, SEED, 32, -1000, 1001, device=device)
    cols = [dev.DeviceColumn("v", v, ("sum",))]
    for _ in range(max(args.warmup, 3)):
        r = dev.groupby_composite([a, b], cols)
    torch.cuda.synchronize()
    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        r = dev.groupby_composite([a, b], cols)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ng = r.ngroups
    peak, peak_kind = peaks()
    alg = 12.0 * rows + 32.0 * ng
    line = {"metric": COMPOSITE_METRIC, "value": rows / (ms / 1e3) / 1e6, "unit": "Mrows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 in, int64 exact sums/counts",
            "data": "synthetic (device Philox, seed 42, streams 30-32)",
            "config": {"workload": "composite_100M_rows_1000x10000_tuples", "rows": rows, "groups": ng,
                       "l2": "inputs 1.2 GB > L2: no flush needed"},
            "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg,
                         "kernel": "composite codes (pack, radix sort, runs) + group-by of the codes"},
            "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import nf_oracle as O
        sample = 10_000_000
        ha, hb, hv = comp_inputs_host(sample)
        t0 = time.perf_counter()
        O.composite_groupby_sum_count([ha, hb], hv)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": sample / dt / 1e6, "unit": "Mrows/s", "cores": 1, "kind": "port",
                                "sample": "%d-row sample of the workload, one run (%.1f s)" % (sample, dt)}
    return line if rank == 0 else None


def run_reference_composite(args, world):
    from oracle import nf_oracle as O
    rows = 10_000_000
    ha, hb, hv = comp_inputs_host(rows)
    for _ in range(args.warmup):
        O.composite_groupby_sum_count([ha, hb], hv)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.composite_groupby_sum_count([ha, hb], hv)
    dt = time.perf_counter() - t0
    value = rows * args.steps / dt / 1e6
    line = _reference_line(args, world, COMPOSITE_METRIC, value, "Mrows/s", dt / args.steps * 1e3,
                           {"workload": "composite_100M_rows_1000x10000_tuples"},
                           "%d-row sample of the workload, per step" % rows, "int64")
    print(json.dumps(line), flush=True)


def run_sorted_wl(args, rank, world, local_rank):
    """The headline's rows with the keys sorted (uniform over the 10M-key domain, then
    sorted; values and NULLs as the headline): the group-by takes the one-pass run
    strategy; the atomic strategies are timed on the same input for comparison."""
    import torch
    from numfast_b200 import device as dev
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    rows = args.rows
    k, v, f, bms = make_inputs(rows, device, args.span)
    k = torch.sort(k)[0].contiguous()
    cols = [dev.DeviceColumn("v", v, ("sum", "min", "max"), bms[1]),
            dev.DeviceColumn("f", f, ("sum", "min", "max"), bms[2])]
    bufs = dev.GroupbyBuffers(rows, cols, device)

    def timed(strategy, steps):
        for _ in range(max(args.warmup, 3)):
            r = dev.groupby(k, cols, bms[0], buffers=bufs, strategy=strategy)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            r = dev.groupby(k, cols, bms[0], buffers=bufs, strategy=strategy)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, r

    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    ms, r = timed("auto", args.steps)
    clk = clocks.stop()
    assert r.strategy == "sorted", r.strategy
    ng = r.ngroups
    others = {st: timed(st, max(3, args.steps // 4))[0] for st in ("dense_global", "partition")}
    peak, peak_kind = peaks()
    alg = ALG_IN_BYTES_PER_ROW * rows + ALG_OUT_BYTES_PER_GROUP * ng
    line = {"metric": SORTED_METRIC, "value": rows / (ms / 1e3) / 1e6, "unit": "Mrows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64 exact + f64",
            "data": "synthetic (device Philox, seed 42; keys sorted)",
            "config": dict(CONFIG, workload="sorted_keys_groupby_100M_rows_10M_keys_5pct_nulls", rows=rows,
                           groups=ng, strategy=r.strategy, other_strategies_ms=others),
            "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg, "kernel": "sorted group-by call (probe, run pass, piece merge)"},
            "clocks": clk}
    return line if rank == 0 else None


def run_topk_wl(args, rank, world, local_rank):
    """sort("f", desc=True).limit(1000) on the headline's float64 column (lognormal, 5% NULLs,
    100M rows): nfc_sort_topk against the full stable argsort it replaces; the first k entries
    of the full permutation are checked equal before timing."""
    import torch
    from numfast_b200 import device as dev
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    rows = args.rows
    _, _, f, bms = make_inputs(rows, device, args.span)
    vb = bms[2]
    full = dev.sort_perm(f, True, vb)
    top = dev.sort_topk(f, TOPK_K, True, vb)
    torch.cuda.synchronize()
    assert torch.equal(full[:TOPK_K], top), "top-k differs from the full argsort"
    del full

    def timed(fn, steps):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    ms = timed(lambda: dev.sort_topk(f, TOPK_K, True, vb), args.steps)
    clk = clocks.stop()
    full_ms = timed(lambda: dev.sort_perm(f, True, vb), max(3, args.steps // 4))
    peak, peak_kind = peaks()
    alg = (8 + 1 / 8.0) * rows + 4 * TOPK_K
    line = {"metric": TOPK_METRIC, "value": rows / (ms / 1e3) / 1e6, "unit": "Mkeys/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 keys, int32 permutation",
            "data": "synthetic (device Philox, seed 42: the headline's lognormal column and its NULLs)",
            "config": {"workload": "topk_1000_of_100M_f64_desc_5pct_nulls", "rows": rows, "k": TOPK_K,
                       "full_argsort_ms": full_ms},
            "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg,
                         "kernel": "top-k call (digit histogram, one split pass, candidate and selection sorts)"},
            "clocks": clk}
    return line if rank == 0 else None


def run_side_workloads(args, local_rank):
    """The other configurations, measured in the same run as the headline (one GPU): sorted
    keys, top-k of the float64 column, radix unique over 200M keys (full range and runs), the
    batched persistent launch, and the learned-planner stream.  Each entry keeps its metric, time, roofline and clocks."""
    import copy
    import torch
    keep = ("metric", "value", "unit", "ms_per_step", "steps", "roofline", "clocks", "e2e", "gpu_launches")
    out = {}
    plan = [("sorted", run_sorted_wl, {"workload": "sorted", "steps": 10}),
            ("topk", run_topk_wl, {"workload": "topk", "steps": 20}),
            ("unique_full", run_unique, {"workload": "unique_full", "steps": 10}),
            ("unique_runs", run_unique, {"workload": "unique_runs", "steps": 10}),
            ("batch", run_batch, {"workload": "batch", "steps": 10}),
            ("planner", run_planner, {"workload": "planner"})]
    for name, fn, kw in plan:
        a = copy.copy(args)
        a.no_cpu_baseline = True
        a.rows, a.span = N_ROWS, SPAN
        a.dump = None
        for key, val in kw.items():
            setattr(a, key, val)
        t0 = time.time()
        try:
            line = fn(a, 0, 1, local_rank)
            ent = {key: line[key] for key in keep if key in line}
            cfg = dict(line.get("config", {}))
            if name == "planner":
                cfg = {key: cfg.get(key) for key in ("workload", "inputs", "rows", "groups", "total_ms",
                                                     "learned_speedup_vs_fixed", "learned_speedup_vs_auto",
                                                     "learned_fallbacks", "result_mismatches", "strategy_counts")}
            elif name == "batch":
                cfg = {key: cfg.get(key) for key in ("workload", "queries", "rows", "groups", "deferred_queries",
                                                     "plans", "autotune")}
            ent["config"] = cfg
        except Exception as e:  # one failing configuration must not hide the others
            ent = {"error": "%s: %s" % (type(e).__name__, str(e)[:300])}
        ent["wall_s"] = round(time.time() - t0, 1)
        out[name] = ent
        torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    single = {"batch": run_batch, "planner": run_planner, "filter": run_filter, "sorted": run_sorted_wl,
              "topk": run_topk_wl,
              "count_distinct": run_count_distinct, "composite": run_composite,
              "unique_full": run_unique, "unique_runs": run_unique}
    if args.workload in single:
        line = single[args.workload](args, rank, world, local_rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        line = run_cuda(args, rank, world, local_rank)
        if line is not None:
            if world == 1 and not args.no_workloads:
                line["workloads"] = run_side_workloads(args, local_rank)
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
