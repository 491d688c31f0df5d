"""Executor for the group-by path's IR nodes on the GPU.

Mirrors the node contract of the reference executor (cpu_execute,
src/Drivers/CPU/_lib/cpu.py:2734-4107) for the nodes on this path:

  series          bufs[out] = column, bufs[out+"#validity"] = bool mask (if any)
  groupby_multi   cpu.py:3435-3704 -> bufs[out] (dict, or ColumnCarry when
                  result="carry"), bufs[out+"#carry"], bufs[out+"#strategy"],
                  bufs[out+"#groupindex"]
  sort            cpu.py:3177-3187 -> int32 stable permutation, invalid rows last
  gather          cpu.py:3170-3176 -> values[idx] (+ gathered validity)
  unique_inverse  cpu.py:4006-4040 -> uniq, #inv (int32, -1 for invalid), #ng
  filter          values[mask] (host-side adjacency of the path)

Host numpy buffers in and out; every computation on the path is a
libnumfast_cuda kernel.  There is no CPU fallback: a missing library or a
device error raises.
"""

import os
import time

import numpy as np
import torch

from . import _lib
from . import device as dev
from .carry import ColumnCarry


class ExecError(ValueError):
    pass


_DEVICE = None


def _device():
    global _DEVICE
    if _DEVICE is None:
        if not torch.cuda.is_available():
            raise _lib.NativeUnavailable("no CUDA device: the group-by path runs only on the GPU")
        _lib.load()
        _DEVICE = torch.device("cuda", torch.cuda.current_device())
    return _DEVICE


def _to_dev(a):
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a)
    return t.to(_device(), non_blocking=False)


def _bitmap_dev(mask):
    return _to_dev(dev.pack_validity(mask))


_DTYPE_NAMES = {"int32": np.int32, "int64": np.int64, "float64": np.float64, "float32": np.float32,
                "bool": np.bool_, "int16": np.int16, "int8": np.int8, "uint8": np.uint8}


def _series(params, out, bufs):
    want = _DTYPE_NAMES.get(params.get("dtype", "int32"))
    if want is None:
        raise ExecError("series %r: unsupported dtype %r" % (out, params.get("dtype")))
    vals = params["values"]
    arr = np.asarray(vals)
    if want == np.int32 and arr.dtype.kind in "iu" and arr.size:
        if int(arr.min()) < -2 ** 31 or int(arr.max()) > 2 ** 31 - 1:
            raise ExecError("series %r: values outside int32" % out)
    bufs[out] = np.ascontiguousarray(arr.astype(want, copy=False))
    if params.get("validity") is not None:
        m = np.ascontiguousarray(np.asarray(params["validity"], dtype=bool))
        if m.size != bufs[out].size:
            raise ExecError("series %r: validity size %d != %d" % (out, m.size, bufs[out].size))
        bufs[out + "#validity"] = m


def _key_array(k, name):
    k = np.asarray(k)
    if not np.issubdtype(k.dtype, np.integer):
        raise ExecError("groupby_multi needs integer keys (encode categoricals to int codes first)")
    if k.dtype != np.int32:
        if k.size and (int(k.min()) < -2 ** 31 or int(k.max()) > 2 ** 31 - 1):
            raise ExecError("groupby_multi keys %r exceed int32" % name)
        k = k.astype(np.int32)
    return np.ascontiguousarray(k)



_PLANNER = {}


def _planner():
    """Strategy planner named by NUMFAST_CUDA_PLANNER: unset/auto (the library's span rule),
    fixed (the reference's plan_groupby rule) or learned (sketch + MLP, fixed as fallback)."""
    mode = os.environ.get("NUMFAST_CUDA_PLANNER", "auto").strip().lower() or "auto"
    if mode not in ("auto", "fixed", "learned"):
        raise ValueError("NUMFAST_CUDA_PLANNER must be auto, fixed or learned, not %r" % mode)
    if mode != "learned":
        return mode, None
    if "learned" not in _PLANNER:
        from .planner import LearnedPlanner
        _PLANNER["learned"] = LearnedPlanner.load()
    return mode, _PLANNER["learned"]


def _pack_keys(p, bufs):
    """pack_keys (cpu.py:2872-3020): mode "pack" -> int64 (hi << 32) | (uint32) lo; mode
    "radix" -> mixed-radix int64 ((c0 * M1 + c1) * M2 ...); mode "hash" -> the tuple of
    columns kept as the key (#tuple_cols), grouped by composite codes."""
    ins = [np.asarray(bufs[i]) for i in p["inputs"]]
    for a in ins:
        if not np.issubdtype(a.dtype, np.integer):
            raise ExecError("pack_keys needs int32 code series")
    mode = p["params"].get("mode", "pack")
    out = p["out"]
    if mode == "pack":
        if len(ins) == 1:
            bufs[out] = ins[0].astype(np.int64)
        else:
            bufs[out] = (ins[0].astype(np.int64) << 32) | (ins[1].astype(np.int64) & 0xFFFFFFFF)
    elif mode == "radix":
        rad = p["params"].get("radix") or [int(a.max()) + 1 if a.size else 1 for a in ins]
        total = 1
        for m in rad:
            total *= int(m)
        if total > 2 ** 63 - 1:
            raise ExecError("pack_keys radix product %d overflows int64" % total)
        comp = np.zeros(ins[0].size, dtype=np.int64)
        for a, m in zip(ins, rad):
            comp = comp * np.int64(m) + a.astype(np.int64)
        bufs[out] = comp
    elif mode == "hash":
        bufs[out + "#tuple_cols"] = [np.ascontiguousarray(a.astype(np.int32)) for a in ins]
        bufs[out] = np.zeros(ins[0].size, dtype=np.int64)
    else:
        raise ExecError("pack_keys mode %r" % mode)
    masks = [bufs[i + "#validity"] for i in p["inputs"] if i + "#validity" in bufs]
    if masks:
        m = masks[0]
        for x in masks[1:]:
            m = m & x
        bufs[out + "#validity"] = m


def _groupby_multi(p, bufs):
    params = p["params"]
    cols = params.get("cols")
    if cols is None:
        cols, multi = [p["inputs"][0]], False
        key_name = p["inputs"][1]
        ops_map = {cols[0]: list(params["ops"])}
    else:
        multi = True
        key_name = p["inputs"][len(cols)]
        ops_map = {c: list(params["ops"][c]) for c in cols}
    tuple_cols = bufs.get(key_name + "#tuple_cols")
    kraw = np.asarray(bufs[key_name])
    if tuple_cols is None and np.issubdtype(kraw.dtype, np.integer) and kraw.size and (
            int(kraw.min()) < -2 ** 31 or int(kraw.max()) > 2 ** 31 - 1):
        # int64 keys beyond int32: the (signed high, unsigned low) halves as a composite
        # key give the same order as the int64 values.
        k64 = kraw.astype(np.int64)
        tuple_cols = [(k64 >> 32).astype(np.int32), (k64 & 0xFFFFFFFF).astype(np.uint32).view(np.int32)]
        int64_key = True
    else:
        int64_key = False
    if tuple_cols is not None:
        if not int64_key and any("min" in ops_map[c] or "max" in ops_map[c] for c in cols):
            raise ExecError("composite groupby_multi needs sum/count/mean (min/max stay single-column)")
        k = np.zeros(tuple_cols[0].size, dtype=np.int32)
    else:
        k = _key_array(bufs[key_name], key_name)
    vs = [np.asarray(bufs[c]) for c in cols]
    for vv in vs:
        if vv.size != k.size:
            raise ExecError("groupby_multi values/keys size mismatch %d != %d" % (vv.size, k.size))
    t0 = time.perf_counter()
    dcols = []
    casts = {}
    for c, v in zip(cols, vs):
        ops = tuple(o for o in ops_map[c] if o != "count")
        if v.dtype == np.bool_ or (v.dtype.kind in "iu" and v.dtype.itemsize < 4) or v.dtype == np.uint32:
            v = v.astype(np.int64 if v.dtype == np.uint32 else np.int32)
        elif v.dtype == np.float32:
            casts[c] = np.float32
            v = v.astype(np.float64)
        elif v.dtype == np.uint64:
            raise ExecError("groupby_multi: uint64 values unsupported")
        vm = bufs.get(c + "#validity")
        dcols.append(dev.DeviceColumn(c, _to_dev(v), ops, _bitmap_dev(vm) if vm is not None else None))
    km = bufs.get(key_name + "#validity")
    rf = None
    if params.get("filter") is not None:
        fm = np.asarray(bufs[params["filter"]], dtype=bool)
        if fm.size != k.size:
            raise ExecError("groupby_multi filter size %d != %d" % (fm.size, k.size))
        rf = _bitmap_dev(fm)
    mode, planner = _planner()
    if tuple_cols is not None:
        res = dev.groupby_composite([_to_dev(c) for c in tuple_cols], dcols,
                                    _bitmap_dev(km) if km is not None else None, row_filter=rf)
        torch.cuda.synchronize()
        kc = [c.cpu().numpy() for c in res.key_columns]
        if int64_key:
            ukeys = (kc[0].astype(np.int64) << 32) | (kc[1].astype(np.int64) & 0xFFFFFFFF)
        else:
            ukeys = np.empty(kc[0].size, dtype=object)
            ukeys[:] = list(zip(*[c.tolist() for c in kc]))
    else:
        res = dev.groupby(_to_dev(k), dcols, _bitmap_dev(km) if km is not None else None,
                          strategy=params.get("strategy", "auto"), planner_mode=mode, planner=planner, row_filter=rf)
        torch.cuda.synchronize()
        ukeys = res.ukeys.cpu().numpy()
    counts = res.counts.cpu().numpy()
    sums = {c: t.cpu().numpy() for c, t in res.sums.items()}
    mins = {c: t.cpu().numpy() for c, t in res.mins.items()}
    maxs = {c: t.cpu().numpy() for c, t in res.maxs.items()}
    for c, dt in casts.items():
        if c in mins:
            mins[c] = mins[c].astype(dt)
        if c in maxs:
            maxs[c] = maxs[c].astype(dt)
    for c in cols:
        if c not in sums and "mean" in ops_map[c]:
            raise ExecError("internal: mean without sum lane")
    carry = ColumnCarry(ukeys, counts, sums, mins or None, maxs or None)
    out = p["out"]
    bufs[out + "#carry"] = carry
    if params.get("result", "dict") == "carry":
        bufs[out] = carry
    elif multi:
        bufs[out] = carry.to_dict_multi(cols, ops_map)
    else:
        bufs[out] = carry.to_dict_single(cols[0], ops_map[cols[0]])
    bufs[out + "#strategy"] = res.strategy
    bufs[out + "#groupindex"] = {"strategy": res.strategy, "backend": "cuda",
                                 "reason": "libnumfast_cuda %s" % res.strategy,
                                 "gi_ms": (time.perf_counter() - t0) * 1000, **res.probe}


def _valid_mask(bufs, *names):
    masks = [bufs[n + "#validity"] for n in names if n + "#validity" in bufs]
    if not masks:
        return None
    m = masks[0]
    for extra in masks[1:]:
        m = m & extra
    return m


def _sort_key_dev(k):
    if k.dtype == np.bool_ or (k.dtype.kind in "iu" and k.dtype.itemsize < 4):
        k = k.astype(np.int32)
    elif k.dtype == np.uint32:
        k = k.astype(np.int64)
    elif k.dtype == np.float32:
        k = k.astype(np.float64)
    elif k.dtype.kind not in "if" or k.dtype == np.uint64:
        raise ExecError("sort key dtype %s unsupported" % k.dtype)
    return _to_dev(k)


def sort_topk_device(key, desc, k, valid=None):
    """The first k rows of sort_perm_device([key], [desc], valid) as a DEVICE int32 tensor,
    by radix selection (only the kept rows are sorted)."""
    key = np.ascontiguousarray(np.asarray(key))
    vb = _bitmap_dev(valid) if valid is not None else None
    return dev.sort_topk(_sort_key_dev(key), k, bool(desc), vb)


def sort_perm_device(keys, desc, valid=None):
    """Stable sort permutation of host key arrays as a DEVICE int32 tensor (cpu.py:1154-1225:
    descending by key-group reversal, rows whose validity is false last)."""
    keys = [np.ascontiguousarray(np.asarray(k)) for k in keys]
    n = keys[0].size
    for k in keys:
        if k.size != n:
            raise ExecError("sort keys size mismatch %d != %d" % (k.size, n))
    if len(desc) != len(keys):
        raise ExecError("sort descending len %d != keys %d" % (len(desc), len(keys)))
    dkeys = [_sort_key_dev(k) for k in keys]
    vb = _bitmap_dev(valid) if valid is not None else None
    if len(dkeys) == 1:
        return dev.sort_perm(dkeys[0], bool(desc[0]), vb)
    return dev.lexsort_perm(dkeys, [bool(d) for d in desc], vb)


def _sort(p, bufs):
    keys = [bufs[i] for i in p["inputs"]]
    desc = p["params"].get("descending", [False] * len(keys))
    perm = sort_perm_device(keys, desc, _valid_mask(bufs, *p["inputs"]))
    bufs[p["out"]] = perm.cpu().numpy()


def _slice(p, bufs):
    """values[offset:offset+limit] (nodes.py:189-208; validity sliced alongside)."""
    a = np.asarray(bufs[p["inputs"][0]])
    off = int(p["params"].get("offset", 0))
    lim = p["params"].get("limit")
    end = a.size if lim is None else min(a.size, off + int(lim))
    bufs[p["out"]] = a[off:end] if off < a.size else a[:0]
    vv = bufs.get(p["inputs"][0] + "#validity")
    if vv is not None:
        vv = np.asarray(vv)
        bufs[p["out"] + "#validity"] = vv[off:end] if off < vv.size else np.zeros(0, dtype=bool)


def _gather(p, bufs):
    a = np.ascontiguousarray(np.asarray(bufs[p["inputs"][0]]))
    idx = np.ascontiguousarray(np.asarray(bufs[p["inputs"][1]]).astype(np.int32))
    if a.dtype.itemsize in (4, 8) and a.dtype.kind in "iuf":
        out = dev.gather(_to_dev(a), _to_dev(idx)).cpu().numpy()
    else:
        if idx.size and (idx.min() < 0 or idx.max() >= a.size):
            raise ExecError("gather index out of range")
        out = a[idx]
    bufs[p["out"]] = out
    vv = bufs.get(p["inputs"][0] + "#validity")
    if vv is not None:
        bufs[p["out"] + "#validity"] = np.asarray(vv)[idx]


def _unique_inverse(p, bufs):
    a = np.ascontiguousarray(np.asarray(bufs[p["inputs"][0]]))
    if a.dtype.kind == "b":
        a = a.astype(np.int32)
    if a.dtype.kind not in "iu":
        raise ExecError("unique_inverse needs int32/int64 keys")
    mv = bufs.get(p["inputs"][0] + "#validity")
    keys = a if mv is None else a[np.asarray(mv, dtype=bool)]
    if keys.dtype == np.int32 or (keys.size and keys.min() >= -2 ** 31 and keys.max() < 2 ** 31):
        r = dev.unique(_to_dev(keys.astype(np.int32)), with_inverse=True)
        uniq = r["uniq"].cpu().numpy().astype(a.dtype)
        inv_v = r["inverse"].cpu().numpy()
    else:
        # int64 keys beyond int32: the library's nf_unique_inverse_i64 (GPU radix sort).
        import ctypes
        k64 = np.ascontiguousarray(keys.astype(np.int64))
        n = k64.size
        uniq = np.empty(max(n, 1), dtype=np.int64)
        inv_v = np.empty(max(n, 1), dtype=np.int32)
        scratch = np.empty(max(n, 1), dtype=np.int64)
        vp = lambda x: ctypes.c_void_p(x.ctypes.data)
        ng = _lib.check("nf_unique_inverse_i64", _lib.load().nf_unique_inverse_i64(
            vp(k64), n, vp(uniq), vp(inv_v), vp(scratch), vp(scratch), vp(scratch), vp(scratch)))
        uniq = uniq[:ng].astype(a.dtype)
        inv_v = inv_v[:n]
    if mv is None:
        inv = inv_v
    else:
        inv = np.full(a.shape, -1, dtype=np.int32)
        inv[np.asarray(mv, dtype=bool)] = inv_v
    bufs[p["out"]] = np.ascontiguousarray(uniq)
    bufs[p["out"] + "#inv"] = np.ascontiguousarray(inv)
    bufs[p["out"] + "#ng"] = int(uniq.size)


def _filter(p, bufs):
    v = np.asarray(bufs[p["inputs"][0]])
    m = np.asarray(bufs[p["inputs"][1]], dtype=bool)
    if m.size != v.size:
        raise ExecError("filter mask size %d != %d" % (m.size, v.size))
    bufs[p["out"]] = np.ascontiguousarray(v[m])
    vv = bufs.get(p["inputs"][0] + "#validity")
    if vv is not None:
        bufs[p["out"] + "#validity"] = np.asarray(vv)[m]


def _group_count_distinct(p, bufs):
    """group_count_distinct (cpu.py:3705-3768): integer values and keys, rows with a NULL
    key or value dropped; result {key: nunique} (or the carry with result="carry")."""
    vname, kname = p["inputs"][0], p["inputs"][1]
    v, k = np.asarray(bufs[vname]), np.asarray(bufs[kname])
    if v.size != k.size:
        raise ExecError("group_count_distinct values/keys size mismatch %d != %d" % (v.size, k.size))
    if not np.issubdtype(k.dtype, np.integer) or not np.issubdtype(v.dtype, np.integer):
        raise ExecError("group_count_distinct needs integer keys and values")
    for name, a in ((kname, k), (vname, v)):
        if a.size and (a.min() < -2 ** 31 or a.max() > 2 ** 31 - 1):
            raise ExecError("group_count_distinct: %s outside int32" % name)
    km, vm = bufs.get(kname + "#validity"), bufs.get(vname + "#validity")
    uk, nu = dev.group_count_distinct(_to_dev(k.astype(np.int32)), _to_dev(v.astype(np.int32)),
                                      _bitmap_dev(km) if km is not None else None,
                                      _bitmap_dev(vm) if vm is not None else None)
    torch.cuda.synchronize()
    ukeys, nunique = uk.cpu().numpy(), nu.cpu().numpy()
    carry = ColumnCarry(ukeys, nunique, {"v": nunique})
    out = p["out"]
    bufs[out + "#carry"] = carry
    bufs[out] = carry if p["params"].get("result", "dict") == "carry" else carry.to_dict_flat("count")
    bufs[out + "#strategy"] = "sorted_dedup"


_HANDLERS = {
    "groupby_multi": _groupby_multi,
    "group_count_distinct": _group_count_distinct,
    "pack_keys": _pack_keys,
    "slice": _slice,
    "sort": _sort,
    "gather": _gather,
    "unique_inverse": _unique_inverse,
    "filter": _filter,
}


def execute(jobs, bufs=None):
    """Run a list of IR jobs; returns the buffer dict (like cpu_execute)."""
    bufs = {} if bufs is None else bufs
    for p in jobs:
        op = p["op"]
        if op == "series":
            _series(p["params"], p["out"], bufs)
            continue
        h = _HANDLERS.get(op)
        if h is None:
            raise ExecError("op %r is outside the group-by path" % op)
        h(p, bufs)
    return bufs
