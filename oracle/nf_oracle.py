"""CPU oracle for the group-by hot path -- TEST INFRASTRUCTURE ONLY.

A NumPy restatement of the reference executor's algorithm for this path.  It is the
checker: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
leg may import it.  The product (numfast_b200) never calls it.

Pinned: tests/test_oracle_golden.py checks every function here against golden vectors
produced by running the reference itself (tests/golden/make_golden.py).

Functions and the reference code they restate (paths relative to the reference
project root):
  philox_rows / fill_i32 / fill_f64   src/Drivers/CPU/_lib/rng.py:37-141
  valid_mask                          src/Drivers/CPU/_lib/cpu.py:1374-1382
  groupby_multi                       src/Drivers/CPU/_lib/cpu.py:3435-3563
                                        (compaction :3508-3511, dense_by_code
                                         groupindex.py:136-175, unique fallback
                                         groupindex.py:192-211, _fused_soa_by_code
                                         cpu.py:2344-2371, _group_minmax :2470-2601)
  stable_desc_idx / sort_perm         src/Drivers/CPU/_lib/cpu.py:1154-1225
  unique_inverse                      src/Drivers/CPU/_lib/cpu.py:4006-4040
  unique_first_count                  np.unique(return_index, return_counts) over the
                                        same sorted labelling (unique.rs:30-91)
"""

import numpy as np

_M64 = 0xFFFFFFFFFFFFFFFF


# ---------------------------------------------------------------- RNG (rng.py:37-141)

def _splitmix64_out(state):
    state = (state + 0x9E3779B97F4A7C15) & _M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return (z ^ (z >> 31)) & _M64


def derive_key(seed, stream):
    st = ((int(seed) & _M64) + 0x9E3779B97F4A7C15 + ((int(stream) & _M64) * 0xBF58476D1CE4E5B9 & _M64)) & _M64
    k = _splitmix64_out(st)
    return k & 0xFFFFFFFF, (k >> 32) & 0xFFFFFFFF


def philox_rows(n, seed, stream, offset=0):
    """(r0, r1, r2, r3) uint32 arrays for lanes offset..offset+n-1 (Philox4x32-10)."""
    g = (np.arange(n, dtype=np.uint64) + np.uint64(int(offset) & _M64))
    a0 = (g & np.uint64(0xFFFFFFFF)).astype(np.uint64)
    a1 = (g >> np.uint64(32)).astype(np.uint64)
    s = int(stream) & _M64
    a2 = np.full(n, (s & 0xFFFFFFFF) ^ 0xC0FFEE00, dtype=np.uint64)
    a3 = np.full(n, ((s >> 32) & 0xFFFFFFFF) ^ 0x9E3779B9, dtype=np.uint64)
    k0, k1 = derive_key(seed, s)
    m32 = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = a0 * np.uint64(0xD2511F53)
        p1 = a2 * np.uint64(0xCD9E8D57)
        hi0, lo0 = p0 >> np.uint64(32), p0 & m32
        hi1, lo1 = p1 >> np.uint64(32), p1 & m32
        a0, a1, a2, a3 = hi1 ^ a1 ^ np.uint64(k0), lo1, hi0 ^ a3 ^ np.uint64(k1), lo0
        k0 = (k0 + 0x9E3779B9) & 0xFFFFFFFF
        k1 = (k1 + 0xBB67AE85) & 0xFFFFFFFF
    return tuple(x.astype(np.uint32) for x in (a0, a1, a2, a3))


def fill_i32(n, seed, stream=0, offset=0, lo=0, hi=100):
    width = int(hi) - int(lo)
    if n == 0:
        return np.empty(0, dtype=np.int32)
    if width == 1:
        return np.full(n, lo, dtype=np.int32)
    r0 = philox_rows(n, seed, stream, offset)[0]
    v = ((r0.astype(np.uint64) * np.uint64(width)) >> np.uint64(32)).astype(np.int64)
    return (v + np.int64(lo)).astype(np.int32)


def fill_f64(n, seed, stream=0, offset=0, lo=0.0, hi=1.0):
    if n == 0:
        return np.empty(0, dtype=np.float64)
    r0, r1, _, _ = philox_rows(n, seed, stream, offset)
    u = ((r0 >> np.uint32(5)).astype(np.uint64) << np.uint64(26)) | (r1 >> np.uint32(6)).astype(np.uint64)
    f = u.astype(np.float64) / float(2 ** 53)
    return float(lo) + f * (float(hi) - float(lo))


# ---------------------------------------------------------------- group-by

def valid_mask(*masks):
    """AND of the validity masks present (None = all valid)."""
    ms = [np.asarray(m, dtype=bool) for m in masks if m is not None]
    if not ms:
        return None
    out = ms[0].copy()
    for m in ms[1:]:
        out &= m
    return out


def _group_index(k):
    """ukeys ascending + a code per row.  Dense keys take the by-code route
    (bincount over the key itself), others the unique/inverse route; both label
    groups identically and accumulate in row order."""
    k = np.asarray(k)
    if k.size == 0:
        return np.zeros(0, dtype=np.int64), None, 0, None
    kmin, kmax = int(k.min()), int(k.max())
    if kmin >= 0 and kmax + 1 <= max(4 * k.size, 1 << 16):
        k64 = k.astype(np.int64)
        m = kmax + 1
        counts_m = np.bincount(k64, minlength=m)
        ukeys = np.flatnonzero(counts_m).astype(np.int64)
        return ukeys, k64, m, counts_m
    ukeys, inv = np.unique(k, return_inverse=True)
    return ukeys.astype(np.int64), inv.astype(np.int64), ukeys.size, None


def groupby_multi(keys, values, ops_map, validity=None):
    """Reference groupby_multi over host arrays.

    keys: int array; values: {col: array}; ops_map: {col: ops}; validity: {name: mask}
    with name "__key__" for the key column.  Returns a dict with ukeys, counts and
    sums/mins/maxs per column (dtypes as the reference's ColumnCarry)."""
    validity = validity or {}
    cols = list(values)
    m = valid_mask(validity.get("__key__"), *[validity.get(c) for c in cols])
    k = np.asarray(keys)
    vs = {c: np.asarray(values[c]) for c in cols}
    if m is not None:
        keep = np.nonzero(m)[0]
        k = k[keep]
        vs = {c: v[keep] for c, v in vs.items()}
    ukeys, code, mm, counts_m = _group_index(k)
    ng = ukeys.size
    pos = ukeys if counts_m is not None else None
    if ng == 0:
        counts = np.zeros(0, dtype=np.int64)
    elif counts_m is not None:
        counts = counts_m[pos].astype(np.int64)
    else:
        counts = np.bincount(code, minlength=ng).astype(np.int64)
    out = {"ukeys": ukeys, "counts": counts, "sums": {}, "mins": {}, "maxs": {}}
    for c in cols:
        v = vs[c]
        ops = ops_map[c]
        if "sum" in ops or "mean" in ops:
            if ng == 0:
                s = np.zeros(0, dtype=np.int64 if v.dtype.kind in "iub" else np.float64)
            elif v.dtype.kind in "iub":
                s = np.bincount(code, weights=v.astype(np.int64), minlength=mm)
                s = (s[pos] if pos is not None else s).astype(np.int64)
            else:
                s = np.bincount(code, weights=v.astype(np.float64), minlength=mm)
                s = s[pos] if pos is not None else s
            out["sums"][c] = s
        for kind in ("min", "max"):
            if kind not in ops:
                continue
            if ng == 0:
                out[kind + "s"][c] = np.zeros(0, dtype=v.dtype)
                continue
            if v.dtype.kind in "iu":
                info = np.iinfo(v.dtype)
                fill = info.max if kind == "min" else info.min
            else:
                fill = np.inf if kind == "min" else -np.inf
            dense = np.full(mm, fill, dtype=v.dtype)
            (np.minimum if kind == "min" else np.maximum).at(dense, code, v)
            out[kind + "s"][c] = dense[pos] if pos is not None else dense
    return out


# ---------------------------------------------------------------- sort (cpu.py:1154-1225)

def stable_desc_idx(k):
    asc = np.argsort(k, kind="stable")
    if asc.size == 0:
        return asc
    sk = k[asc]
    ch = np.empty(sk.shape, dtype=bool)
    ch[0] = True
    if sk.size > 1:
        ch[1:] = sk[1:] != sk[:-1]
    grp = np.cumsum(ch)
    rev = grp.max(initial=0) - grp
    return asc[np.argsort(rev, kind="stable")]


def sort_perm(cols, descending, valid=None):
    """Stable lexicographic permutation; invalid rows last in input order."""
    cols = [np.asarray(c) for c in cols]
    if isinstance(descending, bool):
        descending = [descending] * len(cols)
    n = cols[0].size
    if valid is not None:
        vm = np.asarray(valid, dtype=bool)
        vpos = np.flatnonzero(vm)
        ipos = np.flatnonzero(~vm)
    else:
        vpos = np.arange(n)
        ipos = np.zeros(0, dtype=np.int64)
    idx = np.arange(vpos.size)
    for c, desc in zip(reversed(cols), reversed(list(descending))):
        k = c[vpos][idx] if vpos.size else c[:0]
        step = stable_desc_idx(k) if desc else np.argsort(k, kind="stable")
        idx = idx[step]
    perm = np.empty(n, dtype=np.int32)
    perm[:vpos.size] = vpos[idx]
    perm[vpos.size:] = ipos
    return perm


# ---------------------------------------------------------------- unique (cpu.py:4006-4040)

def unique_inverse(keys, valid=None):
    keys = np.asarray(keys)
    if valid is None:
        u, inv = np.unique(keys, return_inverse=True)
        return u, inv.astype(np.int32)
    m = np.asarray(valid, dtype=bool)
    u, iv = np.unique(keys[m], return_inverse=True)
    inv = np.full(keys.shape, -1, dtype=np.int32)
    inv[m] = iv.astype(np.int32)
    return u, inv


def unique_first_count(keys):
    u, first, counts = np.unique(np.asarray(keys), return_index=True, return_counts=True)
    return u, first.astype(np.int32), counts.astype(np.int64)


# ---------------------------------------------------------------- config-1 chain

def chain_group_sort(key, v, ops=("sum", "count"), sort_field="sum", desc=True):
    """group(key, {v: ops}).sort("v.<sort_field>", desc) -> dict of output columns."""
    g = groupby_multi(key, {"v": v}, {"v": ops})
    cols = {"key": g["ukeys"]}
    for op in ops:
        if op == "count":
            cols["v.count"] = g["counts"]
        elif op == "sum":
            cols["v.sum"] = g["sums"]["v"]
        elif op == "mean":
            cols["v.mean"] = g["sums"]["v"].astype(np.float64) / g["counts"]
        elif op == "min":
            cols["v.min"] = g["mins"]["v"]
        elif op == "max":
            cols["v.max"] = g["maxs"]["v"]
    perm = sort_perm([cols["v." + sort_field]], [desc])
    return {k: c[perm] for k, c in cols.items()}


# ---------------------------------------------------------------- batched sum+count

def batch_sum_count(keys, values, row_offsets, key_valid=None, value_valid=None):
    """Per-query groupby_multi with ops ("sum", "count") over row ranges of one
    concatenated key/value column (each query = one executor groupby_multi node,
    cpu.py:3435-3704).  Returns a list of (ukeys, sums, counts) per query."""
    ro = np.asarray(row_offsets, dtype=np.int64)
    out = []
    for q in range(ro.size - 1):
        a, b = int(ro[q]), int(ro[q + 1])
        val = {}
        if key_valid is not None:
            val["__key__"] = np.asarray(key_valid[a:b], dtype=bool)
        if value_valid is not None:
            val["v"] = np.asarray(value_valid[a:b], dtype=bool)
        r = groupby_multi(np.asarray(keys[a:b]), {"v": np.asarray(values[a:b])}, {"v": ("sum", "count")},
                          val or None)
        out.append((np.asarray(r["ukeys"], dtype=np.int64), np.asarray(r["sums"]["v"], dtype=np.int64),
                    np.asarray(r["counts"], dtype=np.int64)))
    return out


# ---------------------------------------------------------------- grouped count distinct

def group_count_distinct(keys, values, valid=None):
    """(ukeys, nunique) over rows where `valid` holds: lexsort by (key, value), then group
    bounds and value transitions (cpu.py:2647-2700, _count_distinct_sorted_dedup)."""
    k = np.asarray(keys).astype(np.int64)
    v = np.asarray(values).astype(np.int64)
    if valid is not None:
        keep = np.asarray(valid, dtype=bool)
        k, v = k[keep], v[keep]
    if k.size == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    perm = np.lexsort((v, k))
    sk, sv = k[perm], v[perm]
    key_head = np.ones(sk.size, bool)
    key_head[1:] = sk[1:] != sk[:-1]
    pair_head = key_head.copy()
    pair_head[1:] |= sv[1:] != sv[:-1]
    starts = np.flatnonzero(key_head)
    nunique = np.add.reduceat(pair_head.astype(np.int64), starts)
    return sk[starts], nunique


# ---------------------------------------------------------------- composite (tuple) keys

def composite_order(cols):
    """Row order in which composite_tuple_index groups tuple keys of int32 columns
    (groupindex.py:520-566): 2 columns by the int64 (c0 << 32) | uint32(c1); 3 by c2, then
    that pack; 4 by the pack of (c0, c1), then the pack of (c2, c3); otherwise plainly
    lexicographic with c0 primary."""
    cols = [np.asarray(c) for c in cols]
    nc = len(cols)

    def pack(x, y):
        return (x.astype(np.int64) << 32) | (y.astype(np.int64) & 0xFFFFFFFF)

    if nc == 1:
        return np.lexsort((cols[0],))
    if nc == 2:
        return np.lexsort((pack(cols[0], cols[1]),))
    if nc == 3:
        return np.lexsort((pack(cols[0], cols[1]), cols[2]))
    if nc == 4:
        return np.lexsort((pack(cols[2], cols[3]), pack(cols[0], cols[1])))
    return np.lexsort(tuple(cols[::-1]))


def composite_groupby_sum_count(cols, values, valid=None):
    """(ukeys (ng x nc), counts, sums) of groupby_multi (sum, count) over tuple keys, rows
    with any NULL dropped first (cpu.py:3458-3500)."""
    cols = [np.asarray(c) for c in cols]
    v = np.asarray(values).astype(np.int64)
    if valid is not None:
        keep = np.asarray(valid, dtype=bool)
        cols = [c[keep] for c in cols]
        v = v[keep]
    n = v.size
    if n == 0:
        return np.zeros((0, len(cols)), np.int64), np.zeros(0, np.int64), np.zeros(0, np.int64)
    order = composite_order(cols)
    sc = [c[order] for c in cols]
    diff = np.zeros(n, bool)
    diff[0] = True
    for c in sc:
        diff[1:] |= c[1:] != c[:-1]
    starts = np.flatnonzero(diff)
    ukeys = np.stack([c[starts].astype(np.int64) for c in sc], axis=1)
    gid = np.cumsum(diff) - 1
    counts = np.bincount(gid, minlength=starts.size).astype(np.int64)
    sums = np.bincount(gid, weights=v[order], minlength=starts.size).astype(np.int64)
    return ukeys, counts, sums
