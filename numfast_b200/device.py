"""Device-resident group-by / sort / unique over torch CUDA tensors.

torch provides device memory and streams only; every computation is a
libnumfast_cuda kernel reached through the C ABI (nfc_* entry points).
"""

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib

_DTYPES = {torch.int32: _lib.I32, torch.int64: _lib.I64, torch.float64: _lib.F64}
_OPS_BITS = {"sum": _lib.AGG_SUM, "mean": _lib.AGG_SUM, "min": _lib.AGG_MIN, "max": _lib.AGG_MAX}
_STRATEGIES = {v: k for k, v in _lib.STRATEGY_NAMES.items()}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream_handle(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def pack_validity(mask):
    """bool/uint8 byte mask (numpy or torch) -> LSB-first bitmap (Arrow layout)."""
    if isinstance(mask, torch.Tensor):
        mask = mask.cpu().numpy()
    return np.packbits(np.asarray(mask, dtype=bool), bitorder="little")


@dataclass
class DeviceColumn:
    """One value column: values (int32/int64/float64 CUDA tensor), optional LSB validity
    bitmap (uint8 CUDA tensor) and the aggregates requested for it."""

    name: str
    values: torch.Tensor
    ops: tuple = ("sum",)
    validity: torch.Tensor = None


@dataclass
class DeviceCarry:
    """Columnar group-by result on the device (same fields as ColumnCarry)."""

    ukeys: torch.Tensor
    counts: torch.Tensor
    sums: dict = field(default_factory=dict)
    mins: dict = field(default_factory=dict)
    maxs: dict = field(default_factory=dict)
    strategy: str = ""
    probe: dict = field(default_factory=dict)
    key_columns: list = field(default_factory=list)  # composite keys: one int32 tensor per key column

    @property
    def ngroups(self):
        return int(self.ukeys.shape[0])


class GroupbyBuffers:
    """Reusable output buffers for repeated group-by calls of the same shape."""

    def __init__(self, cap, cols, device):
        self.cap = int(cap)
        self.ukeys = torch.empty(self.cap, dtype=torch.int64, device=device)
        self.counts = torch.empty(self.cap, dtype=torch.int64, device=device)
        self.sum, self.min, self.max = {}, {}, {}
        for c in cols:
            ops = set(c.ops)
            sdt = torch.float64 if c.values.dtype == torch.float64 else torch.int64
            if ops & {"sum", "mean"}:
                self.sum[c.name] = torch.empty(self.cap, dtype=sdt, device=device)
            if "min" in ops:
                self.min[c.name] = torch.empty(self.cap, dtype=c.values.dtype, device=device)
            if "max" in ops:
                self.max[c.name] = torch.empty(self.cap, dtype=c.values.dtype, device=device)


def groupby(keys, cols, key_validity=None, strategy="auto", stream=None, buffers=None, timing=False,
            distinct_hint=0, planner_mode=None, planner=None, row_filter=None):
    """Group-by with validity on the device.

    keys: int32 CUDA tensor.  cols: list of DeviceColumn (at most 4 per call; more are
    processed in batches of 4 over the same grouping).  A row counts only if its key and
    every value column are valid (cpu.py:1374-1382, :3508-3511) and, when row_filter (an LSB
    bitmap) is given, its filter bit is set -- a filter fused into the group-by instead of a
    compaction of every column before it.  Returns DeviceCarry with
    ascending int64 ukeys, int64 counts, int64 (integer columns) / float64 sums and
    min/max in the value dtype.
    """
    lib = _lib.load()
    if keys.dtype != torch.int32 or not keys.is_cuda:
        raise TypeError("keys must be an int32 CUDA tensor")
    keys = keys.contiguous()
    n = int(keys.numel())
    cols = list(cols)
    if len(cols) > _lib.MAX_COLS:
        return _groupby_batched(keys, cols, key_validity, strategy, stream, row_filter)
    if buffers is None:
        buffers = GroupbyBuffers(max(n, 1), cols, keys.device)
    vc = (_lib.ValueCol * max(len(cols), 1))()
    keep = [keys]
    for i, c in enumerate(cols):
        v = c.values.contiguous()
        if v.dtype not in _DTYPES or not v.is_cuda or int(v.numel()) != n:
            raise TypeError("column %r must be an int32/int64/float64 CUDA tensor of %d rows" % (c.name, n))
        keep.append(v)
        bits = 0
        for op in c.ops:
            if op not in _OPS_BITS and op != "count":
                raise ValueError("unknown aggregate %r" % op)
            bits |= _OPS_BITS.get(op, 0)
        vc[i].dtype = _DTYPES[v.dtype]
        vc[i].aggs = bits
        vc[i].data = v.data_ptr()
        vc[i].validity = c.validity.data_ptr() if c.validity is not None else None
        vc[i].sum_out = buffers.sum[c.name].data_ptr() if c.name in buffers.sum else None
        vc[i].min_out = buffers.min[c.name].data_ptr() if c.name in buffers.min else None
        vc[i].max_out = buffers.max[c.name].data_ptr() if c.name in buffers.max else None
    args = _lib.GroupbyArgs()
    args.n = n
    args.keys = keys.data_ptr() if n else None
    args.key_validity = key_validity.data_ptr() if key_validity is not None else None
    args.ncols = len(cols)
    args.cols = vc
    args.out_cap = buffers.cap
    args.ukeys_out = buffers.ukeys.data_ptr()
    args.counts_out = buffers.counts.data_ptr()
    # A fused upstream filter: one more bitmap ANDed into the probe's validity.
    args.row_filter = row_filter.data_ptr() if row_filter is not None else None
    stats = _lib.GroupbyStats()
    stats.timing = 1 if timing else 0
    stats.distinct_hint = int(distinct_hint)
    strat = _STRATEGIES[strategy] if isinstance(strategy, str) else int(strategy)
    if planner_mode is not None and strat == _lib.STRAT_AUTO:
        # The planner picks the strategy (fixed: the reference's rule; learned: sketch + MLP).
        mode = {"auto": _lib.PLANNER_AUTO, "fixed": _lib.PLANNER_FIXED, "learned": _lib.PLANNER_LEARNED}[planner_mode]
        if mode == _lib.PLANNER_LEARNED and planner is None:
            raise ValueError("planner_mode='learned' needs a planner (numfast_b200.planner.LearnedPlanner)")
        ng = _lib.check("nfc_groupby_planned", lib.nfc_groupby_planned(
            ctypes.byref(args), mode, planner.handle if planner is not None else None, _stream_handle(stream),
            ctypes.byref(stats)))
    else:
        ng = _lib.check("nfc_groupby", lib.nfc_groupby(ctypes.byref(args), strat, _stream_handle(stream),
                                                       ctypes.byref(stats)))
    ng = int(ng)
    out = DeviceCarry(buffers.ukeys[:ng], buffers.counts[:ng],
                      {k: t[:ng] for k, t in buffers.sum.items()},
                      {k: t[:ng] for k, t in buffers.min.items()},
                      {k: t[:ng] for k, t in buffers.max.items()},
                      strategy=_lib.STRATEGY_NAMES.get(stats.strategy, str(stats.strategy)),
                      probe={"n_valid": stats.probe.n_valid, "kmin": stats.probe.kmin,
                             "kmax": stats.probe.kmax, "sorted": bool(stats.probe.sorted),
                             "buckets": stats.buckets, "launches": stats.launches,
                             "overflowed": int(stats.overflowed),
                             "stage_ms": [stats.stage_ms[i] for i in range(stats.nstages)]})
    return out


def _groupby_batched(keys, cols, key_validity, strategy, stream, row_filter=None):
    # Validity of EVERY column gates every row, so each batch carries the other
    # columns' bitmaps through key_validity-style AND: fold them into the key bitmap.
    bms = [c.validity for c in cols if c.validity is not None]
    if key_validity is not None:
        bms.append(key_validity)
    if row_filter is not None:
        bms.append(row_filter)
    kv = None
    if bms:
        kv = bms[0].clone()
        for b in bms[1:]:
            kv &= b
    result = None
    for i in range(0, len(cols), _lib.MAX_COLS):
        part = [DeviceColumn(c.name, c.values, c.ops, None) for c in cols[i:i + _lib.MAX_COLS]]
        r = groupby(keys, part, kv, strategy, stream)
        if result is None:
            result = r
        else:
            result.sums.update(r.sums)
            result.mins.update(r.mins)
            result.maxs.update(r.maxs)
    return result


def sort_perm(keys, descending=False, validity=None, stream=None):
    """Stable argsort permutation (int32) of one key column on the device."""
    lib = _lib.load()
    dt = _DTYPES.get(keys.dtype)
    if dt is None or not keys.is_cuda:
        raise TypeError("sort keys must be an int32/int64/float64 CUDA tensor")
    keys = keys.contiguous()
    n = int(keys.numel())
    perm = torch.empty(n, dtype=torch.int32, device=keys.device)
    if n:
        _lib.check("nfc_sort_perm", lib.nfc_sort_perm(dt, keys.data_ptr(),
                                                      validity.data_ptr() if validity is not None else None,
                                                      n, 1 if descending else 0, perm.data_ptr(),
                                                      _stream_handle(stream)))
    return perm


def sort_topk(keys, k, descending=False, validity=None, stream=None):
    """The first k entries of sort_perm(keys, descending, validity): radix selection of the
    k-th key and a sort of only the rows it keeps (int32 device tensor of k)."""
    lib = _lib.load()
    dt = _DTYPES.get(keys.dtype)
    if dt is None or not keys.is_cuda:
        raise TypeError("sort keys must be an int32/int64/float64 CUDA tensor")
    keys = keys.contiguous()
    n = int(keys.numel())
    k = int(k)
    if k < 0 or k > n:
        raise ValueError("topk: k must be in [0, %d], got %d" % (n, k))
    perm = torch.empty(k, dtype=torch.int32, device=keys.device)
    if k:
        _lib.check("nfc_sort_topk", lib.nfc_sort_topk(dt, keys.data_ptr(),
                                                      validity.data_ptr() if validity is not None else None,
                                                      n, 1 if descending else 0, k, perm.data_ptr(),
                                                      _stream_handle(stream)))
    return perm


def lexsort_perm(cols, descending, validity=None, stream=None):
    """Lexicographic stable permutation: successive stable passes from the LAST key
    (cpu.py:1174-1225).  Invalid rows (validity bit 0) go last in input order."""
    if isinstance(descending, bool):
        descending = [descending] * len(cols)
    n = int(cols[0].numel())
    dev = cols[0].device
    if validity is not None:
        shifts = torch.arange(8, device=dev, dtype=torch.uint8)
        vbits = ((validity.to(dev)[:, None] >> shifts) & 1).flatten()[:n].bool()
        vpos = torch.nonzero(vbits).flatten().to(torch.int32)
        ipos = torch.nonzero(~vbits).flatten().to(torch.int32)
    else:
        vpos, ipos = None, None
    idx = None
    for c, desc in zip(reversed(cols), reversed(list(descending))):
        k = c if vpos is None else gather(c, vpos)
        if idx is not None:
            k = gather(k, idx)
        step = sort_perm(k, bool(desc), stream=stream)
        idx = step if idx is None else gather(idx, step)
    if vpos is None:
        return idx
    return torch.cat([gather(vpos, idx), ipos])


def gather(values, idx, stream=None):
    """values[idx] on the device (idx int32); out-of-range indices raise."""
    lib = _lib.load()
    values = values.contiguous()
    idx = idx.contiguous()
    out = torch.empty(int(idx.numel()), dtype=values.dtype, device=values.device)
    if idx.numel():
        _lib.check("nfc_gather", lib.nfc_gather(values.element_size(), values.data_ptr(), int(values.numel()),
                                                idx.data_ptr(), int(idx.numel()), out.data_ptr(),
                                                _stream_handle(stream)))
    return out


def unique(keys, with_inverse=False, stream=None):
    """Sorted unique int32 keys with first-occurrence row and count (and inverse)."""
    lib = _lib.load()
    keys = keys.contiguous()
    n = int(keys.numel())
    dev = keys.device
    uniq = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    first = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    counts = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    inv = torch.empty(max(n, 1), dtype=torch.int32, device=dev) if with_inverse else None
    ng = 0
    if n:
        ng = int(_lib.check("nfc_unique", lib.nfc_unique(keys.data_ptr(), n, uniq.data_ptr(), first.data_ptr(),
                                                         counts.data_ptr(),
                                                         inv.data_ptr() if inv is not None else None,
                                                         _stream_handle(stream))))
    res = {"uniq": uniq[:ng], "first": first[:ng], "counts": counts[:ng], "ng": ng}
    if with_inverse:
        res["inverse"] = inv[:n]
    return res


# ---- seeded synthetic inputs (Philox lanes, bit-exact with the reference RNG) ----

def group_count_distinct(keys, values, key_validity=None, value_validity=None, stream=None):
    """Per key, the number of distinct values among rows with valid key and value
    (cpu.py:3705-3768).  Returns (ukeys int64 ascending, nunique int64) device tensors."""
    lib = _lib.load()
    if keys.dtype != torch.int32 or values.dtype != torch.int32:
        raise TypeError("group_count_distinct: keys and values must be int32 CUDA tensors")
    keys, values = keys.contiguous(), values.contiguous()
    n = int(keys.numel())
    if int(values.numel()) != n:
        raise ValueError("group_count_distinct: values/keys size mismatch %d != %d" % (values.numel(), n))
    uk = torch.empty(max(n, 1), dtype=torch.int64, device=keys.device)
    nu = torch.empty(max(n, 1), dtype=torch.int64, device=keys.device)
    ng = _lib.check("nfc_group_count_distinct", lib.nfc_group_count_distinct(
        keys.data_ptr() if n else None, key_validity.data_ptr() if key_validity is not None else None,
        values.data_ptr() if n else None, value_validity.data_ptr() if value_validity is not None else None,
        n, max(n, 1), uk.data_ptr(), nu.data_ptr(), _stream_handle(stream)))
    return uk[:ng], nu[:ng]


SIGNED = 0x80000000


def composite_codes(a, b, a_signed=True, b_signed=False, validity=None, stream=None):
    """Dense int32 codes of (a, b) pairs ranked by a (signed or unsigned) then b (signed or
    unsigned); rows not valid in `validity` get -1.  Returns (codes, ua, ub): ua[c], ub[c]
    is the pair of code c."""
    lib = _lib.load()
    if a.dtype != torch.int32 or b.dtype != torch.int32:
        raise TypeError("composite_codes: int32 key columns")
    a, b = a.contiguous(), b.contiguous()
    n = int(a.numel())
    codes = torch.empty(max(n, 1), dtype=torch.int32, device=a.device)
    ua = torch.empty(max(n, 1), dtype=torch.int32, device=a.device)
    ub = torch.empty(max(n, 1), dtype=torch.int32, device=a.device)
    ng = _lib.check("nfc_composite_codes", lib.nfc_composite_codes(
        a.data_ptr() if n else None, SIGNED if a_signed else 0, b.data_ptr() if n else None,
        SIGNED if b_signed else 0, validity.data_ptr() if validity is not None else None, n,
        codes.data_ptr(), ua.data_ptr(), ub.data_ptr(), _stream_handle(stream)))
    return codes[:n], ua[:ng], ub[:ng]


def composite_keys(keys, validity=None):
    """Codes for tuple keys of 1+ int32 columns, in the order the reference's
    composite_tuple_index groups them (groupindex.py:520-639): two columns by (k0 signed,
    k1 unsigned); three by k2, then (k0, k1 unsigned); four by (k0, k1 unsigned), then
    (k2, k3 unsigned); more by plain lexicographic order.  Returns (codes, decode) where
    decode(code tensor) gives one int32 tensor per key column."""
    nc = len(keys)
    if nc == 1:
        return keys[0], lambda c: [c.to(torch.int32)]

    def fold(a, af, b, bf):
        c, ua, ub = composite_codes(a, b, af, bf, validity)
        return c, ua.long(), ub.long()

    if nc == 2:
        c, u0, u1 = fold(keys[0], True, keys[1], False)
        return c, lambda x: [u0[x.long()].int(), u1[x.long()].int()]
    if nc == 3:
        c01, u0, u1 = fold(keys[0], True, keys[1], False)
        c, u2, u01 = fold(keys[2], True, c01, False)
        return c, lambda x: [u0[u01[x.long()]].int(), u1[u01[x.long()]].int(), u2[x.long()].int()]
    if nc == 4:
        c01, u0, u1 = fold(keys[0], True, keys[1], False)
        c23, u2, u3 = fold(keys[2], True, keys[3], False)
        c, x01, x23 = fold(c01, False, c23, False)
        return c, lambda x: [u0[x01[x.long()]].int(), u1[x01[x.long()]].int(), u2[x23[x.long()]].int(),
                             u3[x23[x.long()]].int()]
    # Plain lexicographic: fold from the left, every column signed.
    c, u0, u1 = fold(keys[0], True, keys[1], True)
    decoders = [lambda x, u=u0: u[x], lambda x, u=u1: u[x]]
    for k in keys[2:]:
        prev = decoders
        c, uc, uk = fold(c, False, k, True)
        decoders = [lambda x, f=f, uc=uc: f(uc[x]) for f in prev] + [lambda x, uk=uk: uk[x]]
    return c, lambda x: [f(x.long()).int() for f in decoders]


_SIGNED, _UNSIGNED = 0x80000000, 0


def composite_order_plan(nc):
    """(column, flip) in significance order: the lexicographic order that the reference's
    composite_tuple_index (groupindex.py:520-639) gives tuples of nc int32 columns."""
    if nc == 2:
        return [(0, _SIGNED), (1, _UNSIGNED)]
    if nc == 3:
        return [(2, _SIGNED), (0, _SIGNED), (1, _UNSIGNED)]
    if nc == 4:
        return [(0, _SIGNED), (1, _UNSIGNED), (2, _SIGNED), (3, _UNSIGNED)]
    return [(i, _SIGNED) for i in range(nc)]


def _u32_array(vals):
    return (ctypes.c_uint32 * len(vals))(*[int(v) & 0xFFFFFFFF for v in vals])


def key_bits_layout(keys, flips, validity=None, stream=None):
    """(mins, widths) of a bit-packed tuple key over `keys` (int32 CUDA tensors, most
    significant first), or None when the flipped ranges need more than 31 bits."""
    lib = _lib.load()
    nc = len(keys)
    if nc > _lib.MAX_KEY_COLS:
        return None
    n = int(keys[0].numel())
    ptrs = (ctypes.c_void_p * nc)(*[k.data_ptr() for k in keys])
    mins, maxs = (ctypes.c_uint32 * nc)(), (ctypes.c_uint32 * nc)()
    nvalid = _lib.check("nfc_key_ranges", lib.nfc_key_ranges(
        ptrs, _u32_array(flips), nc, _ptr(validity), n, mins, maxs, _stream_handle(stream)))
    if nvalid == 0:
        return [0] * nc, [0] * nc
    widths = [int(maxs[c] - mins[c]).bit_length() for c in range(nc)]
    if sum(widths) > 31:
        return None
    return [int(mins[c]) for c in range(nc)], widths


def pack_key_bits(keys, flips, mins, widths, stream=None):
    lib = _lib.load()
    nc = len(keys)
    n = int(keys[0].numel())
    out = torch.empty(n, dtype=torch.int32, device=keys[0].device)
    ptrs = (ctypes.c_void_p * nc)(*[k.data_ptr() for k in keys])
    _lib.check("nfc_pack_key_bits", lib.nfc_pack_key_bits(
        ptrs, _u32_array(flips), _u32_array(mins), (ctypes.c_int32 * nc)(*widths), nc, n,
        _ptr(out if n else None), _stream_handle(stream)))
    return out


def unpack_key_bits(codes, flips, mins, widths, stream=None):
    """int64 codes -> one int32 tensor per key column (inverse of pack_key_bits)."""
    lib = _lib.load()
    nc = len(flips)
    ng = int(codes.numel())
    outs = [torch.empty(ng, dtype=torch.int32, device=codes.device) for _ in range(nc)]
    codes = codes.contiguous()
    ptrs = (ctypes.c_void_p * nc)(*[o.data_ptr() if ng else 0 for o in outs])
    _lib.check("nfc_unpack_key_bits", lib.nfc_unpack_key_bits(
        _ptr(codes if ng else None), ng, _u32_array(flips), _u32_array(mins), (ctypes.c_int32 * nc)(*widths), nc,
        ptrs, _stream_handle(stream)))
    return outs


def groupby_composite(keys, cols, key_validity=None, **kw):
    """group-by over tuple keys (1+ int32 columns) in the reference's composite order,
    carrying the key columns of each group (DeviceCarry.key_columns).  When the columns'
    ranges fit in 31 bits the tuple becomes one bit-packed int32 key (no sort); otherwise
    the tuples become dense codes by pairwise sorted folds."""
    keys = list(keys)
    if len(keys) >= 2:
        plan = composite_order_plan(len(keys))
        ordered = [keys[c].contiguous() for c, _ in plan]
        flips = [f for _, f in plan]
        lay = key_bits_layout(ordered, flips, key_validity, kw.get("stream"))
        if lay is not None:
            mins, widths = lay
            codes = pack_key_bits(ordered, flips, mins, widths, kw.get("stream"))
            r = groupby(codes, cols, key_validity, **kw)
            cols_sig = unpack_key_bits(r.ukeys, flips, mins, widths, kw.get("stream"))
            r.key_columns = [None] * len(keys)
            for (c, _), t in zip(plan, cols_sig):
                r.key_columns[c] = t
            return r
    codes, decode = composite_keys(keys, key_validity)
    # A code is -1 exactly where the key bitmap marks the row null, so that bitmap is
    # also the validity of the codes.
    r = groupby(codes.contiguous(), cols, key_validity, **kw)
    r.key_columns = decode(r.ukeys)
    return r


def pack_validity_dev(mask):
    """LSB bitmap (uint8) of a bool CUDA tensor."""
    n = int(mask.numel())
    pad = (-n) % 8
    m = torch.cat([mask, mask.new_zeros(pad)]) if pad else mask
    w = (2 ** torch.arange(8, device=mask.device, dtype=torch.int32)).view(1, 8)
    return (m.view(-1, 8).to(torch.int32) * w).sum(1).to(torch.uint8)


def rng_fill_i32(n, seed, stream_id=0, lo=0, hi=100, offset=0, device="cuda"):
    lib = _lib.load()
    out = torch.empty(n, dtype=torch.int32, device=device)
    _lib.check("nfc_rng_fill_i32", lib.nfc_rng_fill_i32(n, seed, stream_id, offset, lo, hi,
                                                        out.data_ptr() if n else None, _stream_handle(None)))
    return out


def rng_fill_f64(n, seed, stream_id=0, lo=0.0, hi=1.0, offset=0, device="cuda"):
    lib = _lib.load()
    out = torch.empty(n, dtype=torch.float64, device=device)
    _lib.check("nfc_rng_fill_f64", lib.nfc_rng_fill_f64(n, seed, stream_id, offset, lo, hi,
                                                        out.data_ptr() if n else None, _stream_handle(None)))
    return out


def gen_lognormal(n, seed, stream_a, stream_b, mu, sigma, device="cuda"):
    lib = _lib.load()
    out = torch.empty(n, dtype=torch.float64, device=device)
    _lib.check("nfc_gen_lognormal", lib.nfc_gen_lognormal(n, seed, stream_a, stream_b, mu, sigma,
                                                          out.data_ptr() if n else None, _stream_handle(None)))
    return out


def gen_zipf(n, seed, stream_id, s, domain, device="cuda"):
    lib = _lib.load()
    out = torch.empty(n, dtype=torch.int32, device=device)
    _lib.check("nfc_gen_zipf", lib.nfc_gen_zipf(n, seed, stream_id, s, domain,
                                                out.data_ptr() if n else None, _stream_handle(None)))
    return out


def gen_validity(n, seed, stream_id, p_null, device="cuda"):
    lib = _lib.load()
    out = torch.empty((n + 7) // 8, dtype=torch.uint8, device=device)
    _lib.check("nfc_gen_validity", lib.nfc_gen_validity(n, seed, stream_id, p_null,
                                                        out.data_ptr() if n else None, _stream_handle(None)))
    return out
