"""The query chain on the group-by path: Table.query().filter().group().sort().compile().

Follows the reference facade (src/Semantic/TableExpr/_lib/chain.py):
  * group(key, {col: ops}) refuses NULL keys before any grouping runs
    (chain.py:405-417) and rebuilds a table {key, "col.op", ...} in ascending
    key order (the two-graph recipe, chain.py:1084-1134);
  * sort(*keys, desc=) is a stable permutation + one gather per column
    (chain.py:978-999), ties keep ascending-key order;
  * filter(mask) keeps the rows where the boolean mask is true.
Every node runs through numfast_b200.executor on the GPU.
"""

import numpy as np

from . import executor, ir

GROUP_OPS = ("sum", "count", "mean", "min", "max", "nunique")


class ChainError(ValueError):
    pass


class Table:
    """Columns by name: numpy values plus an optional bool validity mask each."""

    def __init__(self, columns, validity=None):
        self.columns = {k: np.ascontiguousarray(np.asarray(v)) for k, v in columns.items()}
        self.validity = {k: np.asarray(m, dtype=bool) for k, m in (validity or {}).items()}
        sizes = {v.size for v in self.columns.values()}
        if len(sizes) > 1:
            raise ChainError("columns differ in length: %s" % sorted(sizes))

    @property
    def num_rows(self):
        return next(iter(self.columns.values())).size if self.columns else 0

    def column(self, name):
        return self.columns[name]

    def to_dict(self):
        return dict(self.columns)

    def query(self):
        return Chain(self)


def from_numpy(columns, validity=None):
    return Table(columns, validity)


class _PendingSort:
    """A sort waiting for the step that consumes it: every later step but limit() needs
    the whole permutation; limit() needs only its first rows, which for one key column
    come from a radix selection that sorts only the rows kept (sort -> slice,
    cpu.py:3170-3200)."""

    def __init__(self, cols, desc, valid):
        self.cols, self.desc, self.valid = cols, desc, valid
        self._full = None

    def full(self):
        if self._full is None:
            self._full = executor.sort_perm_device(self.cols, self.desc, self.valid)
        return self._full

    def first(self, m):
        if self._full is None and len(self.cols) == 1:
            return executor.sort_topk_device(self.cols[0], self.desc[0], m, self.valid)
        return self.full()[:m]


class Chain:
    """One step of the chain.  A filter is kept pending (`_mask`) so that a following
    group() fuses it into the group-by as a row bitmap instead of compacting every column
    first; any other step materialises it (the reference's filter node, chain.py:945)."""

    def __init__(self, table, mask=None, perm=None):
        self._t = table
        self._mask = mask
        self._perm = perm  # pending sort (_PendingSort), applied by the step that consumes it

    def _take(self, idx):
        """Rows idx (host int array) of every column and validity mask."""
        cols = {n: np.ascontiguousarray(v[idx]) for n, v in self._t.columns.items()}
        val = {n: m[idx] for n, m in self._t.validity.items()}
        return Chain(Table(cols, val))

    def _materialized(self):
        if self._perm is not None:
            # Gather every column through the device permutation (ir_gather).
            names = list(self._t.columns)
            jobs = self._jobs(names)
            jobs.append(ir.ir_series("__perm", self._perm.full().cpu().numpy(), "int32"))
            for n in names:
                jobs.append(ir.ir_gather("s_" + n, n, "__perm"))
            b = executor.execute(jobs)
            cols = {n: b["s_" + n] for n in names}
            val = {n: b["s_" + n + "#validity"] for n in names if "s_" + n + "#validity" in b}
            return Chain(Table(cols, val))
        if self._mask is None:
            return self
        jobs = self._jobs(list(self._t.columns))
        jobs.append(ir.ir_series("__mask", self._mask, "bool"))
        for n in self._t.columns:
            jobs.append(ir.ir_filter("f_" + n, n, "__mask"))
        b = executor.execute(jobs)
        cols = {n: b["f_" + n] for n in self._t.columns}
        val = {n: b["f_" + n + "#validity"] for n in self._t.columns if "f_" + n + "#validity" in b}
        return Chain(Table(cols, val))

    def _col(self, name, where):
        if name not in self._t.columns:
            raise ChainError("%s: unknown column %r (have %s)" % (where, name, list(self._t.columns)))
        return name

    def _jobs(self, names):
        jobs = []
        for n in names:
            v = self._t.columns[n]
            jobs.append(ir.ir_series(n, v, str(v.dtype), self._t.validity.get(n)))
        return jobs

    def filter(self, mask):
        base = self._materialized()  # sees the rows (and order) of the steps before it
        m = np.asarray(mask(base._t) if callable(mask) else mask, dtype=bool)
        if m.size != base._t.num_rows:
            raise ChainError("filter: mask has %d rows, table %d" % (m.size, base._t.num_rows))
        return Chain(base._t, m)

    def group(self, key, aggs):
        if self._perm is not None:
            return self._materialized().group(key, aggs)
        self._col(key, "group")
        if not isinstance(aggs, dict) or not aggs:
            raise ChainError("group: aggs must be a non-empty {col: (ops,)} dict, got %r" % (aggs,))
        specs = {}
        for col, ops in aggs.items():
            self._col(col, "group")
            ops_t = (ops,) if isinstance(ops, str) else tuple(ops)
            if not ops_t or any(o not in GROUP_OPS for o in ops_t):
                raise ChainError("group: unknown aggregate in %r for %r" % (ops_t, col))
            specs[col] = ops_t
        kv = self._t.validity.get(key)
        if kv is not None:
            live = kv if self._mask is None else (kv | ~self._mask)
            if not bool(np.all(live)):
                raise ChainError("group: key column %r has %d NULL rows; NULL keys are not grouped. "
                                 "Filter those rows out before group()." % (key, int((~live).sum())))
        # nunique runs as one group_count_distinct node per column, next to one
        # groupby_multi node for every other aggregate (chain.py:1046-1080).
        gb = {c: tuple(o for o in ops if o != "nunique") for c, ops in specs.items()}
        gb = {c: ops for c, ops in gb.items() if ops}
        nuniq = [c for c, ops in specs.items() if "nunique" in ops]
        carry = None
        if gb:
            cols = list(gb)
            jobs = self._jobs(cols + ([key] if key not in cols else []))
            filt = None
            if self._mask is not None:
                jobs.append(ir.ir_series("__mask", self._mask, "bool"))
                filt = "__mask"
            if len(cols) == 1:
                jobs.append(ir.ir_groupby_multi("G", cols[0], key, gb[cols[0]], result="carry", row_filter=filt))
            else:
                jobs.append(ir.ir_groupby_multi("G", cols, key, {c: gb[c] for c in cols}, result="carry",
                                                row_filter=filt))
            carry = executor.execute(jobs)["G"]
        distinct = {}
        if nuniq:
            base = self._materialized()
            for col in nuniq:
                jobs = base._jobs([col] + ([key] if key != col else []))
                jobs.append(ir.ir_count_distinct("D", col, key))
                distinct[col] = executor.execute(jobs)["D"]
        if carry is not None:
            ukeys = np.asarray(carry.ukeys, dtype=np.int64)
        else:
            ukeys = np.asarray(sorted(int(x) for x in distinct[nuniq[0]]), dtype=np.int64)
        out = {key: ukeys}
        for col, ops in specs.items():
            for op in ops:
                field = "%s.%s" % (col, op)
                if op == "nunique":
                    lut = distinct[col]
                    missing = [int(x) for x in ukeys.tolist() if int(x) not in lut]
                    if missing:
                        raise ChainError("group: key %d has no valid %r value, so it has no nunique "
                                         "(filter NULL %r rows out first)" % (missing[0], col, col))
                    out[field] = np.asarray([lut[int(x)] for x in ukeys.tolist()], dtype=np.int64)
                elif op == "count":
                    out[field] = carry.counts
                elif op == "mean":
                    out[field] = carry.means(col)
                elif op == "min":
                    out[field] = carry.mins[col]
                elif op == "max":
                    out[field] = carry.maxs[col]
                else:
                    out[field] = carry.sums[col]
        return Chain(Table(out))

    def sort(self, *keys, desc=False):
        """Stable sort by the key columns (all ascending or all descending; NULL rows
        last).  Nothing runs until the next step: compile() and the other steps sort every
        row and gather them; limit() computes only the rows it keeps (one key column: radix
        selection of the k-th key and a sort of the kept rows; several: the full lexsort),
        then gathers those (top-k = sort -> slice -> gather)."""
        if self._mask is not None or self._perm is not None:
            return self._materialized().sort(*keys, desc=desc)
        if not keys:
            raise ChainError("sort needs >=1 key column")
        if isinstance(desc, (list, tuple)):
            raise ChainError("sort takes one desc flag for all keys")
        for k in keys:
            self._col(k, "sort")
        masks = [self._t.validity[k] for k in keys if k in self._t.validity]
        valid = None
        for m in masks:
            valid = m if valid is None else (valid & m)
        return Chain(self._t, perm=_PendingSort([self._t.columns[k] for k in keys], [bool(desc)] * len(keys),
                                                valid))

    def limit(self, n, offset=0):
        """Rows [offset, offset + n) (chain.py:1001-1008).  After sort() only those rows'
        indices leave the device and only those rows are gathered."""
        if isinstance(n, bool) or not isinstance(n, int) or n < 0:
            raise ChainError("limit: n must be a non-negative int, got %r" % (n,))
        if isinstance(offset, bool) or not isinstance(offset, int) or offset < 0:
            raise ChainError("limit: offset must be a non-negative int, got %r" % (offset,))
        if self._perm is not None:
            m = min(offset + n, self._t.num_rows)
            idx = self._perm.first(m)[offset:m].cpu().numpy().astype(np.int64)
            return self._take(idx)
        base = self._materialized()
        rows = base._t.num_rows
        return base._take(np.arange(min(offset, rows), min(offset + n, rows)))

    def compile(self):
        return self._materialized()._t
