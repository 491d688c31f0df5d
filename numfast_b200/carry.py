"""ColumnCarry: the columnar group-by result (src/Drivers/CPU/_lib/carry.py:21-115).

ukeys (int64, ascending) + counts (int64) + per-column sums (int64 for integer columns,
float64 otherwise) + optional mins/maxs (value dtype).  Mean is derived sums/counts.
The dict materialisers produce the same nested shapes as the reference's
to_dict_flat / to_dict_single / to_dict_multi, with Python scalars.
"""

import numpy as np


class ColumnCarry:
    __slots__ = ("ukeys", "counts", "sums", "mins", "maxs", "_means")

    def __init__(self, ukeys, counts, sums, mins=None, maxs=None):
        if isinstance(ukeys, np.ndarray) and ukeys.dtype == object:
            self.ukeys = ukeys  # composite keys: one tuple per group (groupindex.py:520-639)
        else:
            self.ukeys = np.ascontiguousarray(np.asarray(ukeys, dtype=np.int64))
        self.counts = np.ascontiguousarray(np.asarray(counts, dtype=np.int64))
        self.sums = {c: np.ascontiguousarray(np.asarray(s)) for c, s in (sums or {}).items()}
        self.mins = {c: np.ascontiguousarray(np.asarray(s)) for c, s in (mins or {}).items()}
        self.maxs = {c: np.ascontiguousarray(np.asarray(s)) for c, s in (maxs or {}).items()}
        self._means = {}

    @property
    def ngroups(self):
        return int(self.ukeys.shape[0])

    def means(self, col):
        m = self._means.get(col)
        if m is None:
            m = self._means[col] = self.sums[col].astype(np.float64) / self.counts
        return m

    def _cell(self, col, ops, i, lists):
        sub = {}
        for op in ops:
            if op == "count":
                sub["count"] = lists["count"][i]
            else:
                sub[op] = lists[(col, op)][i]
        return sub

    def _lists(self, cols_ops):
        out = {"count": self.counts.tolist()}
        for col, ops in cols_ops:
            for op in ops:
                if op == "sum":
                    out[(col, op)] = self.sums[col].tolist()
                elif op == "mean":
                    out[(col, op)] = self.means(col).tolist()
                elif op == "min":
                    out[(col, op)] = self.mins[col].tolist()
                elif op == "max":
                    out[(col, op)] = self.maxs[col].tolist()
        return out

    def to_dict_flat(self, op, col=None):
        """{key: scalar} (legacy groupby shape)."""
        if col is None:
            src = {"sum": self.sums, "mean": self.sums, "min": self.mins, "max": self.maxs}.get(op, self.sums)
            col = next(iter(src)) if src else None
        lists = self._lists([(col, (op,))] if op != "count" else [])
        keys = self.ukeys.tolist()
        vals = lists["count"] if op == "count" else lists[(col, op)]
        return dict(zip(keys, vals))

    def to_dict_single(self, col, ops):
        """{key: {op: val}} (groupby_multi single-column shape)."""
        ops = [o for o in ("sum", "count", "mean", "min", "max") if o in ops]
        lists = self._lists([(col, ops)])
        return {k: self._cell(col, ops, i, lists) for i, k in enumerate(self.ukeys.tolist())}

    def to_dict_multi(self, cols, ops_map):
        """{key: {col: {op: val}}} (groupby_multi multi-column shape)."""
        norm = [(c, [o for o in ("sum", "count", "mean", "min", "max") if o in ops_map[c]]) for c in cols]
        lists = self._lists(norm)
        return {k: {c: self._cell(c, ops, i, lists) for c, ops in norm}
                for i, k in enumerate(self.ukeys.tolist())}
