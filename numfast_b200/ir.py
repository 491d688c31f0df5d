"""IR node constructors for the group-by path (src/Semantic/IR/_lib/nodes.py).

Same op names, inputs order and params as the reference, so job lists built for the
reference executor run unchanged through numfast_b200.executor.execute:
  ir_series           nodes.py:32   source column (+ optional validity)
  ir_groupby_multi    nodes.py:304  fused multi-aggregate (inputs [*values, keys])
  ir_sort             nodes.py:162  stable permutation (inputs = keys)
  ir_gather           nodes.py:~620 values[idx]
  ir_unique_inverse   nodes.py:652  sorted unique + inverse
  ir_filter           row mask applied to one column (nodes.py filter)
"""

GROUPBY_OPS = ("sum", "count", "mean", "min", "max")


class IRError(ValueError):
    pass


def ir_series(out, values, dtype="int32", validity=None):
    params = {"values": values, "dtype": dtype}
    if validity is not None:
        params["validity"] = validity
    return {"op": "series", "inputs": [], "params": params, "out": out}


def ir_groupby_multi(out, values, keys, ops=("sum", "count"), result="dict", row_filter=None):
    """groupby_multi node (src/Semantic/IR/_lib/nodes.py).  row_filter (not in the reference's
    IR): name of a bool series; rows where it is false take no part, as if a filter node had
    compacted them out first -- the fused filter -> group of the chain."""
    node = _ir_groupby_multi(out, values, keys, ops, result)
    if row_filter is not None:
        node["params"]["filter"] = row_filter
        node["inputs"] = node["inputs"] + [row_filter]
    return node


def _ir_groupby_multi(out, values, keys, ops=("sum", "count"), result="dict"):
    if result not in ("dict", "carry"):
        raise IRError("unknown groupby_multi result %r: use one of dict/carry." % (result,))
    if isinstance(values, str):
        ops = tuple(ops)
        if not ops or any(o not in GROUPBY_OPS for o in ops):
            raise IRError("groupby_multi ops must be a non-empty subset of %s, got %s." % (list(GROUPBY_OPS), list(ops)))
        params = {"ops": list(ops)}
        if result != "dict":
            params["result"] = result
        return {"op": "groupby_multi", "inputs": [values, keys], "params": params, "out": out}
    cols = list(values)
    if not cols or any(not isinstance(c, str) for c in cols):
        raise IRError("groupby_multi values must be a series name or non-empty [names], got %r." % (values,))
    if not isinstance(ops, dict) or set(ops) != set(cols):
        raise IRError("groupby_multi multi-col ops must be {col: (ops)} for %s, got %r." % (cols, ops))
    norm = {}
    for c in cols:
        oc = tuple(ops[c])
        if not oc or any(o not in GROUPBY_OPS for o in oc):
            raise IRError("groupby_multi ops for %r must be a non-empty subset of %s, got %s." % (c, list(GROUPBY_OPS), list(oc)))
        norm[c] = list(oc)
    params = {"ops": norm, "cols": cols}
    if result != "dict":
        params["result"] = result
    return {"op": "groupby_multi", "inputs": cols + [keys], "params": params, "out": out}


def ir_sort(out, *keys, descending=False):
    if not keys:
        raise IRError("sort needs >=1 key series.")
    if isinstance(descending, bool):
        desc = [descending] * len(keys)
    else:
        desc = [bool(d) for d in descending]
        if len(desc) != len(keys):
            raise IRError("sort descending needs one bool per key.")
    return {"op": "sort", "inputs": list(keys), "params": {"descending": desc}, "out": out}


def ir_gather(out, values, indices):
    return {"op": "gather", "inputs": [values, indices], "params": {}, "out": out}


def ir_unique_inverse(out, values):
    return {"op": "unique_inverse", "inputs": [values], "params": {}, "out": out}


def ir_filter(out, values, mask):
    return {"op": "filter", "inputs": [values, mask], "params": {}, "out": out}


def ir_count_distinct(out, values, keys=None):
    """COUNT DISTINCT (src/Semantic/IR/_lib/nodes.py:675-688): keys=None is the global
    count (a unique node); with keys, a group_count_distinct node over [values, keys]."""
    if keys is None:
        return {"op": "unique", "inputs": [values], "params": {}, "out": out}
    return {"op": "group_count_distinct", "inputs": [values, keys], "params": {}, "out": out}


def ir_pack_keys(out, *key_series, mode="pack", radix=None):
    """Composite keys (src/Semantic/IR/_lib/nodes.py:353-390): "pack" (1-2 series ->
    int64), "radix" (mixed-radix int64), "hash" (tuple keys for groupby_multi)."""
    if mode not in ("pack", "radix", "hash"):
        raise IRError("pack_keys mode must be pack/radix/hash, got %r." % (mode,))
    if mode == "pack" and not 1 <= len(key_series) <= 2:
        raise IRError("pack_keys needs 1-2 key series, got %d." % len(key_series))
    if len(key_series) < 1:
        raise IRError("pack_keys needs >=1 key series.")
    params = {"mode": mode}
    if mode == "radix" and radix is not None:
        params["radix"] = [int(m) for m in radix]
    return {"op": "pack_keys", "inputs": list(key_series), "params": params, "out": out}


def ir_slice(out, values, limit=None, offset=0):
    """values[offset:offset+limit] (src/Semantic/IR/_lib/nodes.py:189-208); top-k is
    sort -> slice -> gather."""
    if limit is not None and (isinstance(limit, bool) or not isinstance(limit, int)):
        raise IRError("slice limit must be a non-negative int or None, got %r." % (limit,))
    if isinstance(offset, bool) or not isinstance(offset, int):
        raise IRError("slice offset must be a non-negative int, got %r." % (offset,))
    if (limit is not None and limit < 0) or offset < 0:
        raise IRError("slice needs limit>=0 and offset>=0, got limit=%s offset=%s." % (limit, offset))
    return {"op": "slice", "inputs": [values], "params": {"limit": limit, "offset": offset}, "out": out}
