"""Golden vectors for grouped COUNT DISTINCT from the REFERENCE executor.

Run where the reference checkout is readable:

    python tests/golden/make_distinct_golden.py /path/to/numfast-reference

It runs the reference's group_count_distinct node (ir_count_distinct with keys) through its
own compile/optimize/cpu_execute on seeded cases -- with NULLs in keys and values, extreme
int32 keys and values, and a single-group case -- and writes distinct_golden.npz next to this
file.  Tests load only the .npz.
"""

import os
import sys

import numpy as np


def main(ref_root):
    os.environ["NUMFAST_NATIVE_DISABLE"] = "1"
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.path.insert(0, os.path.join(ref_root, "src"))
    import numfast as nf

    a = nf.get_kernel(fresh=True).alias
    g = {}

    def run(jobs):
        graph = a["optimize"](a["compile"](jobs))
        return a["cpu_execute"](graph["nodes"])

    rs = np.random.default_rng(17)
    cases = [
        ("small", rs.integers(0, 40, 3000), rs.integers(0, 25, 3000), None, None),
        ("nulls", rs.integers(-500, 500, 20000), rs.integers(-10 ** 6, 10 ** 6, 20000),
         rs.random(20000) > 0.1, rs.random(20000) > 0.2),
        ("extreme", np.array([2 ** 31 - 1, -2 ** 31, 0, 2 ** 31 - 1, -2 ** 31, 2 ** 31 - 1] * 5),
         np.array([2 ** 31 - 1, 2 ** 31 - 1, -2 ** 31, -2 ** 31, -2 ** 31, 7] * 5), None, None),
        ("onegroup", np.full(5000, 3), rs.integers(0, 900, 5000), None, None),
        ("empty", np.zeros(0, np.int64), np.zeros(0, np.int64), None, None),
    ]
    for tag, k, v, kval, vval in cases:
        k = np.asarray(k, dtype=np.int32)
        v = np.asarray(v, dtype=np.int32)
        jobs = [a["ir_series"]("v", v.tolist(), "int32", **({"validity": vval.astype(int).tolist()} if vval is not None else {})),
                a["ir_series"]("k", k.tolist(), "int32", **({"validity": kval.astype(int).tolist()} if kval is not None else {})),
                a["ir_count_distinct"]("D", "v", "k")]
        d = run(jobs)["D"]
        g[tag + "_k"], g[tag + "_v"] = k, v
        if kval is not None:
            g[tag + "_kval"] = kval
        if vval is not None:
            g[tag + "_vval"] = vval
        items = sorted(d.items()) if isinstance(d, dict) else []
        g[tag + "_ukeys"] = np.array([x for x, _ in items], dtype=np.int64)
        g[tag + "_nunique"] = np.array([c for _, c in items], dtype=np.int64)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "distinct_golden.npz")
    np.savez_compressed(out, **g)
    print("wrote", out, len(g), "arrays")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NUMFAST_REFERENCE")
    if not root:
        sys.exit("usage: %s <reference checkout> (or set NUMFAST_REFERENCE)" % sys.argv[0])
    main(root)
