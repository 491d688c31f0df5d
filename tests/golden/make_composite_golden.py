"""Golden vectors for composite (tuple) group keys from the REFERENCE executor.

Run where the reference checkout is readable:

    python tests/golden/make_composite_golden.py /path/to/numfast-reference

Cases: pack_keys(mode="hash") over 2, 3 and 4 int32 columns with negative values and NULLs
followed by groupby_multi (sum, count) -- the reference's composite_tuple_index order -- and
pack_keys(mode="pack") over 2 columns (an int64 key beyond int32) followed by groupby_multi.
Writes composite_golden.npz next to this file; tests load only the .npz.
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

    rs = np.random.default_rng(31)
    n = 6000
    for nc in (2, 3, 4, 5):
        keys = [rs.integers(-4, 5, n).astype(np.int32) for _ in range(nc)]
        v = rs.integers(-1000, 1001, n).astype(np.int32)
        kval = rs.random(n) > 0.05
        vval = rs.random(n) > 0.05
        jobs = [a["ir_series"]("k%d" % i, keys[i].tolist(), "int32",
                               **({"validity": kval.astype(int).tolist()} if i == 0 else {}))
                for i in range(nc)]
        jobs += [a["ir_series"]("v", v.tolist(), "int32", validity=vval.astype(int).tolist()),
                 a["ir_pack_keys"]("K", *["k%d" % i for i in range(nc)], mode="hash"),
                 a["ir_groupby_multi"]("G", "v", "K", ("sum", "count"), result="carry")]
        c = run(jobs)["G"]
        tag = "hash%d" % nc
        for i in range(nc):
            g["%s_k%d" % (tag, i)] = keys[i]
        g[tag + "_v"], g[tag + "_kval"], g[tag + "_vval"] = v, kval, vval
        g[tag + "_ukeys"] = np.asarray([list(t) for t in c.ukeys], dtype=np.int64).reshape(-1, nc)
        g[tag + "_counts"] = np.asarray(c.counts, dtype=np.int64)
        g[tag + "_sums"] = np.asarray(c.sums["v"], dtype=np.int64)
    # pack mode: int64 keys (hi << 32 | uint32 lo) grouped directly.
    hi = rs.integers(-3, 3, n).astype(np.int32)
    lo = rs.integers(-5, 5, n).astype(np.int32)
    v = rs.integers(-1000, 1001, n).astype(np.int32)
    jobs = [a["ir_series"]("h", hi.tolist(), "int32"), a["ir_series"]("l", lo.tolist(), "int32"),
            a["ir_series"]("v", v.tolist(), "int32"), a["ir_pack_keys"]("K", "h", "l", mode="pack"),
            a["ir_groupby_multi"]("G", "v", "K", ("sum", "count"), result="carry")]
    c = run(jobs)["G"]
    g["pack_hi"], g["pack_lo"], g["pack_v"] = hi, lo, v
    g["pack_ukeys"] = np.asarray(c.ukeys, dtype=np.int64)
    g["pack_counts"] = np.asarray(c.counts, dtype=np.int64)
    g["pack_sums"] = np.asarray(c.sums["v"], dtype=np.int64)
    # radix mode over non-negative codes.
    c0 = rs.integers(0, 50, n).astype(np.int32)
    c1 = rs.integers(0, 70, n).astype(np.int32)
    jobs = [a["ir_series"]("c0", c0.tolist(), "int32"), a["ir_series"]("c1", c1.tolist(), "int32"),
            a["ir_series"]("v", v.tolist(), "int32"), a["ir_pack_keys"]("K", "c0", "c1", mode="radix"),
            a["ir_groupby_multi"]("G", "v", "K", ("sum", "count"), result="carry")]
    c = run(jobs)["G"]
    g["radix_c0"], g["radix_c1"] = c0, c1
    g["radix_ukeys"] = np.asarray(c.ukeys, dtype=np.int64)
    g["radix_sums"] = np.asarray(c.sums["v"], dtype=np.int64)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "composite_golden.npz")
    np.savez_compressed(out, **g)
    print("wrote", out, len(g), "arrays")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NUMFAST_REFERENCE")
    if not root:
        sys.exit("usage: %s <reference checkout> (or set NUMFAST_REFERENCE)" % sys.argv[0])
    main(root)
