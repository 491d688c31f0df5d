"""Generate golden vectors by running the REFERENCE NumFast (NumPy executor).

Run in a container where the reference checkout is readable:

    python tests/golden/make_golden.py /path/to/numfast-reference

It imports the reference from <root>/src with its native library disabled (the NumPy
executor is the reference's own implementation of the whole path), runs the
group-by / sort / unique / RNG cases below and writes golden.npz next to this file.
The tests load golden.npz only; the reference itself is never needed at test time.
"""

import os
import sys

import numpy as np


def main(ref_root):
    os.environ["NUMFAST_NATIVE_DISABLE"] = "1"
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.path.insert(0, os.path.join(ref_root, "src"))
    import numfast as nf
    import pandas as pd

    a = nf.get_kernel(fresh=True).alias
    g = {}

    def run(jobs):
        graph = a["optimize"](a["compile"](jobs))
        return a["cpu_execute"](graph["nodes"])

    # --- RNG: Philox lanes (rng.py:111-141) ------------------------------
    rng_cases = [(4096, 42, 0, 0, 0, 1000), (4096, 42, 1, 0, -100, 101), (1000, 7, 5, 123456, -2 ** 31, 2 ** 31),
                 (333, 2 ** 63 + 5, 2 ** 40 + 3, 2 ** 33, -5, 5)]
    for i, (n, seed, stream, off, lo, hi) in enumerate(rng_cases):
        g["rng_i32_%d" % i] = nf.to_numpy(nf.rng_fill_i32(n, seed, stream=stream, offset=off, lo=lo, hi=hi))
        g["rng_i32_%d_args" % i] = np.array([n, seed, stream, off, lo, hi], dtype=object).astype(str)
    f_cases = [(4096, 42, 2, 0, 0.0, 1.0), (1000, 42, 4, 77, -3.5, 2.25)]
    for i, (n, seed, stream, off, lo, hi) in enumerate(f_cases):
        g["rng_f64_%d" % i] = nf.to_numpy(nf.rng_fill_f64(n, seed, stream=stream, offset=off, lo=lo, hi=hi))
        g["rng_f64_%d_args" % i] = np.array([n, seed, stream, off, lo, hi], dtype=np.float64)

    # --- groupby_multi with validity + min/max (cfg2-shaped, small) ---------
    def gb_case(tag, k, v, f, kval, vval, fval):
        jobs = [a["ir_series"]("v", v.tolist(), "int32", validity=vval.astype(int).tolist()),
                a["ir_series"]("f", f.tolist(), "float64", validity=fval.astype(int).tolist()),
                a["ir_series"]("k", k.tolist(), "int32", validity=kval.astype(int).tolist()),
                a["ir_groupby_multi"]("G", ["v", "f"], "k",
                                      {"v": ("sum", "count", "min", "max"), "f": ("sum", "min", "max")},
                                      result="carry")]
        c = run(jobs)["G"]
        g[tag + "_in_k"], g[tag + "_in_v"], g[tag + "_in_f"] = k, v, f
        g[tag + "_in_kval"], g[tag + "_in_vval"], g[tag + "_in_fval"] = kval, vval, fval
        g[tag + "_ukeys"] = np.asarray(c.ukeys)
        g[tag + "_counts"] = np.asarray(c.counts)
        g[tag + "_v_sum"] = np.asarray(c.sums["v"])
        g[tag + "_v_min"] = np.asarray(c.mins["v"])
        g[tag + "_v_max"] = np.asarray(c.maxs["v"])
        g[tag + "_f_sum"] = np.asarray(c.sums["f"])
        g[tag + "_f_min"] = np.asarray(c.mins["f"])
        g[tag + "_f_max"] = np.asarray(c.maxs["f"])

    rs = np.random.default_rng(42)
    n = 6000
    k = rs.integers(0, 700, n).astype(np.int32)
    v = rs.integers(-1000, 1001, n).astype(np.int32)
    f = np.exp(3 + rs.standard_normal(n))
    gb_case("gb_dense", k, v, f, rs.random(n) >= 0.05, rs.random(n) >= 0.05, rs.random(n) >= 0.05)
    # sparse keys over the whole int32 range (hash plan)
    k2 = rs.integers(-2 ** 31, 2 ** 31, 800).astype(np.int32)
    k2 = np.concatenate([k2, k2[:300], k2[:50]])
    n2 = k2.size
    gb_case("gb_sparse", k2, rs.integers(-2 ** 31, 2 ** 31, n2).astype(np.int32), rs.standard_normal(n2) * 1e3,
            rs.random(n2) >= 0.1, rs.random(n2) >= 0.1, np.ones(n2, dtype=bool))
    # int32 boundary values: sums must widen to int64 exactly
    k3 = np.array([0, 0, 0, 1, 1, 2, 2, 2, 2], dtype=np.int32)
    v3 = np.array([2 ** 31 - 1, 2 ** 31 - 1, 5, -2 ** 31, -2 ** 31, 7, -7, 2 ** 31 - 1, -2 ** 31], dtype=np.int32)
    gb_case("gb_bound", k3, v3, v3.astype(np.float64), np.ones(9, bool), np.ones(9, bool), np.ones(9, bool))
    # sorted keys with a group whose rows are all NULL (absent key)
    k4 = np.repeat(np.arange(50, dtype=np.int32), 7)
    vv4 = np.ones(k4.size, dtype=bool)
    vv4[k4 == 13] = False
    gb_case("gb_sorted", k4, (k4 * 3 - 40).astype(np.int32), np.linspace(-1, 1, k4.size), np.ones(k4.size, bool),
            vv4, np.ones(k4.size, bool))
    # float min/max with NaN and signed zeros
    k5 = np.array([0, 0, 0, 1, 1, 2, 2], dtype=np.int32)
    f5 = np.array([1.0, np.nan, -3.0, -0.0, 2.5, np.inf, -np.inf])
    gb_case("gb_nan", k5, np.arange(7, dtype=np.int32), f5, np.ones(7, bool), np.ones(7, bool), np.ones(7, bool))

    # --- sort (cpu.py:1154-1225) ------------------------------------------
    sk = np.array([3, -2 ** 31, 5, 3, 2 ** 31 - 1, 0, 5, -2 ** 31, 3, 0], dtype=np.int32)
    sval = np.array([1, 1, 1, 0, 1, 1, 1, 1, 0, 1], dtype=bool)
    for desc in (False, True):
        b = run([a["ir_series"]("k", sk.tolist(), "int32"), a["ir_sort"]("p", "k", descending=desc)])
        g["sort_i32_%s" % ("desc" if desc else "asc")] = np.asarray(b["p"])
        b = run([a["ir_series"]("k", sk.tolist(), "int32", validity=sval.astype(int).tolist()),
                 a["ir_sort"]("p", "k", descending=desc)])
        g["sort_i32_null_%s" % ("desc" if desc else "asc")] = np.asarray(b["p"])
    g["sort_in_k"], g["sort_in_val"] = sk, sval
    fk = np.array([1.5, np.nan, -0.0, 0.0, -np.inf, np.nan, 1.5, np.inf, -2.0, 0.0])
    for desc in (False, True):
        b = run([a["ir_series"]("k", fk.tolist(), "float64"), a["ir_sort"]("p", "k", descending=desc)])
        g["sort_f64_%s" % ("desc" if desc else "asc")] = np.asarray(b["p"])
    g["sort_in_f"] = fk
    # random int64 keys with ties, both directions
    rk = rs.integers(-50, 50, 5000).astype(np.int64) * (2 ** 40)
    for desc in (False, True):
        b = run([a["ir_series"]("k", rk, "int64"), a["ir_sort"]("p", "k", descending=desc)])
        g["sort_i64_%s" % ("desc" if desc else "asc")] = np.asarray(b["p"])
    g["sort_in_i64"] = rk
    # lexicographic two-key sort, mixed directions
    l1 = rs.integers(0, 5, 3000).astype(np.int32)
    l2 = rs.integers(-3, 3, 3000).astype(np.int32)
    b = run([a["ir_series"]("a", l1, "int32"), a["ir_series"]("b", l2, "int32"),
             a["ir_sort"]("p", "a", "b", descending=[True, False])])
    g["sort_lex"], g["sort_lex_a"], g["sort_lex_b"] = np.asarray(b["p"]), l1, l2

    # --- unique_inverse (cpu.py:4006-4040) ---------------------------------
    uk = rs.integers(-1000, 1000, 4000).astype(np.int32)
    uval = rs.random(4000) >= 0.2
    b = run([a["ir_series"]("k", uk, "int32"), a["ir_unique_inverse"]("u", "k")])
    g["uniq_in"], g["uniq_u"], g["uniq_inv"] = uk, np.asarray(b["u"]), np.asarray(b["u#inv"])
    b = run([a["ir_series"]("k", uk, "int32", validity=uval.astype(int).tolist()), a["ir_unique_inverse"]("u", "k")])
    g["uniq_val"], g["uniq_null_u"], g["uniq_null_inv"] = uval, np.asarray(b["u"]), np.asarray(b["u#inv"])

    # --- config 1 chain: 1M rows, 1000 keys, group + sort desc ------------
    n1 = 1_000_000
    key = nf.to_numpy(nf.rng_fill_i32(n1, 42, stream=0, lo=0, hi=1000))
    val = nf.to_numpy(nf.rng_fill_i32(n1, 42, stream=1, lo=-100, hi=101))
    t = nf.from_pandas(pd.DataFrame({"key": key, "v": val}))
    out = t.query().group("key", {"v": ("sum", "count")}).sort("v.sum", desc=True).compile()
    df = nf.to_pandas(out)
    g["cfg1_key"] = df["key"].to_numpy().astype(np.int64)
    g["cfg1_v_sum"] = df["v.sum"].to_numpy().astype(np.int64)
    g["cfg1_v_count"] = df["v.count"].to_numpy().astype(np.int64)
    g["cfg1_key_head"] = key[:4096]
    g["cfg1_v_head"] = val[:4096]

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")
    np.savez_compressed(path, **g)
    print("wrote", path, len(g), "arrays")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NUMFAST_REFERENCE")
    if not root:
        sys.exit("usage: %s <reference checkout> (or set NUMFAST_REFERENCE)" % sys.argv[0])
    main(root)
