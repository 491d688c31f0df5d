"""IR jobs through the executor and the query chain (config 1) on the GPU."""

import numpy as np
import pytest

from numfast_b200 import chain, executor, ir
from oracle import nf_oracle as O

pytestmark = pytest.mark.gpu


def test_groupby_multi_dict_and_carry(cuda, golden):
    tag = "gb_dense"
    jobs = [ir.ir_series("v", golden[tag + "_in_v"], "int32", golden[tag + "_in_vval"]),
            ir.ir_series("f", golden[tag + "_in_f"], "float64", golden[tag + "_in_fval"]),
            ir.ir_series("k", golden[tag + "_in_k"], "int32", golden[tag + "_in_kval"]),
            ir.ir_groupby_multi("G", ["v", "f"], "k", {"v": ("sum", "count", "min", "max"), "f": ("sum", "min", "max")},
                                result="carry"),
            ir.ir_groupby_multi("D", ["v", "f"], "k", {"v": ("sum", "count", "mean"), "f": ("max",)})]
    b = executor.execute(jobs)
    c = b["G"]
    np.testing.assert_array_equal(c.ukeys, golden[tag + "_ukeys"])
    np.testing.assert_array_equal(c.sums["v"], golden[tag + "_v_sum"])
    np.testing.assert_array_equal(c.maxs["f"], golden[tag + "_f_max"])
    d = b["D"]
    k0 = int(golden[tag + "_ukeys"][0])
    assert d[k0]["v"]["sum"] == int(golden[tag + "_v_sum"][0])
    assert d[k0]["v"]["count"] == int(golden[tag + "_counts"][0])
    assert list(d) == golden[tag + "_ukeys"].tolist()


def test_legacy_single_column_and_sort(cuda):
    jobs = [ir.ir_series("v", [1, 2, 3, 4, 5, 6], "int32"), ir.ir_series("k", [2, 0, 2, 1, 0, 2], "int32"),
            ir.ir_groupby_multi("g", "v", "k", ("sum", "count", "mean"))]
    b = executor.execute(jobs)
    assert b["g"] == {0: {"sum": 7, "count": 2, "mean": 3.5}, 1: {"sum": 4, "count": 1, "mean": 4.0},
                      2: {"sum": 10, "count": 3, "mean": 10 / 3}}
    jobs = [ir.ir_series("s", [2, 2, 1, 1, 1, 1], "int64"), ir.ir_sort("p", "s", descending=True)]
    assert executor.execute(jobs)["p"].tolist() == [0, 1, 2, 3, 4, 5]


def test_unique_inverse_with_validity(cuda, golden):
    jobs = [ir.ir_series("k", golden["uniq_in"], "int32", golden["uniq_val"]), ir.ir_unique_inverse("u", "k")]
    b = executor.execute(jobs)
    np.testing.assert_array_equal(b["u"], golden["uniq_null_u"])
    np.testing.assert_array_equal(b["u#inv"], golden["uniq_null_inv"])
    assert b["u#ng"] == golden["uniq_null_u"].size


def test_config1_chain(cuda, golden):
    from numfast_b200 import device as dev
    n = 1_000_000
    key = dev.rng_fill_i32(n, 42, 0, 0, 1000).cpu().numpy()
    v = dev.rng_fill_i32(n, 42, 1, -100, 101).cpu().numpy()
    t = chain.from_numpy({"key": key, "v": v})
    out = t.query().group("key", {"v": ("sum", "count")}).sort("v.sum", desc=True).compile()
    np.testing.assert_array_equal(out.column("key"), golden["cfg1_key"])
    np.testing.assert_array_equal(out.column("v.sum"), golden["cfg1_v_sum"])
    np.testing.assert_array_equal(out.column("v.count"), golden["cfg1_v_count"])


def test_chain_filter_then_group(cuda):
    rs = np.random.default_rng(8)
    k = rs.integers(0, 50, 10_000).astype(np.int32)
    v = rs.integers(-5, 5, 10_000).astype(np.int32)
    t = chain.from_numpy({"k": k, "v": v})
    out = t.query().filter(lambda tb: tb.column("v") > 0).group("k", {"v": ("sum", "min")}).compile()
    ref = O.groupby_multi(k[v > 0], {"v": v[v > 0]}, {"v": ("sum", "min")})
    np.testing.assert_array_equal(out.column("k"), ref["ukeys"])
    np.testing.assert_array_equal(out.column("v.sum"), ref["sums"]["v"])
    np.testing.assert_array_equal(out.column("v.min"), ref["mins"]["v"])


def test_chain_filter_fusion_cases(cuda):
    """filter -> group fuses the mask into the group-by; filter -> filter, filter -> sort
    and filter -> compile still see exactly the kept rows; a filter may hide NULL keys."""
    rs = np.random.default_rng(21)
    n = 50_000
    k = rs.integers(0, 700, n).astype(np.int32)
    v = rs.integers(-1000, 1001, n).astype(np.int32)
    kval = rs.random(n) > 0.1
    t = chain.from_numpy({"k": k, "v": v}, validity={"k": kval})
    # The filter removes every NULL-key row, so group() is allowed.
    out = t.query().filter(kval & (v > -500)).group("k", {"v": ("sum", "count")}).compile()
    m = kval & (v > -500)
    ref = O.groupby_multi(k[m], {"v": v[m]}, {"v": ("sum", "count")})
    np.testing.assert_array_equal(out.column("k"), ref["ukeys"])
    np.testing.assert_array_equal(out.column("v.sum"), ref["sums"]["v"])
    np.testing.assert_array_equal(out.column("v.count"), ref["counts"])
    # Two filters: the second mask is over the rows the first kept.
    q = t.query().filter(kval).filter(lambda tb: tb.column("v") % 3 == 0).group("k", {"v": "sum"}).compile()
    m2 = kval.copy()
    m2[kval] = v[kval] % 3 == 0
    ref2 = O.groupby_multi(k[m2], {"v": v[m2]}, {"v": ("sum",)})
    np.testing.assert_array_equal(q.column("v.sum"), ref2["sums"]["v"])
    # filter -> compile and filter -> sort materialise the kept rows.
    c = t.query().filter(v > 900).compile()
    np.testing.assert_array_equal(c.column("v"), v[v > 900])
    srt = t.query().filter(v > 900).sort("v").compile()
    np.testing.assert_array_equal(srt.column("v"), np.sort(v[v > 900], kind="stable"))
    with pytest.raises(chain.ChainError):
        t.query().filter(v > 0).group("k", {"v": "sum"})


def test_topk_sort_slice_gather_composition(cuda):
    """sort -> slice -> gather is top-k (the reference's test_ops_sort composition)."""
    vals = np.array([5, 1, 4, 1, 5, 9, 2, 6], dtype=np.int32)
    jobs = [ir.ir_series("v", vals, "int32"), ir.ir_sort("p", "v", descending=True),
            ir.ir_slice("t", "p", limit=3), ir.ir_gather("g", "v", "t")]
    b = executor.execute(jobs)
    assert [int(x) for x in b["g"]] == [9, 6, 5]
    jobs = [ir.ir_series("v", vals, "int32"), ir.ir_slice("s", "v", limit=4, offset=6)]
    assert [int(x) for x in executor.execute(jobs)["s"]] == [2, 6]


def test_chain_sort_limit_on_device(cuda):
    """sort() keeps its permutation on the device; limit() gathers only the kept rows and
    equals slicing the fully sorted table (stable ties, NULL keys last)."""
    rs = np.random.default_rng(23)
    n = 200_000
    k = rs.integers(-500, 500, n).astype(np.int32)
    v = rs.integers(0, 10 ** 6, n).astype(np.int64)
    kval = rs.random(n) > 0.1
    t = chain.from_numpy({"k": k, "v": v}, validity={"k": kval})
    for desc in (False, True):
        full = t.query().sort("k", desc=desc).compile()
        perm = O.sort_perm([k], [desc], kval)
        np.testing.assert_array_equal(full.column("v"), v[perm])
        for lim, off in ((10, 0), (1000, 5000), (50, n - 20), (5, n + 3), (0, 0)):
            top = t.query().sort("k", desc=desc).limit(lim, off).compile()
            np.testing.assert_array_equal(top.column("v"), full.column("v")[off:off + lim])
            np.testing.assert_array_equal(top.column("k"), full.column("k")[off:off + lim])
    # limit without a sort is a plain row range; sort -> group still works.
    np.testing.assert_array_equal(t.query().limit(7, 3).compile().column("v"), v[3:10])
    g = chain.from_numpy({"k": k, "v": v}).query().sort("v").group("k", {"v": "sum"}).compile()
    ref = O.groupby_multi(k, {"v": v}, {"v": ("sum",)})
    np.testing.assert_array_equal(g.column("v.sum"), ref["sums"]["v"])
