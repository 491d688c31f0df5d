"""Composite (tuple) and int64 group keys: the oracle against the reference's own results
(CPU) and the CUDA path -- pairwise folds of dense codes -- against both (GPU)."""

import os

import numpy as np
import pytest

from oracle import nf_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def cgold():
    return np.load(os.path.join(HERE, "golden", "composite_golden.npz"))


@pytest.mark.parametrize("nc", [2, 3, 4, 5])
def test_oracle_tuple_keys_match_reference(cgold, nc):
    tag = "hash%d" % nc
    cols = [cgold["%s_k%d" % (tag, i)] for i in range(nc)]
    valid = cgold[tag + "_kval"] & cgold[tag + "_vval"]
    uk, cnt, sm = O.composite_groupby_sum_count(cols, cgold[tag + "_v"], valid)
    np.testing.assert_array_equal(uk, cgold[tag + "_ukeys"])
    np.testing.assert_array_equal(cnt, cgold[tag + "_counts"])
    np.testing.assert_array_equal(sm, cgold[tag + "_sums"])


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [2, 3, 4, 5])
def test_executor_tuple_keys_match_reference(cuda, cgold, nc):
    from numfast_b200 import executor, ir
    tag = "hash%d" % nc
    jobs = [ir.ir_series("k%d" % i, cgold["%s_k%d" % (tag, i)], "int32", cgold[tag + "_kval"] if i == 0 else None)
            for i in range(nc)]
    jobs += [ir.ir_series("v", cgold[tag + "_v"], "int32", cgold[tag + "_vval"]),
             ir.ir_pack_keys("K", *["k%d" % i for i in range(nc)], mode="hash"),
             ir.ir_groupby_multi("G", "v", "K", ("sum", "count"), result="carry")]
    c = executor.execute(jobs)["G"]
    np.testing.assert_array_equal(np.asarray([list(t) for t in c.ukeys]), cgold[tag + "_ukeys"])
    np.testing.assert_array_equal(c.counts, cgold[tag + "_counts"])
    np.testing.assert_array_equal(c.sums["v"], cgold[tag + "_sums"])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["pack", "radix"])
def test_executor_packed_keys_match_reference(cuda, cgold, mode):
    from numfast_b200 import executor, ir
    a, b = (cgold["pack_hi"], cgold["pack_lo"]) if mode == "pack" else (cgold["radix_c0"], cgold["radix_c1"])
    jobs = [ir.ir_series("a", a, "int32"), ir.ir_series("b", b, "int32"), ir.ir_series("v", cgold["pack_v"], "int32"),
            ir.ir_pack_keys("K", "a", "b", mode=mode),
            ir.ir_groupby_multi("G", "v", "K", ("sum", "count"), result="carry")]
    c = executor.execute(jobs)["G"]
    np.testing.assert_array_equal(np.asarray(c.ukeys, dtype=np.int64), cgold[mode + "_ukeys"])
    np.testing.assert_array_equal(c.sums["v"], cgold[mode + "_sums"])


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [2, 3, 4, 6])
def test_device_composite_large(cuda, nc):
    """2M rows, wide key ranges (full int32 in one column), NULL keys and values."""
    import torch
    from numfast_b200 import device as dev
    rs = np.random.default_rng(40 + nc)
    n = 2_000_000
    cols = [rs.integers(-300, 300, n).astype(np.int32) for _ in range(nc)]
    cols[1] = rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32) % 97 * 44_000_000  # wide, repeated
    v = rs.integers(-1000, 1001, n).astype(np.int32)
    kval = rs.random(n) > 0.03
    vval = rs.random(n) > 0.03
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    r = dev.groupby_composite([t(c) for c in cols], [dev.DeviceColumn("v", t(v), ("sum",), t(dev.pack_validity(vval)))],
                              t(dev.pack_validity(kval)))
    uk, cnt, sm = O.composite_groupby_sum_count(cols, v, kval & vval)
    got = np.stack([c.cpu().numpy().astype(np.int64) for c in r.key_columns], axis=1)
    np.testing.assert_array_equal(got, uk)
    np.testing.assert_array_equal(r.counts.cpu().numpy(), cnt)
    np.testing.assert_array_equal(r.sums["v"].cpu().numpy(), sm)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["full_range", "constant", "single", "min_max"])
def test_device_composite_packing_widths(cuda, kind):
    """A pair is packed into the bit widths of its two ranges: full-width (64-bit words),
    zero-width and single-row cases, the int32 extremes, with and without NULL keys."""
    import torch
    from numfast_b200 import device as dev
    rs = np.random.default_rng(77)
    n = 300_000
    if kind == "full_range":
        a = (rs.integers(0, 3000, n) * 1_431_655 - 2 ** 31).astype(np.int32)
        b = rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)
        b[500:] = b[:n - 500] % 11
        a[:2], b[:2] = [-2 ** 31, 2 ** 31 - 1], [2 ** 31 - 1, -2 ** 31]
    elif kind == "constant":
        a = np.full(n, 2 ** 31 - 1, np.int32)
        b = np.full(n, -2 ** 31, np.int32)
    elif kind == "single":
        a = np.array([-2 ** 31], np.int32)
        b = np.array([2 ** 31 - 1], np.int32)
    else:
        ext = np.array([-2 ** 31, -1, 0, 2 ** 31 - 1], np.int64)
        a = rs.choice(ext, n).astype(np.int32)
        b = rs.choice(ext, n).astype(np.int32)
    v = rs.integers(-1000, 1001, a.size).astype(np.int32)
    kval = rs.random(a.size) > 0.05
    kval[0] = True
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    for bm in (None, kval):
        r = dev.groupby_composite([t(a), t(b)], [dev.DeviceColumn("v", t(v), ("sum",))],
                                  t(dev.pack_validity(bm)) if bm is not None else None)
        uk, cnt, sm = O.composite_groupby_sum_count([a, b], v, bm)
        got = np.stack([c.cpu().numpy().astype(np.int64) for c in r.key_columns], axis=1)
        np.testing.assert_array_equal(got, uk)
        np.testing.assert_array_equal(r.counts.cpu().numpy(), cnt)
        np.testing.assert_array_equal(r.sums["v"].cpu().numpy(), sm)


@pytest.mark.gpu
@pytest.mark.parametrize("nc,bits", [(2, 24), (3, 30), (4, 31), (5, 20), (8, 31), (2, 32), (3, 33)])
def test_device_bit_packed_keys(cuda, nc, bits):
    """Tuples whose flipped ranges fit in 31 bits take the bit-packed int32 key (no sort);
    32+ bits fall back to the sorted folds.  Both give the reference's composite order."""
    import torch
    from numfast_b200 import device as dev
    rs = np.random.default_rng(bits * 10 + nc)
    n = 500_000
    per = [bits // nc + (1 if i < bits % nc else 0) for i in range(nc)]
    cols = []
    for i, w in enumerate(per):
        lo = -(1 << (w - 1)) if i % 2 == 0 else 17  # signed ranges around 0, unsigned-ish offsets
        c = rs.integers(lo, lo + (1 << w), n).astype(np.int32)
        c[i] = lo
        c[i + nc] = lo + (1 << w) - 1  # hit both ends: the range is exactly w bits
        cols.append(c)
    v = rs.integers(-1000, 1001, n).astype(np.int32)
    kval = rs.random(n) > 0.02
    kval[: 2 * nc] = True
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    plan = dev.composite_order_plan(nc)
    lay = dev.key_bits_layout([t(cols[c]) for c, _ in plan], [f for _, f in plan], t(dev.pack_validity(kval)))
    # Flipped ranges of unsigned-ordered columns are the same widths as signed here.
    assert (lay is not None) == (bits <= 31)
    r = dev.groupby_composite([t(c) for c in cols], [dev.DeviceColumn("v", t(v), ("sum",))],
                              t(dev.pack_validity(kval)))
    uk, cnt, sm = O.composite_groupby_sum_count(cols, v, kval)
    got = np.stack([c.cpu().numpy().astype(np.int64) for c in r.key_columns], axis=1)
    np.testing.assert_array_equal(got, uk)
    np.testing.assert_array_equal(r.counts.cpu().numpy(), cnt)
    np.testing.assert_array_equal(r.sums["v"].cpu().numpy(), sm)


def test_bit_plan_orders_match_oracle():
    """composite_order_plan restates the fold orders: sorting the tuples by the plan's
    flipped columns gives the oracle's composite order (CPU only)."""
    from numfast_b200 import device as dev
    rs = np.random.default_rng(9)
    for nc in (2, 3, 4, 5, 7):
        cols = [rs.integers(-4, 4, 3000).astype(np.int32) for _ in range(nc)]
        plan = dev.composite_order_plan(nc)
        keys = [(cols[c].view(np.uint32) ^ np.uint32(f)) for c, f in reversed(plan)]
        order = np.lexsort(keys)
        want = O.composite_order(cols)
        tup = lambda o: [tuple(int(cols[c][i]) for c in range(nc)) for i in o]  # noqa: E731
        assert tup(order) == tup(want)
