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
