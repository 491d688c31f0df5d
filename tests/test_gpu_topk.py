"""Top-k by radix selection (nfc_sort_topk) against the full stable argsort.

The reference answers sort -> slice by sorting every row and slicing
(src/Drivers/CPU/_lib/cpu.py:3170-3200) in the order of _sort_perm (cpu.py:1154-1225):
stable ascending, descending by key-group reversal (every NaN its own group, so NaNs
first in reverse input order), NULL rows last in input order.  nfc_sort_topk must return
exactly the first k entries of that permutation: checked against the oracle's sort_perm
at sizes it handles, and against the device's full argsort (itself pinned to the oracle)
at 100M rows.  Sizes start at 65,536 rows so the selection path runs (smaller inputs and
k > n / 8 take the full argsort).
"""

import numpy as np
import pytest
import torch

from numfast_b200 import chain as C
from numfast_b200 import device as dev
from oracle import nf_oracle as O
from tests.gpu_util import bitmap, to_dev

pytestmark = pytest.mark.gpu

N = 300_000


def _keys(kind, n, rs):
    if kind == "i32":
        return rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)
    if kind == "i32_ties":
        return rs.integers(-5, 5, n).astype(np.int32)
    if kind == "i64":
        return rs.integers(-2 ** 62, 2 ** 62, n).astype(np.int64)
    if kind == "i64_ties":
        return (rs.integers(0, 40, n) * (2 ** 40) - 2 ** 45).astype(np.int64)
    f = rs.standard_normal(n) * 1e3
    if kind == "f64_special":
        f[rs.random(n) < 0.02] = np.nan
        f[rs.random(n) < 0.01] = -0.0
        f[rs.random(n) < 0.01] = 0.0
        f[rs.random(n) < 0.005] = np.inf
        f[rs.random(n) < 0.005] = -np.inf
    return f


@pytest.mark.parametrize("kind", ["i32", "i32_ties", "i64", "i64_ties", "f64", "f64_special"])
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("nulls", [False, True])
def test_topk_matches_oracle(cuda, kind, desc, nulls):
    kinds = ["i32", "i32_ties", "i64", "i64_ties", "f64", "f64_special"]
    rs = np.random.default_rng(100 + 4 * kinds.index(kind) + 2 * desc + nulls)
    k = _keys(kind, N, rs)
    valid = rs.random(N) > 0.1 if nulls else None
    ref = O.sort_perm([k], desc, valid)
    dk = to_dev(k)
    vb = bitmap(valid)
    for kk in (1, 2, 7, 100, 2048, 2049, 5000, N // 8):
        got = dev.sort_topk(dk, kk, desc, vb).cpu().numpy()
        np.testing.assert_array_equal(got, ref[:kk], err_msg="k=%d" % kk)


def test_topk_nan_block_descending(cuda):
    """Descending float64: more NaNs than k, exactly k, and fewer; the NaN block is
    the last NaN rows in reverse input order."""
    rs = np.random.default_rng(11)
    n = 200_000
    f = rs.standard_normal(n)
    nan_rows = rs.choice(n, 3000, replace=False)
    f[nan_rows] = np.nan
    ref = O.sort_perm([f], True)
    df = to_dev(f)
    for kk in (1, 50, 2999, 3000, 3001, 4000, 20_000):
        np.testing.assert_array_equal(dev.sort_topk(df, kk, True).cpu().numpy(), ref[:kk], err_msg="k=%d" % kk)


def test_topk_nulls_fill_the_tail(cuda):
    """k beyond the valid rows: every valid row sorted, then NULL rows in input order."""
    rs = np.random.default_rng(12)
    n = 500_000
    k = rs.integers(0, 1000, n).astype(np.int32)
    valid = rs.random(n) < 0.00002 * 4  # ~40 valid rows
    ref = O.sort_perm([k], False, valid)
    nv = int(valid.sum())
    for kk in (nv, nv + 1, nv + 5000, n // 8):
        got = dev.sort_topk(to_dev(k), kk, False, bitmap(valid)).cpu().numpy()
        np.testing.assert_array_equal(got, ref[:kk], err_msg="k=%d" % kk)
    allnull = np.zeros(n, bool)
    got = dev.sort_topk(to_dev(k), 100, False, bitmap(allnull)).cpu().numpy()
    np.testing.assert_array_equal(got, np.arange(100))


def test_topk_one_value_and_edges(cuda):
    n = 400_000
    k = np.full(n, 42, np.int32)
    for desc in (False, True):
        ref = O.sort_perm([k], desc)
        for kk in (1, 999, n // 8):
            np.testing.assert_array_equal(dev.sort_topk(to_dev(k), kk, desc).cpu().numpy(), ref[:kk])
    rs = np.random.default_rng(3)
    k = rs.integers(-100, 100, n).astype(np.int32)
    assert dev.sort_topk(to_dev(k), 0).numel() == 0
    ref = O.sort_perm([k], False)
    np.testing.assert_array_equal(dev.sort_topk(to_dev(k), n).cpu().numpy(), ref)   # full-sort path
    np.testing.assert_array_equal(dev.sort_topk(to_dev(k), n // 8 + 1).cpu().numpy(), ref[:n // 8 + 1])
    small = k[:1000]
    np.testing.assert_array_equal(dev.sort_topk(to_dev(small), 10).cpu().numpy(), O.sort_perm([small], False)[:10])
    with pytest.raises(ValueError):
        dev.sort_topk(to_dev(k), n + 1)


@pytest.mark.parametrize("desc", [False, True])
def test_topk_full_size(cuda, desc):
    """100M int32 keys over the full range with 5% NULLs: first 1,000 and 100,000 rows
    against the device's full argsort."""
    n = 100_000_000
    keys = dev.rng_fill_i32(n, 42, 0, -2 ** 31, 2 ** 31 - 1)
    vb = dev.gen_validity(n, 42, 1, 0.05)
    full = dev.sort_perm(keys, desc, vb)
    for kk in (1000, 100_000):
        got = dev.sort_topk(keys, kk, desc, vb)
        assert torch.equal(got, full[:kk])


def test_chain_sort_limit_uses_selection(cuda):
    """sort().limit() through the chain equals sort().compile() sliced, for one key
    (selection) and two keys (full lexsort)."""
    rs = np.random.default_rng(5)
    n = 200_000
    cols = {"a": rs.integers(-50, 50, n).astype(np.int32), "b": rs.standard_normal(n),
            "c": rs.integers(0, 10, n).astype(np.int64)}
    valid = {"a": rs.random(n) > 0.05}
    t = C.Table(cols, valid)
    for keys in (("a",), ("b",), ("a", "c")):
        for desc in (False, True):
            full = C.Chain(t).sort(*keys, desc=desc).compile()
            part = C.Chain(t).sort(*keys, desc=desc).limit(123, offset=17).compile()
            for name in cols:
                np.testing.assert_array_equal(part.columns[name], full.columns[name][17:140])


@pytest.mark.parametrize("desc", [False, True])
def test_topk_two_levels_before_candidates(cuda, desc):
    """Keys in [0, 2^20): every row shares the top 11-bit digit, so the first level leaves
    5M rows on the prefix (more than the candidate buffer) and the second level resolves the
    candidates; with NULLs, against the oracle."""
    rs = np.random.default_rng(21 + desc)
    n = 5_000_000
    k = rs.integers(0, 2 ** 20, n).astype(np.int32)
    valid = rs.random(n) > 0.05
    ref = O.sort_perm([k], desc, valid)
    dk, vb = to_dev(k), bitmap(valid)
    for kk in (1, 1000, 70_000):
        np.testing.assert_array_equal(dev.sort_topk(dk, kk, desc, vb).cpu().numpy(), ref[:kk], err_msg="k=%d" % kk)
