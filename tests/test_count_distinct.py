"""Grouped COUNT DISTINCT: the oracle against the reference's own results (CPU), and the
CUDA path against both (GPU), including the all-ones pair that doubles as the filler of
invalid rows."""

import os

import numpy as np
import pytest

from oracle import nf_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ("small", "nulls", "extreme", "onegroup", "empty")


@pytest.fixture(scope="module")
def dgold():
    return np.load(os.path.join(HERE, "golden", "distinct_golden.npz"))


def _case(z, tag):
    k, v = z[tag + "_k"], z[tag + "_v"]
    valid = np.ones(k.size, bool)
    if tag + "_kval" in z:
        valid &= z[tag + "_kval"]
    if tag + "_vval" in z:
        valid &= z[tag + "_vval"]
    return k, v, valid, z.get(tag + "_kval"), z.get(tag + "_vval")


@pytest.mark.parametrize("tag", CASES)
def test_oracle_matches_reference(dgold, tag):
    k, v, valid, _, _ = _case(dgold, tag)
    uk, nu = O.group_count_distinct(k, v, valid)
    np.testing.assert_array_equal(uk, dgold[tag + "_ukeys"])
    np.testing.assert_array_equal(nu, dgold[tag + "_nunique"])


@pytest.mark.gpu
@pytest.mark.parametrize("tag", CASES)
def test_device_matches_reference(cuda, dgold, tag):
    import torch
    from numfast_b200 import device as dev
    k, v, _, kval, vval = _case(dgold, tag)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    uk, nu = dev.group_count_distinct(t(k), t(v), t(dev.pack_validity(kval)) if kval is not None else None,
                                      t(dev.pack_validity(vval)) if vval is not None else None)
    np.testing.assert_array_equal(uk.cpu().numpy(), dgold[tag + "_ukeys"])
    np.testing.assert_array_equal(nu.cpu().numpy(), dgold[tag + "_nunique"])


@pytest.mark.gpu
def test_device_large_and_filler_pair(cuda):
    import torch
    from numfast_b200 import device as dev
    rs = np.random.default_rng(3)
    n = 3_000_000
    k = rs.integers(-2000, 2000, n).astype(np.int32)
    v = rs.integers(-30000, 30000, n).astype(np.int32)
    # Valid (INT32_MAX, INT32_MAX) pairs next to invalid rows (whose filler is the same bits).
    k[:100] = 2 ** 31 - 1
    v[:100] = 2 ** 31 - 1
    kval = rs.random(n) > 0.05
    kval[:50] = True
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    uk, nu = dev.group_count_distinct(t(k), t(v), t(dev.pack_validity(kval)))
    ruk, rnu = O.group_count_distinct(k, v, kval)
    np.testing.assert_array_equal(uk.cpu().numpy(), ruk)
    np.testing.assert_array_equal(nu.cpu().numpy(), rnu)


@pytest.mark.gpu
def test_executor_node(cuda, dgold):
    from numfast_b200 import executor, ir
    k, v, _, kval, vval = _case(dgold, "nulls")
    jobs = [ir.ir_series("v", v, "int32", vval), ir.ir_series("k", k, "int32", kval),
            ir.ir_count_distinct("D", "v", "k")]
    d = executor.execute(jobs)["D"]
    want = dict(zip(dgold["nulls_ukeys"].tolist(), dgold["nulls_nunique"].tolist()))
    assert d == want


@pytest.mark.gpu
def test_chain_group_with_nunique(cuda):
    """group(key, {v: (sum, nunique), w: nunique}) like the reference chain: a groupby_multi
    node plus one count-distinct node per nunique column, aligned by key; also after a
    fused filter."""
    from numfast_b200 import chain
    rs = np.random.default_rng(5)
    n = 40_000
    k = rs.integers(0, 300, n).astype(np.int32)
    v = rs.integers(-50, 50, n).astype(np.int32)
    w = rs.integers(0, 7, n).astype(np.int32)
    t = chain.from_numpy({"k": k, "v": v, "w": w})
    out = t.query().group("k", {"v": ("sum", "nunique"), "w": "nunique"}).compile()
    ref = O.groupby_multi(k, {"v": v}, {"v": ("sum",)})
    np.testing.assert_array_equal(out.column("k"), ref["ukeys"])
    np.testing.assert_array_equal(out.column("v.sum"), ref["sums"]["v"])
    np.testing.assert_array_equal(out.column("v.nunique"), O.group_count_distinct(k, v)[1])
    np.testing.assert_array_equal(out.column("w.nunique"), O.group_count_distinct(k, w)[1])
    m = v > 0
    f = t.query().filter(m).group("k", {"w": "nunique"}).compile()
    uk, nu = O.group_count_distinct(k[m], w[m])
    np.testing.assert_array_equal(f.column("k"), uk)
    np.testing.assert_array_equal(f.column("w.nunique"), nu)


def _cd_edge(kind, rs):
    n = 200_000
    if kind == "full_range":  # both halves span all of int32: a 64-bit word, 8 passes
        k = (rs.integers(0, 5000, n) * 858_993 - 2 ** 31).astype(np.int32)  # repeats within a wide range
        v = rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)
        v[1000:] = v[:n - 1000] % 3  # repeated pairs
        k[:3] = [-2 ** 31, 2 ** 31 - 1, 0]
        v[:3] = [2 ** 31 - 1, -2 ** 31, 5]
    elif kind == "constant":  # zero-width halves
        k = np.full(n, -7, np.int32)
        v = np.full(n, 2 ** 31 - 1, np.int32)
    elif kind == "const_key":
        k = np.full(n, -2 ** 31, np.int32)
        v = rs.integers(-100, 100, n).astype(np.int32)
    elif kind == "single":
        k = np.array([-2 ** 31], np.int32)
        v = np.array([-2 ** 31], np.int32)
    else:  # "min_max": only the two extremes
        k = rs.choice(np.array([-2 ** 31, 2 ** 31 - 1], np.int64), n).astype(np.int32)
        v = rs.choice(np.array([-2 ** 31, 2 ** 31 - 1], np.int64), n).astype(np.int32)
    kval = rs.random(k.size) > 0.1
    if k.size == 1:
        kval[:] = True
    return k, v, kval


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["full_range", "constant", "const_key", "single", "min_max"])
def test_device_packing_widths(cuda, kind):
    """The pair is packed into the bit widths of the key and value ranges: extremes,
    zero-width and full-width halves, with NULL rows (the filler) mixed in."""
    import torch
    from numfast_b200 import device as dev
    k, v, kval = _cd_edge(kind, np.random.default_rng(11))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    for bm in (None, kval):
        uk, nu = dev.group_count_distinct(t(k), t(v), t(dev.pack_validity(bm)) if bm is not None else None)
        ruk, rnu = O.group_count_distinct(k, v, bm)
        np.testing.assert_array_equal(uk.cpu().numpy(), ruk)
        np.testing.assert_array_equal(nu.cpu().numpy(), rnu)
