"""Group-by parity: the CUDA path against the oracle, every strategy and edge case."""

import numpy as np
import pytest
import torch

from numfast_b200 import device as dev
from oracle import nf_oracle as O
from tests.gpu_util import OPS, assert_carry_equal, cfg2_inputs, device_groupby, to_dev

pytestmark = pytest.mark.gpu

STRATS = ["auto", "dense_smem", "dense_global", "partition", "hash", "shared_hash", "sort"]


@pytest.mark.parametrize("strategy", STRATS)
@pytest.mark.parametrize("n,span,kmin", [(1, 1, 0), (5, 3, -2), (130, 40, 7), (4099, 1000, 0),
                                         (100_003, 2000, -1000)])
def test_small_cases(cuda, strategy, n, span, kmin):
    k, cols, val = cfg2_inputs(n, span, seed=n, kmin=kmin)
    got = device_groupby(k, cols, val, strategy)
    ref = O.groupby_multi(k, cols, OPS, val)
    assert_carry_equal(got, ref)


@pytest.mark.parametrize("strategy", ["auto", "dense_global", "partition", "hash", "shared_hash", "sort"])
def test_medium_span(cuda, strategy):
    k, cols, val = cfg2_inputs(2_000_000, 300_000, seed=3)
    got = device_groupby(k, cols, val, strategy)
    assert_carry_equal(got, O.groupby_multi(k, cols, OPS, val))


@pytest.mark.parametrize("n,span", [(50_000, 20_000_000), (300_000, 20_000_000), (2_000_001, 12_000_000)])
def test_partition_wide_two_level(cuda, n, span):
    """Two-level scatter over many coarse buckets: refine tiles that span more
    than 256 fine buckets (sparse rows) and tiles inside one or two."""
    k, cols, val = cfg2_inputs(n, span, seed=11, kmin=-span // 2)
    got = device_groupby(k, cols, val, "partition")
    assert_carry_equal(got, O.groupby_multi(k, cols, OPS, val))


def _shape_cols(shape, n, rs):
    if shape == "count":
        return {}
    if shape == "i32":
        return {"v": rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)}
    if shape == "i64":
        return {"w": rs.integers(-2 ** 40, 2 ** 40, n).astype(np.int64)}  # sums exact in the reference (< 2^53)
    if shape == "f64":
        f = rs.lognormal(3.0, 1.0, n)
        f[rs.random(n) < 0.01] = np.nan
        f[rs.random(n) < 0.01] = -0.0
        f[rs.random(n) < 0.005] = -np.inf
        return {"f": f}
    return {"a": rs.integers(-1000, 1001, n).astype(np.int32), "b": rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)}


@pytest.mark.parametrize("shape", ["count", "i32", "i64", "f64", "i32x2"])
@pytest.mark.parametrize("span", [1_500_000, 100_000])
def test_partition_aggregate_shapes(cuda, shape, span):
    """Record shapes of one or two words, sparse (about 1 row per key: the
    sorted aggregate, with a few hot keys reduced by whole warps and split
    over several slices) and dense (15 rows per key: the shared-state one)."""
    rs = np.random.default_rng(21)
    n = 1_500_000
    k = rs.integers(0, span, n).astype(np.int32)
    hot = rs.random(n) < 0.2
    k[hot] = rs.integers(0, 6, int(hot.sum())) * (span // 6)
    cols = _shape_cols(shape, n, rs)
    ops = {c: ("sum", "min", "max") for c in cols}
    val = {"__key__": rs.random(n) > 0.03}
    for c in cols:
        val[c] = rs.random(n) > 0.03
    got = device_groupby(k, cols, val, "partition", ops=ops)
    ref = O.groupby_multi(k, cols, ops, val)
    assert_carry_equal(got, ref)


@pytest.mark.parametrize("val", [32767, -32767, 32768, -32768])
def test_partition_int32_sum_range_edges(cuda, val):
    """A hot key over several 65,536-row slices whose int32 values sit on
    either side of the +-32767 bound of the one-atomic sum."""
    n = 300_000
    k = np.zeros(n, dtype=np.int32)
    k[::7] = np.arange(0, n, 7, dtype=np.int32) * 11
    v = np.full(n, val, dtype=np.int32)
    v[1::5] = -val if abs(val) < 32768 else 7
    cols = {"v": v}
    ops = {"v": ("sum", "min", "max")}
    got = device_groupby(k, cols, {}, "partition", ops=ops)
    assert_carry_equal(got, O.groupby_multi(k, cols, ops, {}))


def test_partition_multi_slice_zipf(cuda):
    """Skewed keys: one bucket far larger than a slice -> split-and-merge path."""
    n = 3_000_000
    kd = dev.gen_zipf(n, 42, 7, 1.1, 1_000_000)
    k = kd.cpu().numpy()
    v = O.fill_i32(n, 42, 1, 0, -1000, 1001)
    f = O.fill_f64(n, 42, 2, 0, 0.0, 10.0)
    val = {"v": O.fill_f64(n, 42, 5) >= 0.05}
    got = device_groupby(k, {"v": v, "f": f}, val, "partition")
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, val))


@pytest.mark.parametrize("strategy", ["auto", "hash", "dense_global", "shared_hash", "sort"])
def test_extreme_keys(cuda, strategy):
    k = np.array([2 ** 31 - 1, -2 ** 31, 0, 2 ** 31 - 1, -2 ** 31, 5], dtype=np.int32)
    v = np.array([2 ** 31 - 1, 2 ** 31 - 1, -2 ** 31, 1, -2 ** 31, 0], dtype=np.int32)
    f = np.array([1.0, np.nan, -0.5, np.inf, 2.0, -np.inf])
    if strategy == "dense_global":
        k = k[2:]; v = v[2:]; f = f[2:]
        k = np.array([3, 3, 9, 0], dtype=np.int32)
    got = device_groupby(k, {"v": v, "f": f}, {}, strategy)
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, {}))


def test_sparse_full_range(cuda):
    rs = np.random.default_rng(1)
    k = rs.integers(-2 ** 31, 2 ** 31, 500_000).astype(np.int32)
    k = np.concatenate([k, k[:100_000]])
    v = rs.integers(-2 ** 31, 2 ** 31, k.size).astype(np.int32)
    f = rs.standard_normal(k.size)
    val = {"__key__": rs.random(k.size) > 0.1, "f": rs.random(k.size) > 0.1}
    got = device_groupby(k, {"v": v, "f": f}, val)
    assert got["strategy"] == "hash"
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, val))


@pytest.mark.parametrize("strategy", ["shared_hash", "sort"])
def test_sparse_low_cardinality_strategies(cuda, strategy):
    """Few distinct keys spread over the whole int32 range, long runs of one key, and
    a hot key with more than 65,536 rows (the shared tables' 16-bit split sums must be
    flushed in time)."""
    rs = np.random.default_rng(5)
    pool = rs.integers(-2 ** 31, 2 ** 31, 300).astype(np.int32)
    k = np.concatenate([pool[rs.integers(0, 300, 400_000)], np.repeat(pool[:3], 90_000),
                        np.full(200_000, pool[7], np.int32)])
    v = rs.integers(-2 ** 31, 2 ** 31, k.size).astype(np.int32)
    f = np.exp(rs.standard_normal(k.size)) * 10.0  # positive: sums without cancellation
    val = {"__key__": rs.random(k.size) > 0.05, "v": rs.random(k.size) > 0.05}
    got = device_groupby(k, {"v": v, "f": f}, val, strategy)
    assert got["strategy"] == strategy
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, val))


def test_shared_hash_low_hint_retries_exactly(cuda):
    """A distinct hint far too low overflows the shared strategy's global table; the
    pass stops and is repeated with a full-size table, and the result stays exact."""
    rs = np.random.default_rng(6)
    k = rs.integers(-2 ** 31, 2 ** 31, 1_200_000).astype(np.int32)
    v = rs.integers(-1000, 1001, k.size).astype(np.int32)
    kd, vd = to_dev(k), to_dev(v)
    r = dev.groupby(kd, [dev.DeviceColumn("v", vd, ("sum", "min", "max"))], strategy="shared_hash",
                    distinct_hint=10)
    torch.cuda.synchronize()
    assert r.probe["overflowed"] == 1
    ref = O.groupby_multi(k, {"v": v}, {"v": ("sum", "count", "min", "max")})
    np.testing.assert_array_equal(r.ukeys.cpu().numpy(), ref["ukeys"])
    np.testing.assert_array_equal(r.counts.cpu().numpy(), ref["counts"])
    np.testing.assert_array_equal(r.sums["v"].cpu().numpy(), ref["sums"]["v"])
    np.testing.assert_array_equal(r.mins["v"].cpu().numpy(), ref["mins"]["v"])
    r2 = dev.groupby(kd, [dev.DeviceColumn("v", vd, ("sum", "min", "max"))], strategy="shared_hash",
                     distinct_hint=400_000)
    torch.cuda.synchronize()
    assert not r2.probe["overflowed"]
    np.testing.assert_array_equal(r2.sums["v"].cpu().numpy(), ref["sums"]["v"])


def test_empty_and_all_invalid(cuda):
    k = np.zeros(0, dtype=np.int32)
    got = device_groupby(k, {"v": np.zeros(0, np.int32), "f": np.zeros(0)}, {})
    assert got["ukeys"].size == 0
    k = np.arange(1000, dtype=np.int32)
    val = {"v": np.zeros(1000, dtype=bool)}
    got = device_groupby(k, {"v": k.copy(), "f": np.ones(1000)}, val)
    assert got["ukeys"].size == 0 and got["counts"].size == 0


def test_unaligned_and_int64_columns(cuda):
    rs = np.random.default_rng(5)
    n = 10_001
    base = to_dev(rs.integers(0, 300, n + 1).astype(np.int32))
    vals = to_dev(rs.integers(-2 ** 40, 2 ** 40, n + 1).astype(np.int64))
    keys = base[1:]   # 4-byte aligned, not 16
    v64 = vals[1:]    # 8-byte aligned, not 16
    r = dev.groupby(keys, [dev.DeviceColumn("w", v64, ("sum", "min", "max"))])
    torch.cuda.synchronize()
    k_np, w_np = keys.cpu().numpy(), v64.cpu().numpy()
    ref = O.groupby_multi(k_np, {"w": w_np}, {"w": ("sum", "min", "max")})
    np.testing.assert_array_equal(r.ukeys.cpu().numpy(), ref["ukeys"])
    np.testing.assert_array_equal(r.sums["w"].cpu().numpy(), ref["sums"]["w"])
    np.testing.assert_array_equal(r.mins["w"].cpu().numpy(), ref["mins"]["w"])
    np.testing.assert_array_equal(r.maxs["w"].cpu().numpy(), ref["maxs"]["w"])


def test_more_than_four_columns(cuda):
    rs = np.random.default_rng(9)
    n = 50_000
    k = rs.integers(0, 5000, n).astype(np.int32)
    cols = {"c%d" % i: rs.integers(-9, 9, n).astype(np.int32) for i in range(6)}
    val = {"c3": rs.random(n) > 0.2}
    ops = {c: ("sum", "max") for c in cols}
    got = device_groupby(k, cols, val, ops=ops)
    ref = O.groupby_multi(k, cols, ops, val)
    assert_carry_equal(got, ref, float_cols=())


def test_golden_through_device(cuda, golden):
    for tag in ["gb_dense", "gb_sparse", "gb_bound", "gb_sorted", "gb_nan"]:
        k = golden[tag + "_in_k"]
        cols = {"v": golden[tag + "_in_v"], "f": golden[tag + "_in_f"]}
        val = {"__key__": golden[tag + "_in_kval"], "v": golden[tag + "_in_vval"], "f": golden[tag + "_in_fval"]}
        got = device_groupby(k, cols, val)
        np.testing.assert_array_equal(got["ukeys"], golden[tag + "_ukeys"])
        np.testing.assert_array_equal(got["counts"], golden[tag + "_counts"])
        np.testing.assert_array_equal(got["sums"]["v"], golden[tag + "_v_sum"])
        np.testing.assert_array_equal(got["mins"]["v"], golden[tag + "_v_min"])
        np.testing.assert_array_equal(got["maxs"]["v"], golden[tag + "_v_max"])
        np.testing.assert_allclose(got["sums"]["f"], golden[tag + "_f_sum"], rtol=1e-12, equal_nan=True)
        np.testing.assert_array_equal(got["mins"]["f"], golden[tag + "_f_min"])
        np.testing.assert_array_equal(got["maxs"]["f"], golden[tag + "_f_max"])


def test_full_size_cfg2a(cuda):
    """100M rows, 10M-key domain, 5% NULLs per column: oracle parity at full size."""
    n, span = 100_000_000, 10_000_000
    kd = dev.rng_fill_i32(n, 42, 0, 0, span)
    vd = dev.rng_fill_i32(n, 42, 1, -1000, 1001)
    fd = dev.gen_lognormal(n, 42, 2, 3, 3.0, 1.0)
    bms = [dev.gen_validity(n, 42, s, 0.05) for s in (4, 5, 6)]
    r = dev.groupby(kd, [dev.DeviceColumn("v", vd, ("sum", "min", "max"), bms[1]),
                         dev.DeviceColumn("f", fd, ("sum", "min", "max"), bms[2])], bms[0])
    torch.cuda.synchronize()
    assert r.strategy == "partition"
    k, v, f = kd.cpu().numpy(), vd.cpu().numpy(), fd.cpu().numpy()
    masks = [np.unpackbits(b.cpu().numpy(), bitorder="little")[:n].astype(bool) for b in bms]
    del kd, vd, fd
    ref = O.groupby_multi(k, {"v": v, "f": f}, OPS, {"__key__": masks[0], "v": masks[1], "f": masks[2]})
    got = {"ukeys": r.ukeys.cpu().numpy(), "counts": r.counts.cpu().numpy(),
           "sums": {c: t.cpu().numpy() for c, t in r.sums.items()},
           "mins": {c: t.cpu().numpy() for c, t in r.mins.items()},
           "maxs": {c: t.cpu().numpy() for c, t in r.maxs.items()}}
    assert_carry_equal(got, ref)


def test_full_size_cfg2b(cuda):
    """100M rows, keys Zipf(s=1.1) over a 50M-key domain, 5% NULLs per column:
    oracle parity at full size (hot keys split over many slices)."""
    n, dom = 100_000_000, 50_000_000
    kd = dev.gen_zipf(n, 42, 7, 1.1, dom)
    vd = dev.rng_fill_i32(n, 42, 1, -1000, 1001)
    fd = dev.gen_lognormal(n, 42, 2, 3, 3.0, 1.0)
    bms = [dev.gen_validity(n, 42, s, 0.05) for s in (4, 5, 6)]
    r = dev.groupby(kd, [dev.DeviceColumn("v", vd, ("sum", "min", "max"), bms[1]),
                         dev.DeviceColumn("f", fd, ("sum", "min", "max"), bms[2])], bms[0])
    torch.cuda.synchronize()
    k, v, f = kd.cpu().numpy(), vd.cpu().numpy(), fd.cpu().numpy()
    masks = [np.unpackbits(b.cpu().numpy(), bitorder="little")[:n].astype(bool) for b in bms]
    del kd, vd, fd
    ref = O.groupby_multi(k, {"v": v, "f": f}, OPS, {"__key__": masks[0], "v": masks[1], "f": masks[2]})
    got = {"ukeys": r.ukeys.cpu().numpy(), "counts": r.counts.cpu().numpy(),
           "sums": {c: t.cpu().numpy() for c, t in r.sums.items()},
           "mins": {c: t.cpu().numpy() for c, t in r.mins.items()},
           "maxs": {c: t.cpu().numpy() for c, t in r.maxs.items()}}
    assert_carry_equal(got, ref)


@pytest.mark.parametrize("strategy", STRATS)
def test_fused_row_filter_matches_filter_then_group(cuda, strategy):
    """A row-filter bitmap fused into the group-by gives exactly the group-by of the rows
    the filter keeps (the reference runs a filter node, then groupby_multi)."""
    n = 300_007
    k, cols, val = cfg2_inputs(n, 20_000, seed=9, kmin=-100)
    keep = O.fill_f64(n, 9, 8) >= 0.4
    dcols = [dev.DeviceColumn(c, to_dev(v), tuple(o for o in OPS[c] if o != "count"),
                              to_dev(dev.pack_validity(val[c])) if c in val else None) for c, v in cols.items()]
    r = dev.groupby(to_dev(k), dcols, to_dev(dev.pack_validity(val["__key__"])), strategy=strategy,
                    row_filter=to_dev(dev.pack_validity(keep)))
    torch.cuda.synchronize()
    got = {"ukeys": r.ukeys.cpu().numpy(), "counts": r.counts.cpu().numpy(),
           "sums": {c: t.cpu().numpy() for c, t in r.sums.items()},
           "mins": {c: t.cpu().numpy() for c, t in r.mins.items()},
           "maxs": {c: t.cpu().numpy() for c, t in r.maxs.items()}}
    ref = O.groupby_multi(k[keep], {c: v[keep] for c, v in cols.items()}, OPS,
                          {c: m[keep] for c, m in val.items()})
    assert_carry_equal(got, ref)


@pytest.mark.parametrize("strategy", ["dense_global", "hash", "shared_hash"])
@pytest.mark.parametrize("case", ["zipf2", "hot_key", "runs"])
def test_warp_aggregated_skew(cuda, strategy, case):
    """Skewed keys through the warp-aggregated atomics: Zipf(s=2) (most rows on a few
    keys), one key holding 60% of the rows, and runs of one key (every lane of a warp
    on the same address) -- with NULLs, int32 extremes and float64 NaN/-0.0."""
    n = 1_000_003
    rs = np.random.default_rng(77)
    if case == "zipf2":
        k = dev.gen_zipf(n, 42, 7, 2.0, 200_000).cpu().numpy()
    elif case == "hot_key":
        k = rs.integers(0, 100_000, n).astype(np.int32)
        k[rs.random(n) < 0.6] = 4242
    else:
        k = np.repeat(rs.integers(0, 50_000, n // 300 + 1), 300)[:n].astype(np.int32)
        k[::2] = k[::2][::-1]  # not sorted, still one key per run of lanes
    k = (k.astype(np.int64) * (1 if strategy == "dense_global" else 9973) - 12345).astype(np.int32)
    v = rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)
    f = rs.lognormal(1.0, 1.0, n)
    f[rs.random(n) < 1e-4] = np.nan
    f[rs.random(n) < 1e-3] = -0.0
    val = {"__key__": rs.random(n) > 0.05, "v": rs.random(n) > 0.05, "f": rs.random(n) > 0.05}
    got = device_groupby(k, {"v": v, "f": f}, val, strategy)
    assert got["strategy"] == strategy
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, val))


@pytest.mark.parametrize("strategy", ["dense_global", "hash", "shared_hash"])
def test_warp_aggregated_int64_and_many_groups(cuda, strategy):
    """int64 columns (64-bit warp reductions) and warps holding more groups of equal
    keys than one call reduces (the remaining lanes apply their own rows)."""
    n = 500_000
    rs = np.random.default_rng(78)
    k = rs.integers(0, 12, n).astype(np.int32) * 1000  # ~12 keys per warp: beyond the reduced groups
    w = rs.integers(-2 ** 40, 2 ** 40, n).astype(np.int64)
    val = {"w": rs.random(n) > 0.1}
    ops = {"w": ("sum", "min", "max")}
    got = device_groupby(k, {"w": w}, val, strategy, ops=ops)
    assert got["strategy"] == strategy
    assert_carry_equal(got, O.groupby_multi(k, {"w": w}, ops, val), float_cols=())
