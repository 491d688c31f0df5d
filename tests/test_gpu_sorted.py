"""SORTED strategy: group-by over nondecreasing keys (one pass over runs), against the oracle.

The reference takes its sorted plan whenever the valid keys are nondecreasing
(src/Runtime/Planner/_lib/planner.py:226) and reduces runs in order
(groupindex.py:259-304, sorted.rs:24-56).  These tests force strategy "sorted" on sorted
inputs with NULLs in every column, at tile edges (16,384 rows per tile, 2,048 per warp
chunk), with runs far
longer than a tile, and at 100M rows.
"""

import numpy as np
import pytest
import torch

from numfast_b200 import device as dev
from oracle import nf_oracle as O
from tests.gpu_util import OPS, assert_carry_equal, device_groupby, to_dev

pytestmark = pytest.mark.gpu

TILE = 16384


def sorted_inputs(n, mean_run, seed, null_p=0.05, kmin=-5000):
    rs = np.random.default_rng(seed)
    if n == 0:
        k = np.zeros(0, dtype=np.int32)
    else:
        lens = rs.integers(1, 2 * mean_run + 1, n // max(mean_run, 1) + 2)
        while lens.sum() < n:
            lens = np.concatenate([lens, lens])
        k = (np.repeat(np.cumsum(rs.integers(1, 4, lens.size)), lens)[:n] + kmin).astype(np.int32)
    v = rs.integers(-1000, 1001, n).astype(np.int32)
    f = rs.lognormal(3.0, 1.0, n)
    val = {"__key__": rs.random(n) >= null_p, "v": rs.random(n) >= null_p, "f": rs.random(n) >= null_p}
    return k, {"v": v, "f": f}, val


@pytest.mark.parametrize("n", [1, 5, 130, 2049, 4099, TILE - 1, TILE, TILE + 1, 100_003, 300_000])
@pytest.mark.parametrize("mean_run", [1, 7, 5000, 40_000])
def test_sorted_cases(cuda, n, mean_run):
    k, cols, val = sorted_inputs(n, mean_run, seed=n + mean_run)
    got = device_groupby(k, cols, val, "sorted")
    assert got["strategy"] == "sorted"
    assert_carry_equal(got, O.groupby_multi(k, cols, OPS, val))


def test_sorted_auto_picks_sorted(cuda):
    k, cols, val = sorted_inputs(200_000, 13, seed=3)
    got = device_groupby(k, cols, val, "auto")
    assert got["strategy"] == "sorted"
    assert_carry_equal(got, O.groupby_multi(k, cols, OPS, val))


def test_sorted_tile_edges(cuda):
    """Runs that end exactly on a tile boundary, a run spanning many tiles, whole tiles
    of NULL rows (the last valid key must reach across them), NULL leading rows."""
    n = 12 * TILE + 777
    k = np.zeros(n, dtype=np.int32)
    k[:TILE] = np.repeat(np.arange(TILE // 64), 64)           # runs end on the boundary
    k[TILE:5 * TILE + 100] = 10_000                            # one run over four tiles
    k[5 * TILE + 100:] = 10_001 + np.arange(n - 5 * TILE - 100) // 3000
    rs = np.random.default_rng(4)
    v = rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)
    f = rs.standard_normal(n)
    kv = rs.random(n) > 0.05
    kv[:50] = False                                            # leading NULLs
    kv[6 * TILE:9 * TILE + 5] = False                          # three NULL tiles, mid-run
    val = {"__key__": kv, "v": rs.random(n) > 0.05}
    got = device_groupby(k, {"v": v, "f": f}, val, "sorted")
    assert got["strategy"] == "sorted"
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, val))


@pytest.mark.parametrize("n", [1, 1000, 5 * TILE + 3, 3_000_000])
def test_sorted_all_one_key(cuda, n):
    rs = np.random.default_rng(n)
    k = np.full(n, -7, dtype=np.int32)
    v = rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)
    f = rs.standard_normal(n)
    val = {"f": rs.random(n) > 0.5}
    got = device_groupby(k, {"v": v, "f": f}, val, "sorted")
    assert got["strategy"] == "sorted"
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, val))


def test_sorted_all_null_and_empty(cuda):
    k = np.arange(70_000, dtype=np.int32)
    got = device_groupby(k, {"v": k.copy(), "f": np.ones(k.size)}, {"v": np.zeros(k.size, bool)}, "sorted")
    assert got["ukeys"].size == 0
    got = device_groupby(np.zeros(0, np.int32), {"v": np.zeros(0, np.int32), "f": np.zeros(0)}, {}, "sorted")
    assert got["ukeys"].size == 0


def test_sorted_hint_on_unsorted_input(cuda):
    """SORTED on keys that are not sorted is only a hint: another strategy runs."""
    rs = np.random.default_rng(8)
    k = rs.integers(0, 5000, 100_000).astype(np.int32)
    v = rs.integers(-1000, 1001, k.size).astype(np.int32)
    f = rs.standard_normal(k.size)
    got = device_groupby(k, {"v": v, "f": f}, {}, "sorted")
    assert got["strategy"] != "sorted"
    assert_carry_equal(got, O.groupby_multi(k, {"v": v, "f": f}, OPS, {}))


@pytest.mark.parametrize("shape", ["count", "i32", "i64", "f64", "six"])
def test_sorted_column_shapes(cuda, shape):
    rs = np.random.default_rng(31)
    n = 400_000
    k = np.sort(rs.integers(-2 ** 31, 2 ** 31, n)).astype(np.int32)
    k[1000:90_000] = k[1000]                                   # a run over several tiles
    k = np.sort(k)
    if shape == "count":
        cols = {}
    elif shape == "i32":
        cols = {"v": rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)}
    elif shape == "i64":
        cols = {"w": rs.integers(-2 ** 40, 2 ** 40, n).astype(np.int64)}
    elif shape == "f64":
        f = rs.lognormal(3.0, 1.0, n)
        f[rs.random(n) < 0.01] = np.nan
        f[rs.random(n) < 0.01] = -0.0
        f[rs.random(n) < 0.005] = -np.inf
        cols = {"f": f}
    else:
        cols = {"c%d" % i: rs.integers(-9, 9, n).astype(np.int32) for i in range(6)}
    ops = {c: ("sum", "min", "max") for c in cols}
    val = {"__key__": rs.random(n) > 0.03}
    for c in cols:
        val[c] = rs.random(n) > 0.03
    got = device_groupby(k, cols, val, "sorted", ops=ops)
    ref = O.groupby_multi(k, cols, ops, val)
    assert_carry_equal(got, ref, float_cols=("f",))


def test_sorted_unaligned(cuda):
    rs = np.random.default_rng(5)
    n = 100_001
    base = to_dev(np.sort(rs.integers(0, 3000, n + 1)).astype(np.int32))
    vals = to_dev(rs.integers(-2 ** 40, 2 ** 40, n + 1).astype(np.int64))
    keys, v64 = base[1:], vals[1:]
    r = dev.groupby(keys, [dev.DeviceColumn("w", v64, ("sum", "min", "max"))], strategy="sorted")
    torch.cuda.synchronize()
    assert r.strategy == "sorted"
    ref = O.groupby_multi(keys.cpu().numpy(), {"w": v64.cpu().numpy()}, {"w": ("sum", "min", "max")})
    np.testing.assert_array_equal(r.ukeys.cpu().numpy(), ref["ukeys"])
    np.testing.assert_array_equal(r.counts.cpu().numpy(), ref["counts"])
    np.testing.assert_array_equal(r.sums["w"].cpu().numpy(), ref["sums"]["w"])
    np.testing.assert_array_equal(r.mins["w"].cpu().numpy(), ref["mins"]["w"])
    np.testing.assert_array_equal(r.maxs["w"].cpu().numpy(), ref["maxs"]["w"])


def _full(kd, n):
    vd = dev.rng_fill_i32(n, 42, 1, -1000, 1001)
    fd = dev.gen_lognormal(n, 42, 2, 3, 3.0, 1.0)
    bms = [dev.gen_validity(n, 42, s, 0.05) for s in (4, 5, 6)]
    r = dev.groupby(kd, [dev.DeviceColumn("v", vd, ("sum", "min", "max"), bms[1]),
                         dev.DeviceColumn("f", fd, ("sum", "min", "max"), bms[2])], bms[0], strategy="sorted")
    torch.cuda.synchronize()
    assert r.strategy == "sorted"
    k, v, f = kd.cpu().numpy(), vd.cpu().numpy(), fd.cpu().numpy()
    masks = [np.unpackbits(b.cpu().numpy(), bitorder="little")[:n].astype(bool) for b in bms]
    got = {"ukeys": r.ukeys.cpu().numpy(), "counts": r.counts.cpu().numpy(),
           "sums": {c: t.cpu().numpy() for c, t in r.sums.items()},
           "mins": {c: t.cpu().numpy() for c, t in r.mins.items()},
           "maxs": {c: t.cpu().numpy() for c, t in r.maxs.items()}}
    del r, vd, fd, bms
    ref = O.groupby_multi(k, {"v": v, "f": f}, OPS, {"__key__": masks[0], "v": masks[1], "f": masks[2]})
    assert_carry_equal(got, ref)


def test_sorted_full_size_uniform(cuda):
    """100M sorted rows over a 10M-key domain, 5% NULLs per column."""
    n = 100_000_000
    kd = torch.sort(dev.rng_fill_i32(n, 42, 0, 0, 10_000_000))[0].contiguous()
    _full(kd, n)


def test_sorted_full_size_runs_and_one_key(cuda):
    """50M rows in sorted runs of length 1..10,000, then 50M rows of one key."""
    n = 50_000_000
    lens = dev.rng_fill_i32(n // 5000 + 100, 42, 12, 1, 10001).long()
    kd = torch.repeat_interleave(torch.arange(lens.numel(), device="cuda", dtype=torch.int32) * 3 - 10 ** 6,
                                 lens)[:n].contiguous()
    _full(kd, n)
    _full(torch.full((n,), 123, dtype=torch.int32, device="cuda"), n)
