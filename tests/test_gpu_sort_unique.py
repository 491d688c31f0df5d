"""Sort / unique / gather / RNG parity on the GPU."""

import numpy as np
import pytest
import torch

from numfast_b200 import device as dev
from oracle import nf_oracle as O
from tests.gpu_util import bitmap, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("desc", [False, True])
def test_sort_golden(cuda, golden, desc):
    d = "desc" if desc else "asc"
    p = dev.sort_perm(to_dev(golden["sort_in_k"]), desc).cpu().numpy()
    np.testing.assert_array_equal(p, golden["sort_i32_" + d])
    p = dev.sort_perm(to_dev(golden["sort_in_k"]), desc, bitmap(golden["sort_in_val"])).cpu().numpy()
    np.testing.assert_array_equal(p, golden["sort_i32_null_" + d])
    p = dev.sort_perm(to_dev(golden["sort_in_f"]), desc).cpu().numpy()
    np.testing.assert_array_equal(p, golden["sort_f64_" + d])
    p = dev.sort_perm(to_dev(golden["sort_in_i64"]), desc).cpu().numpy()
    np.testing.assert_array_equal(p, golden["sort_i64_" + d])


def test_lexsort_golden(cuda, golden):
    p = dev.lexsort_perm([to_dev(golden["sort_lex_a"]), to_dev(golden["sort_lex_b"])], [True, False])
    np.testing.assert_array_equal(p.cpu().numpy(), golden["sort_lex"])


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.float64])
@pytest.mark.parametrize("n", [0, 1, 4095, 4097, 3_000_001])
@pytest.mark.parametrize("desc", [False, True])
def test_sort_random(cuda, dtype, n, desc):
    rs = np.random.default_rng(n + 17)
    if dtype == np.float64:
        k = rs.standard_normal(n)
        if n > 10:
            k[rs.integers(0, n, n // 10)] = np.nan
            k[rs.integers(0, n, n // 10)] = -0.0
            k[rs.integers(0, n, n // 10)] = 0.0
    elif dtype == np.int64:
        k = rs.integers(-2 ** 62, 2 ** 62, n) // (2 ** 50)
    else:
        k = rs.integers(-2 ** 31, 2 ** 31, n).astype(np.int32) >> 12
    k = k.astype(dtype)
    p = dev.sort_perm(to_dev(k), desc).cpu().numpy()
    np.testing.assert_array_equal(p, O.sort_perm([k], [desc]))


def test_sort_with_validity_random(cuda):
    rs = np.random.default_rng(3)
    n = 200_000
    k = rs.integers(-50, 50, n).astype(np.int64)
    m = rs.random(n) > 0.3
    for desc in (False, True):
        p = dev.sort_perm(to_dev(k), desc, bitmap(m)).cpu().numpy()
        np.testing.assert_array_equal(p, O.sort_perm([k], [desc], m))


def test_unique_golden(cuda, golden):
    r = dev.unique(to_dev(golden["uniq_in"]), with_inverse=True)
    np.testing.assert_array_equal(r["uniq"].cpu().numpy(), golden["uniq_u"])
    np.testing.assert_array_equal(r["inverse"].cpu().numpy(), golden["uniq_inv"])


@pytest.mark.parametrize("case", ["full_range", "runs", "long_runs", "tiny"])
def test_unique_first_count(cuda, case):
    rs = np.random.default_rng(11)
    if case == "full_range":
        k = rs.integers(-2 ** 31, 2 ** 31, 5_000_000).astype(np.int32)
    elif case == "long_runs":
        # Too many distinct keys for the shared-hash path, and sorted runs
        # longer than a run tile (whole tiles without a run head).
        vals = rs.integers(-2 ** 31, 2 ** 31, 6000).astype(np.int32)
        lens = rs.integers(1, 12001, 3000)
        k = np.repeat(vals[rs.integers(0, 6000, lens.size)], lens).astype(np.int32)
    elif case == "runs":
        vals = rs.integers(-2 ** 31, 2 ** 31, 1000).astype(np.int32)
        lens = rs.integers(1, 10001, 800)
        k = np.repeat(vals[rs.integers(0, 1000, lens.size)], lens).astype(np.int32)
    else:
        k = np.array([5, -1, 5, 5, 2 ** 31 - 1, -2 ** 31, -1], dtype=np.int32)
    r = dev.unique(to_dev(k), with_inverse=True)
    u, first, counts = O.unique_first_count(k)
    np.testing.assert_array_equal(r["uniq"].cpu().numpy(), u)
    np.testing.assert_array_equal(r["first"].cpu().numpy(), first)
    np.testing.assert_array_equal(r["counts"].cpu().numpy(), counts)
    inv = r["inverse"].cpu().numpy()
    np.testing.assert_array_equal(u[inv], k)


def test_gather_bounds(cuda):
    v = to_dev(np.arange(10, dtype=np.int64) * 3)
    idx = to_dev(np.array([9, 0, 4], dtype=np.int32))
    assert dev.gather(v, idx).cpu().tolist() == [27, 0, 12]
    from numfast_b200 import NativeError
    with pytest.raises(NativeError):
        dev.gather(v, to_dev(np.array([10], dtype=np.int32)))


@pytest.mark.parametrize("i", range(4))
def test_rng_i32_golden(cuda, golden, i):
    n, seed, stream, off, lo, hi = (int(x) for x in golden["rng_i32_%d_args" % i])
    got = dev.rng_fill_i32(n, seed, stream, lo, hi, off).cpu().numpy()
    np.testing.assert_array_equal(got, golden["rng_i32_%d" % i])


@pytest.mark.parametrize("i", range(2))
def test_rng_f64_golden(cuda, golden, i):
    n, seed, stream, off, lo, hi = golden["rng_f64_%d_args" % i]
    got = dev.rng_fill_f64(int(n), int(seed), int(stream), lo, hi, int(off)).cpu().numpy()
    np.testing.assert_array_equal(got, golden["rng_f64_%d" % i])


def test_rng_large_matches_oracle(cuda):
    n = 1 << 20
    np.testing.assert_array_equal(dev.rng_fill_i32(n, 42, 0, 0, 10_000_000).cpu().numpy(),
                                  O.fill_i32(n, 42, 0, 0, 0, 10_000_000))
    np.testing.assert_array_equal(dev.rng_fill_f64(n, 42, 4).cpu().numpy(), O.fill_f64(n, 42, 4))
    bm = dev.gen_validity(n, 42, 4, 0.05).cpu().numpy()
    np.testing.assert_array_equal(np.unpackbits(bm, bitorder="little")[:n].astype(bool), O.fill_f64(n, 42, 4) >= 0.05)


@pytest.mark.parametrize("kind", ["unique_full", "unique_runs"])
def test_unique_config3_full_size(cuda, kind):
    """200M keys: size-independent properties (sorted distinct keys, counts sum to n, every
    first-occurrence row holds its key and no earlier row does, oracle on a prefix)."""
    import bench
    keys = bench.make_unique_keys(kind, 200_000_000, "cuda")
    r = dev.unique(keys, with_inverse=True)
    u, first, counts, inv = r["uniq"], r["first"], r["counts"], r["inverse"]
    assert bool((u[1:] > u[:-1]).all())
    assert int(counts.sum()) == keys.numel()
    assert bool((keys[first.long()] == u).all())
    if kind == "unique_runs":
        assert r["ng"] <= 1000
    # Over all 200M rows: every row's code points at its key, each code's first row is
    # the earliest row holding it (a scatter-min of row numbers by code), and the counts
    # are the code histogram.
    n, ng = keys.numel(), r["ng"]
    il = inv.long()
    assert bool((u[il] == keys).all())
    earliest = torch.full((ng,), n, dtype=torch.int64, device=keys.device)
    earliest.scatter_reduce_(0, il, torch.arange(n, device=keys.device), reduce="amin")
    assert bool((earliest == first.long()).all())
    del earliest
    assert bool((torch.bincount(il, minlength=ng) == counts).all())
    del il, inv
    # first occurrence: a row before first[i] holding u[i] would make first[i] wrong;
    # check through the oracle on the first 2M keys.
    k_small = keys[:2_000_000].cpu().numpy()
    rs = dev.unique(keys[:2_000_000].contiguous())
    uo, fo, co = O.unique_first_count(k_small)
    np.testing.assert_array_equal(rs["uniq"].cpu().numpy(), uo)
    np.testing.assert_array_equal(rs["first"].cpu().numpy(), fo)
    np.testing.assert_array_equal(rs["counts"].cpu().numpy(), co)
