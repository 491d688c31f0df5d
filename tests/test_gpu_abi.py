"""The numfast-native ABI (host buffers) served by the GPU, against the oracle."""

import ctypes

import numpy as np
import pytest

from numfast_b200 import _lib
from oracle import nf_oracle as O

pytestmark = pytest.mark.gpu


def vp(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.fixture(scope="module")
def lib(cuda):
    return _lib.load()


def test_group_sum_count(lib):
    rs = np.random.default_rng(1)
    n, g = 100_000, 777
    k = rs.integers(0, g, n).astype(np.int32)
    v = rs.standard_normal(n)
    sums = np.zeros(g)
    counts = np.zeros(g, dtype=np.int64)
    assert lib.nf_group_sum_count(vp(k), vp(v), n, vp(sums), vp(counts), g) == 0
    np.testing.assert_allclose(sums, np.bincount(k, weights=v, minlength=g), rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(counts, np.bincount(k, minlength=g))
    k[5] = g
    assert lib.nf_group_sum_count(vp(k), vp(v), n, vp(sums), vp(counts), g) == _lib.ERR_RANGE


def test_multi_sum_count(lib):
    rs = np.random.default_rng(2)
    n, g, nc = 50_000, 100, 3
    k = rs.integers(0, g, n).astype(np.int32)
    v = rs.standard_normal(nc * n)
    sums = np.zeros(nc * g)
    counts = np.zeros(g, dtype=np.int64)
    assert lib.nf_group_multi_sum_count(vp(k), vp(v), n, nc, vp(sums), vp(counts), g) == 0
    for c in range(nc):
        np.testing.assert_allclose(sums[c * g:(c + 1) * g], np.bincount(k, weights=v[c * n:(c + 1) * n], minlength=g),
                                   rtol=1e-12, atol=1e-12)


def test_variant_i32_overflow_rule(lib):
    g = 2
    k = np.array([0, 0, 0, 1], dtype=np.int32)
    sums = np.zeros(g, dtype=np.int32)
    counts = np.zeros(g, dtype=np.int64)
    ok = np.array([5, -3, 7, 2 ** 31 - 1], dtype=np.int32)
    assert lib.nf_group_variant_i32(vp(k), vp(ok), 4, 0, vp(sums), vp(counts), g) == 0
    assert sums.tolist() == [9, 2 ** 31 - 1] and counts.tolist() == [3, 1]
    # a running sum leaves int32 even though the final sum fits -> -4 (row-order rule)
    prefix = np.array([2 ** 31 - 1, 1, -1, 0], dtype=np.int32)
    assert lib.nf_group_variant_i32(vp(k), vp(prefix), 4, 0, vp(sums), vp(counts), g) == _lib.ERR_OVERFLOW
    # large magnitudes that never overflow in row order -> ok
    safe = np.array([2 ** 31 - 1, -(2 ** 31 - 1), 2 ** 31 - 1, 0], dtype=np.int32)
    assert lib.nf_group_variant_i32(vp(k), vp(safe), 4, 0, vp(sums), vp(counts), g) == 0
    assert lib.nf_group_variant_i32(vp(k), vp(ok), 4, 1, vp(sums), vp(counts), g) == _lib.ERR_MALFORMED
    unsorted = np.array([1, 0, 0, 1], dtype=np.int32)
    assert lib.nf_group_variant_i32(vp(unsorted), vp(ok), 4, 2, vp(sums), vp(counts), g) == _lib.ERR_UNSORTED


def test_variant_i64_and_f64(lib):
    rs = np.random.default_rng(4)
    n, g = 20_000, 50
    k = np.sort(rs.integers(0, g, n)).astype(np.int32)
    t = rs.integers(-2 ** 40, 2 ** 40, n).astype(np.int64)
    sums = np.zeros(g, dtype=np.int64)
    counts = np.zeros(g, dtype=np.int64)
    for variant in (0, 1, 2):
        assert lib.nf_group_variant_i64(vp(k), vp(t), n, variant, vp(sums), vp(counts), g) == 0
        ref = np.zeros(g, dtype=np.int64)
        np.add.at(ref, k, t)
        np.testing.assert_array_equal(sums, ref)
    assert lib.nf_group_variant_i64(vp(k), vp(t), n, 7, vp(sums), vp(counts), g) == _lib.ERR_MALFORMED
    big = np.array([2 ** 62, 2 ** 62], dtype=np.int64)
    kk = np.array([0, 0], dtype=np.int32)
    assert lib.nf_group_variant_i64(vp(kk), vp(big), 2, 0, vp(sums), vp(counts), 1) == _lib.ERR_OVERFLOW
    f = rs.standard_normal(n)
    fs = np.zeros(g)
    assert lib.nf_group_variant_f64(vp(k), vp(f), n, 2, vp(fs), vp(counts), g) == 0
    np.testing.assert_allclose(fs, np.bincount(k, weights=f, minlength=g), rtol=1e-12, atol=1e-12)


def test_mixed_count_owner(lib):
    rs = np.random.default_rng(5)
    n, g = 30_000, 300
    k = rs.integers(0, g, n).astype(np.int32)
    a = rs.integers(-100, 100, n).astype(np.int32)
    b = rs.integers(-100, 100, n).astype(np.int32)
    c = rs.standard_normal(n)
    iv = np.concatenate([a, b])
    i32s = np.zeros(2 * g, dtype=np.int32)
    f64s = np.zeros(g)
    assert lib.nf_group_mixed_sum_only(vp(k), vp(iv), vp(c), n, 2, 1, vp(i32s), vp(f64s), g) == 0
    np.testing.assert_array_equal(i32s[:g], np.bincount(k, weights=a, minlength=g).astype(np.int64))
    counts = np.zeros(g, dtype=np.int64)
    assert lib.nf_group_count_only(vp(k), n, vp(counts), g) == 0
    np.testing.assert_array_equal(counts, np.bincount(k, minlength=g))
    s1 = np.full(g, 99, dtype=np.int32)
    s2 = np.full(g, 99, dtype=np.int32)
    s3 = np.full(g, 99.0)
    cn = np.full(g, 99, dtype=np.int64)
    assert lib.nf_group_owner_2i32_1f64(vp(k), vp(a), vp(b), vp(c), n, 100, 200, vp(s1), vp(s2), vp(s3), vp(cn),
                                        g) == 0
    np.testing.assert_array_equal(s1[100:200], np.bincount(k, weights=a, minlength=g)[100:200].astype(np.int64))
    assert (s1[:100] == 99).all() and (cn[200:] == 99).all()
    np.testing.assert_array_equal(cn[100:200], np.bincount(k, minlength=g)[100:200])


def test_sorted_run_and_carry(lib):
    k = np.array([1, 1, 3, 3, 3, 8], dtype=np.int32)
    v = np.array([1, 2, 3, 4, 5, 6], dtype=np.int64)
    uk = np.zeros(6, dtype=np.int64)
    s = np.zeros(6, dtype=np.int64)
    c = np.zeros(6, dtype=np.int64)
    assert lib.nf_sorted_run_i64(vp(k), vp(v), 6, vp(uk), vp(s), vp(c)) == 3
    assert uk[:3].tolist() == [1, 3, 8] and s[:3].tolist() == [3, 12, 6] and c[:3].tolist() == [2, 3, 1]
    k2 = k[::-1].copy()
    assert lib.nf_sorted_run_i64(vp(k2), vp(v), 6, vp(uk), vp(s), vp(c)) == -1
    cm = np.array([0, 2, 0, 5, 1], dtype=np.int64)
    sm = np.array([0.0, 1.5, 0.0, -2.0, 7.0])
    uk2 = np.zeros(5, dtype=np.int64)
    c2 = np.zeros(5, dtype=np.int64)
    s2 = np.zeros(5)
    assert lib.nf_carry_build_f64(vp(cm), vp(sm), 5, vp(uk2), vp(c2), vp(s2)) == 3
    assert uk2[:3].tolist() == [1, 3, 4] and c2[:3].tolist() == [2, 5, 1] and s2[:3].tolist() == [1.5, -2.0, 7.0]


@pytest.mark.parametrize("desc", [0, 1])
def test_sort_perm_and_unique(lib, golden, desc):
    k = golden["sort_in_k"]
    n = k.size
    perm = np.zeros(n, dtype=np.int32)
    t0 = np.zeros(n, dtype=np.uint32)
    assert lib.nf_sort_perm_i32(vp(k), n, desc, vp(perm), vp(t0), vp(t0), vp(perm)) == 0
    np.testing.assert_array_equal(perm, golden["sort_i32_" + ("desc" if desc else "asc")])
    k64 = golden["sort_in_i64"]
    perm = np.zeros(k64.size, dtype=np.int32)
    t1 = np.zeros(k64.size, dtype=np.uint64)
    assert lib.nf_sort_perm_i64(vp(k64), k64.size, desc, vp(perm), vp(t1), vp(t1), vp(perm)) == 0
    np.testing.assert_array_equal(perm, golden["sort_i64_" + ("desc" if desc else "asc")])
    u = golden["uniq_in"]
    uq = np.zeros(u.size, dtype=np.int32)
    inv = np.zeros(u.size, dtype=np.int32)
    scratch = np.zeros(u.size, dtype=np.int32)
    ng = lib.nf_unique_inverse_i32(vp(u), u.size, vp(uq), vp(inv), vp(scratch), vp(scratch), vp(scratch), vp(scratch))
    assert ng == golden["uniq_u"].size
    np.testing.assert_array_equal(uq[:ng], golden["uniq_u"])
    np.testing.assert_array_equal(inv, golden["uniq_inv"])


def test_sorted_run_f64_carry_i64_unique_i64(lib):
    """The remaining drop-in variants: float64 sorted runs, int64 carry build and
    int64 unique + inverse (np.unique labelling) against the oracle."""
    rs = np.random.default_rng(31)
    k = np.sort(rs.integers(-50, 50, 5000)).astype(np.int32)
    v = rs.normal(0.0, 10.0, k.size)
    uk = np.zeros(k.size, dtype=np.int64)
    s = np.zeros(k.size)
    c = np.zeros(k.size, dtype=np.int64)
    ng = lib.nf_sorted_run_f64(vp(k), vp(v), k.size, vp(uk), vp(s), vp(c))
    ref = O.groupby_multi(k, {"v": v}, {"v": ("sum", "count")})
    assert ng == ref["ukeys"].size
    np.testing.assert_array_equal(uk[:ng], ref["ukeys"])
    np.testing.assert_array_equal(c[:ng], ref["counts"])
    np.testing.assert_allclose(s[:ng], ref["sums"]["v"], rtol=1e-12, atol=1e-12)
    k2 = k[::-1].copy()
    assert lib.nf_sorted_run_f64(vp(k2), vp(v), k.size, vp(uk), vp(s), vp(c)) == -1

    cm = np.array([3, 0, 0, 1, 0, 2], dtype=np.int64)
    sm = np.array([-7, 0, 0, 2 ** 40, 0, 5], dtype=np.int64)
    uk2 = np.zeros(6, dtype=np.int64)
    c2 = np.zeros(6, dtype=np.int64)
    s2 = np.zeros(6, dtype=np.int64)
    assert lib.nf_carry_build_i64(vp(cm), vp(sm), 6, vp(uk2), vp(c2), vp(s2)) == 3
    assert uk2[:3].tolist() == [0, 3, 5] and c2[:3].tolist() == [3, 1, 2] and s2[:3].tolist() == [-7, 2 ** 40, 5]

    u = rs.integers(-2 ** 63, 2 ** 63 - 1, 20_000, dtype=np.int64)
    u[:500] = u[500:1000]
    u[1000] = -2 ** 63
    u[1001] = 2 ** 63 - 1
    uq = np.zeros(u.size, dtype=np.int64)
    inv = np.zeros(u.size, dtype=np.int32)
    perm = np.zeros(u.size, dtype=np.int32)
    t = np.zeros(u.size, dtype=np.uint64)
    ng = lib.nf_unique_inverse_i64(vp(u), u.size, vp(uq), vp(inv), vp(perm), vp(t), vp(t), vp(perm))
    want_u, want_inv = np.unique(u, return_inverse=True)
    assert ng == want_u.size
    np.testing.assert_array_equal(uq[:ng], want_u)
    np.testing.assert_array_equal(inv, want_inv)


def test_pack_sum_count(lib):
    """Fused pack + aggregate (pack_fused.rs:26-90): codes k1*m2 + k2, sums and counts."""
    rs = np.random.default_rng(9)
    n, m2 = 200_000, 37
    k1 = rs.integers(0, 50, n).astype(np.int32)
    k2 = rs.integers(0, m2, n).astype(np.int32)
    g = 50 * m2
    code = k1.astype(np.int64) * m2 + k2
    vi = rs.integers(-1000, 1001, n).astype(np.int32)
    vf = rs.standard_normal(n)
    si = np.full(g, 7, dtype=np.int32)
    sf = np.full(g, 7.0)
    c = np.full(g, 7, dtype=np.int64)
    assert lib.nf_pack_sum_count_i32(vp(k1), vp(k2), m2, vp(vi), n, vp(si), vp(c), g) == 0
    np.testing.assert_array_equal(si, np.bincount(code, weights=vi, minlength=g).astype(np.int32))
    np.testing.assert_array_equal(c, np.bincount(code, minlength=g))
    assert lib.nf_pack_sum_count_f64(vp(k1), vp(k2), m2, vp(vf), n, vp(sf), vp(c), g) == 0
    np.testing.assert_allclose(sf, np.bincount(code, weights=vf, minlength=g), rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(c, np.bincount(code, minlength=g))
    # a negative component, a code past INT32_MAX, a code outside [0, g) -> -2
    bad = k1.copy()
    bad[17] = -1
    assert lib.nf_pack_sum_count_i32(vp(bad), vp(k2), m2, vp(vi), n, vp(si), vp(c), g) == _lib.ERR_RANGE
    big = k1.copy()
    big[3] = 2 ** 31 // m2 + 1
    assert lib.nf_pack_sum_count_f64(vp(big), vp(k2), m2, vp(vf), n, vp(sf), vp(c), g) == _lib.ERR_RANGE
    assert lib.nf_pack_sum_count_i32(vp(k1), vp(k2), m2, vp(vi), n, vp(si), vp(c), g - 1) == _lib.ERR_RANGE
    # a running int32 sum that leaves int32 in row order -> -4
    z = np.zeros(4, dtype=np.int32)
    ov = np.array([2 ** 31 - 1, 1, -5, 0], dtype=np.int32)
    s4 = np.zeros(1, dtype=np.int32)
    c4 = np.zeros(1, dtype=np.int64)
    assert lib.nf_pack_sum_count_i32(vp(z), vp(z), 3, vp(ov), 4, vp(s4), vp(c4), 1) == _lib.ERR_OVERFLOW
