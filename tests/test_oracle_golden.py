"""The oracle (oracle/nf_oracle.py) against golden vectors produced by the reference."""

import numpy as np
import pytest

from oracle import nf_oracle as O

F64_TOL = dict(rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("i", range(4))
def test_rng_i32(golden, i):
    n, seed, stream, off, lo, hi = (int(x) for x in golden["rng_i32_%d_args" % i])
    got = O.fill_i32(n, seed, stream, off, lo, hi)
    np.testing.assert_array_equal(got, golden["rng_i32_%d" % i])


@pytest.mark.parametrize("i", range(2))
def test_rng_f64(golden, i):
    n, seed, stream, off, lo, hi = golden["rng_f64_%d_args" % i]
    got = O.fill_f64(int(n), int(seed), int(stream), int(off), lo, hi)
    np.testing.assert_array_equal(got, golden["rng_f64_%d" % i])


def test_rng_chunkable():
    full = O.fill_i32(100, 42, 3, 0, -7, 9)
    np.testing.assert_array_equal(full[40:], O.fill_i32(60, 42, 3, 40, -7, 9))


def _gb(golden, tag):
    k, v, f = golden[tag + "_in_k"], golden[tag + "_in_v"], golden[tag + "_in_f"]
    val = {"__key__": golden[tag + "_in_kval"], "v": golden[tag + "_in_vval"], "f": golden[tag + "_in_fval"]}
    return O.groupby_multi(k, {"v": v, "f": f},
                           {"v": ("sum", "count", "min", "max"), "f": ("sum", "min", "max")}, val)


def assert_gb_equal(got, golden, tag):
    np.testing.assert_array_equal(got["ukeys"], golden[tag + "_ukeys"])
    np.testing.assert_array_equal(got["counts"], golden[tag + "_counts"])
    np.testing.assert_array_equal(got["sums"]["v"], golden[tag + "_v_sum"])
    assert got["sums"]["v"].dtype == np.int64
    np.testing.assert_array_equal(got["mins"]["v"], golden[tag + "_v_min"])
    np.testing.assert_array_equal(got["maxs"]["v"], golden[tag + "_v_max"])
    assert got["mins"]["v"].dtype == np.int32
    np.testing.assert_allclose(got["sums"]["f"], golden[tag + "_f_sum"], equal_nan=True, **F64_TOL)
    np.testing.assert_array_equal(got["mins"]["f"], golden[tag + "_f_min"])
    np.testing.assert_array_equal(got["maxs"]["f"], golden[tag + "_f_max"])


@pytest.mark.parametrize("tag", ["gb_dense", "gb_sparse", "gb_bound", "gb_sorted", "gb_nan"])
def test_groupby(golden, tag):
    assert_gb_equal(_gb(golden, tag), golden, tag)


def test_groupby_null_semantics(golden):
    g = _gb(golden, "gb_sorted")
    assert 13 not in set(g["ukeys"].tolist())  # every row of key 13 is NULL -> absent
    g = _gb(golden, "gb_dense")
    m = golden["gb_dense_in_kval"] & golden["gb_dense_in_vval"] & golden["gb_dense_in_fval"]
    assert int(g["counts"].sum()) == int(m.sum())


@pytest.mark.parametrize("desc", [False, True])
def test_sort_i32(golden, desc):
    d = "desc" if desc else "asc"
    np.testing.assert_array_equal(O.sort_perm([golden["sort_in_k"]], [desc]), golden["sort_i32_" + d])
    np.testing.assert_array_equal(O.sort_perm([golden["sort_in_k"]], [desc], golden["sort_in_val"]),
                                  golden["sort_i32_null_" + d])


@pytest.mark.parametrize("desc", [False, True])
def test_sort_f64_i64(golden, desc):
    d = "desc" if desc else "asc"
    np.testing.assert_array_equal(O.sort_perm([golden["sort_in_f"]], [desc]), golden["sort_f64_" + d])
    np.testing.assert_array_equal(O.sort_perm([golden["sort_in_i64"]], [desc]), golden["sort_i64_" + d])


def test_sort_lex(golden):
    np.testing.assert_array_equal(O.sort_perm([golden["sort_lex_a"], golden["sort_lex_b"]], [True, False]),
                                  golden["sort_lex"])


def test_unique(golden):
    u, inv = O.unique_inverse(golden["uniq_in"])
    np.testing.assert_array_equal(u, golden["uniq_u"])
    np.testing.assert_array_equal(inv, golden["uniq_inv"])
    u, inv = O.unique_inverse(golden["uniq_in"], golden["uniq_val"])
    np.testing.assert_array_equal(u, golden["uniq_null_u"])
    np.testing.assert_array_equal(inv, golden["uniq_null_inv"])


def test_config1_chain(golden):
    n = 1_000_000
    key = O.fill_i32(n, 42, 0, 0, 0, 1000)
    v = O.fill_i32(n, 42, 1, 0, -100, 101)
    np.testing.assert_array_equal(key[:4096], golden["cfg1_key_head"])
    np.testing.assert_array_equal(v[:4096], golden["cfg1_v_head"])
    out = O.chain_group_sort(key, v, ("sum", "count"), "sum", True)
    np.testing.assert_array_equal(out["key"], golden["cfg1_key"])
    np.testing.assert_array_equal(out["v.sum"], golden["cfg1_v_sum"])
    np.testing.assert_array_equal(out["v.count"], golden["cfg1_v_count"])
