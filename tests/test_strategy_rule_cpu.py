"""The library's own strategy rule (nfc_plan_strategy: host code, no GPU work) on the
headline's column set, including the DENSE_GLOBAL / PARTITION boundary by valid rows."""

import ctypes

import pytest

from numfast_b200 import _lib

DENSE_SMEM, DENSE_GLOBAL, PARTITION, HASH = 2, 3, 4, 5
I32, F64 = 0, 2
SUM_MIN_MAX = 1 | 2 | 4


@pytest.fixture(scope="module")
def lib():
    return _lib.load()


def pick(lib, n_valid, kmin, kmax, n=None):
    dummy = ctypes.c_void_p(0x1000)  # never dereferenced: the rule reads only dtypes and aggregates
    cols = (_lib.ValueCol * 2)()
    for c, dt in enumerate((I32, F64)):
        cols[c].dtype, cols[c].aggs = dt, SUM_MIN_MAX
        cols[c].data = cols[c].sum_out = cols[c].min_out = cols[c].max_out = dummy
    a = _lib.GroupbyArgs()
    a.n = n if n is not None else max(n_valid, 1)
    a.keys = dummy
    a.ncols = 2
    a.cols = cols
    a.ukeys_out = a.counts_out = dummy
    p = _lib.Probe(n_valid, kmin, kmax, 0, 0)
    return lib.nfc_plan_strategy(ctypes.byref(a), ctypes.byref(p))


def test_strategy_rule(lib):
    assert pick(lib, 0, 0, 0, n=10) == DENSE_GLOBAL               # nothing to group
    assert pick(lib, 100_000_000, 0, 1_999) == DENSE_SMEM         # 2,000 keys: state fits one CTA
    assert pick(lib, 1_000_000, 0, 199_999) == DENSE_GLOBAL       # L2-resident span, few rows
    assert pick(lib, 100_000_000, 0, 199_999) == PARTITION        # same span, many rows
    assert pick(lib, 100_000_000, 0, 9_999_999) == PARTITION      # the headline
    assert pick(lib, 1_000_000, -2 ** 31, 2 ** 31 - 1) == HASH    # sparse over the full range


def test_sorted_keys_take_the_run_pass(lib):
    """Nondecreasing valid keys (the probe's sortedness flag) take SORTED whatever the
    span, like the reference's planner (planner.py:226)."""
    SORTED = 1
    dummy = ctypes.c_void_p(0x1000)
    cols = (_lib.ValueCol * 1)()
    cols[0].dtype, cols[0].aggs = I32, SUM_MIN_MAX
    cols[0].data = cols[0].sum_out = cols[0].min_out = cols[0].max_out = dummy
    a = _lib.GroupbyArgs()
    a.n = 1000
    a.keys = dummy
    a.ncols = 1
    a.cols = cols
    a.ukeys_out = a.counts_out = dummy
    for kmin, kmax in ((0, 5), (0, 9_999_999), (-2 ** 31, 2 ** 31 - 1)):
        p = _lib.Probe(1000, kmin, kmax, 1, 0)
        assert lib.nfc_plan_strategy(ctypes.byref(a), ctypes.byref(p)) == SORTED
    p = _lib.Probe(0, 0, 0, 1, 0)
    assert lib.nfc_plan_strategy(ctypes.byref(a), ctypes.byref(p)) == DENSE_GLOBAL
