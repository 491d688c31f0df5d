"""Failure handling without a GPU fault.  Bounded waits: a decoupled look-back
whose predecessor never publishes and an mbarrier phase that never completes
both give up after their poll limit and report NFC_ERR_TIMEOUT instead of
hanging the GPU.  Allocation failure: an injected out-of-memory on a scratch
allocation is reported as NFC_ERR_NOMEM.  The context stays usable after
either."""

import ctypes
import time

import numpy as np
import pytest

from numfast_b200 import _lib
from oracle import nf_oracle as O
from tests.gpu_util import OPS, assert_carry_equal, cfg2_inputs, device_groupby

pytestmark = pytest.mark.gpu

NFC_ERR_TIMEOUT = -7


def test_waits_give_up_and_report(cuda):
    lib = _lib.load()
    st = (ctypes.c_int32 * 2)()
    t0 = time.perf_counter()
    rc = lib.nfc_selftest_bounded_waits(1 << 14, st, None)
    dt = time.perf_counter() - t0
    assert rc == 0, _lib.last_error()
    assert list(st) == [NFC_ERR_TIMEOUT, NFC_ERR_TIMEOUT]
    assert dt < 10.0
    # The same context runs a normal group-by right after.
    k, cols, val = cfg2_inputs(50_000, 3_000, seed=9)
    assert_carry_equal(device_groupby(k, cols, val, "partition"), O.groupby_multi(k, cols, OPS, val))


@pytest.mark.parametrize("after", [0, 1, 2, 3, 4, 5, 6])
def test_scratch_allocation_failure_is_reported(cuda, after):
    """Host-side fault injection: the n-th scratch allocation of a partition
    group-by fails as if the device were out of memory.  The call returns
    NFC_ERR_NOMEM (kernels already queued finish on their own scratch, which
    is released in stream order) and the next call is correct."""
    lib = _lib.load()
    k, cols, val = cfg2_inputs(300_000, 2_000_000, seed=4)
    lib.nfc_debug_fail_alloc(after)
    try:
        with pytest.raises(_lib.NativeError) as ei:
            device_groupby(k, cols, val, "partition")
        assert ei.value.code == _lib.ERR_NOMEM
    finally:
        lib.nfc_debug_fail_alloc(-1)
    assert_carry_equal(device_groupby(k, cols, val, "partition"), O.groupby_multi(k, cols, OPS, val))
