"""Bounded waits: a decoupled look-back whose predecessor never publishes and an
mbarrier phase that never completes both give up after their poll limit and
report NFC_ERR_TIMEOUT instead of hanging the GPU; the context stays usable."""

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
