"""nfc_groupby_dense_noalloc: the group-by entry point that allocates nothing.

It serves callers that cannot call cudaMalloc (plugins inside a host process that
owns all device memory and forbids foreign allocations, real-time loops that must
not touch the allocator).  Its scratch is one static device array.  This file is collected
last on purpose, and it must pass alone in a fresh process as well as after the
other tests: the static scratch keeps the previous call's contents, so each call
must clear what it relies on.
"""

import ctypes

import numpy as np
import pytest
import torch

from numfast_b200 import _lib
from numfast_b200 import device as dev

pytestmark = pytest.mark.gpu

F64_RTOL = 1e-12


def _inputs(n, span, seed):
    k = dev.rng_fill_i32(n, seed, 0, -7, span - 7)
    v = dev.rng_fill_i32(n, seed, 1, -1000, 1001)
    f = dev.gen_lognormal(n, seed, 2, 3, 3.0, 1.0)
    kv = dev.gen_validity(n, seed, 4, 0.05)
    fv = dev.gen_validity(n, seed, 6, 0.05)
    return k, [dev.DeviceColumn("v", v, ("sum", "min", "max")), dev.DeviceColumn("f", f, ("sum", "min", "max"), fv)], kv


def _noalloc(keys, cols, key_validity, cap):
    """Call the entry point through the C ABI with freshly allocated outputs."""
    lib = _lib.load()
    n = int(keys.numel())
    out = {"ukeys": torch.full((cap,), -1, dtype=torch.int64, device=keys.device),
           "counts": torch.full((cap,), -1, dtype=torch.int64, device=keys.device)}
    vc = (_lib.ValueCol * len(cols))()
    for i, c in enumerate(cols):
        sdt = torch.float64 if c.values.dtype == torch.float64 else torch.int64
        out["sum_" + c.name] = torch.full((cap,), 7, dtype=sdt, device=keys.device)
        out["min_" + c.name] = torch.full((cap,), 7, dtype=c.values.dtype, device=keys.device)
        out["max_" + c.name] = torch.full((cap,), 7, dtype=c.values.dtype, device=keys.device)
        vc[i].dtype = {torch.int32: _lib.I32, torch.int64: _lib.I64, torch.float64: _lib.F64}[c.values.dtype]
        vc[i].aggs = _lib.AGG_SUM | _lib.AGG_MIN | _lib.AGG_MAX
        vc[i].data = c.values.data_ptr()
        vc[i].validity = c.validity.data_ptr() if c.validity is not None else None
        vc[i].sum_out = out["sum_" + c.name].data_ptr()
        vc[i].min_out = out["min_" + c.name].data_ptr()
        vc[i].max_out = out["max_" + c.name].data_ptr()
    args = _lib.GroupbyArgs()
    args.n = n
    args.keys = keys.data_ptr()
    args.key_validity = key_validity.data_ptr() if key_validity is not None else None
    args.ncols = len(cols)
    args.cols = vc
    args.out_cap = cap
    args.ukeys_out = out["ukeys"].data_ptr()
    args.counts_out = out["counts"].data_ptr()
    ng = lib.nfc_groupby_dense_noalloc(ctypes.byref(args),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return ng, out


def _compare(ng, out, ref):
    assert ng == ref.ngroups
    np.testing.assert_array_equal(out["ukeys"][:ng].cpu().numpy(), ref.ukeys.cpu().numpy())
    np.testing.assert_array_equal(out["counts"][:ng].cpu().numpy(), ref.counts.cpu().numpy())
    for name in ("v", "f"):
        for kind, src in (("min", ref.mins), ("max", ref.maxs)):
            np.testing.assert_array_equal(out[kind + "_" + name][:ng].cpu().numpy(), src[name].cpu().numpy())
    np.testing.assert_array_equal(out["sum_v"][:ng].cpu().numpy(), ref.sums["v"].cpu().numpy())
    np.testing.assert_allclose(out["sum_f"][:ng].cpu().numpy(), ref.sums["f"].cpu().numpy(), rtol=F64_RTOL,
                               atol=1e-12)


def test_noalloc_matches_groupby_twice(cuda):
    keys, cols, kv = _inputs(1_000_003, 60_000, 42)
    ref = dev.groupby(keys, cols, kv)
    torch.cuda.synchronize()
    for _ in range(2):  # the second call must not see the first call's scratch
        ng, out = _noalloc(keys, cols, kv, 100_000)
        _compare(ng, out, ref)


def test_noalloc_second_input_after_first(cuda):
    k1, c1, v1 = _inputs(300_000, 5_000, 7)
    k2, c2, v2 = _inputs(200_000, 90_000, 8)
    ng1, out1 = _noalloc(k1, c1, v1, 10_000)
    ng2, out2 = _noalloc(k2, c2, v2, 100_000)
    _compare(ng2, out2, dev.groupby(k2, c2, v2))
    _compare(ng1, out1, dev.groupby(k1, c1, v1))


def test_noalloc_rejects_sizes_beyond_the_limit(cuda):
    lib = _lib.load()
    # Key span beyond the state budget: two keys far apart.
    keys = torch.tensor([0, 10_000_000], dtype=torch.int32, device="cuda")
    v = torch.tensor([1, 2], dtype=torch.int32, device="cuda")
    ng, _ = _noalloc(keys, [dev.DeviceColumn("v", v, ("sum",)), dev.DeviceColumn("f", v.double(), ("sum",))],
                     None, 16)
    assert ng == _lib.ERR_RANGE
    assert "NFC_NOALLOC_STATE_BYTES" in _lib.last_error()
    # More rows than NFC_NOALLOC_MAX_ROWS (rejected on the host, before any launch).
    big = torch.zeros(_lib.NOALLOC_MAX_ROWS + 1, dtype=torch.int32, device="cuda")
    bigf = torch.zeros(_lib.NOALLOC_MAX_ROWS + 1, dtype=torch.float64, device="cuda")
    ng, _ = _noalloc(big, [dev.DeviceColumn("v", big, ("sum",)), dev.DeviceColumn("f", bigf, ("sum",))], None, 16)
    assert ng == _lib.ERR_RANGE
    assert "NFC_NOALLOC_MAX_ROWS" in _lib.last_error()
