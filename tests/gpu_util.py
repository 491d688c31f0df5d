"""Shared helpers for the GPU parity tests."""

import numpy as np
import torch

from numfast_b200 import device as dev
from oracle import nf_oracle as O

F64_RTOL = 1e-12
OPS = {"v": ("sum", "count", "min", "max"), "f": ("sum", "min", "max")}


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def bitmap(mask):
    return None if mask is None else to_dev(dev.pack_validity(mask))


def device_groupby(k, cols, validity, strategy="auto", ops=OPS):
    """cols: {name: np array}; validity: {name or '__key__': bool mask}."""
    dcols = [dev.DeviceColumn(c, to_dev(v), tuple(o for o in ops[c] if o != "count"), bitmap(validity.get(c)))
             for c, v in cols.items()]
    r = dev.groupby(to_dev(k), dcols, bitmap(validity.get("__key__")), strategy=strategy)
    torch.cuda.synchronize()
    out = {"ukeys": r.ukeys.cpu().numpy(), "counts": r.counts.cpu().numpy(),
           "sums": {c: t.cpu().numpy() for c, t in r.sums.items()},
           "mins": {c: t.cpu().numpy() for c, t in r.mins.items()},
           "maxs": {c: t.cpu().numpy() for c, t in r.maxs.items()},
           "strategy": r.strategy}
    return out


def assert_carry_equal(got, ref, float_cols=("f",)):
    np.testing.assert_array_equal(got["ukeys"], ref["ukeys"])
    np.testing.assert_array_equal(got["counts"], ref["counts"])
    for c, s in ref["sums"].items():
        if c in float_cols:
            np.testing.assert_allclose(got["sums"][c], s, rtol=F64_RTOL, atol=1e-12, equal_nan=True)
        else:
            assert got["sums"][c].dtype == np.int64
            np.testing.assert_array_equal(got["sums"][c], s)
    for kind in ("mins", "maxs"):
        for c, s in ref[kind].items():
            assert got[kind][c].dtype == s.dtype, (kind, c, got[kind][c].dtype, s.dtype)
            np.testing.assert_array_equal(got[kind][c], s)


def cfg2_inputs(n, span, seed=42, null_p=0.05, kmin=0):
    k = (O.fill_i32(n, seed, 0, 0, 0, span) + kmin).astype(np.int32)
    v = O.fill_i32(n, seed, 1, 0, -1000, 1001)
    f = np.exp(3.0 + O.fill_f64(n, seed, 2, 0, -2.0, 2.0))
    val = {"__key__": O.fill_f64(n, seed, 4) >= null_p, "v": O.fill_f64(n, seed, 5) >= null_p,
           "f": O.fill_f64(n, seed, 6) >= null_p}
    return k, {"v": v, "f": f}, val
