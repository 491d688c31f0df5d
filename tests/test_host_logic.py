"""Host-side logic that needs no GPU: IR constructors, ColumnCarry shapes, chain
validation, validity packing, and the loud failure without a device."""

import ctypes

import numpy as np
import pytest

from numfast_b200 import carry, chain, ir
from numfast_b200 import device as dev


def test_ir_groupby_multi_shapes():
    j = ir.ir_groupby_multi("g", ["a", "b"], "k", {"a": ("sum",), "b": ("min", "max")}, result="carry")
    assert j["inputs"] == ["a", "b", "k"] and j["params"]["cols"] == ["a", "b"]
    assert j["params"]["result"] == "carry"
    j = ir.ir_groupby_multi("g", "v", "k", ("sum", "count"))
    assert j["inputs"] == ["v", "k"] and j["params"] == {"ops": ["sum", "count"]}
    with pytest.raises(ValueError):
        ir.ir_groupby_multi("g", ["a"], "k", {"b": ("sum",)})
    with pytest.raises(ValueError):
        ir.ir_groupby_multi("g", "v", "k", ("median",))
    with pytest.raises(ValueError):
        ir.ir_sort("p")
    assert ir.ir_sort("p", "a", "b", descending=True)["params"]["descending"] == [True, True]


def test_column_carry_dicts():
    c = carry.ColumnCarry(np.array([1, 5]), np.array([2, 1]), {"v": np.array([10, 3])},
                          {"v": np.array([4, 3], dtype=np.int32)}, {"v": np.array([6, 3], dtype=np.int32)})
    assert c.to_dict_single("v", ("sum", "count", "mean")) == {1: {"sum": 10, "count": 2, "mean": 5.0},
                                                               5: {"sum": 3, "count": 1, "mean": 3.0}}
    assert c.to_dict_multi(["v"], {"v": ("min", "max")}) == {1: {"v": {"min": 4, "max": 6}},
                                                             5: {"v": {"min": 3, "max": 3}}}
    assert c.to_dict_flat("count") == {1: 2, 5: 1}
    assert c.ngroups == 2


def test_pack_validity_lsb_first():
    m = np.array([1, 0, 0, 0, 0, 0, 0, 0, 1, 1], dtype=bool)
    b = dev.pack_validity(m)
    assert b.tolist() == [1, 3]


def test_chain_refuses_null_keys_before_running():
    t = chain.from_numpy({"k": np.array([1, 2, 3], dtype=np.int32), "v": np.array([1, 2, 3], dtype=np.int32)},
                         validity={"k": np.array([1, 0, 1], dtype=bool)})
    with pytest.raises(chain.ChainError, match="NULL"):
        t.query().group("k", {"v": ("sum",)})
    with pytest.raises(chain.ChainError):
        t.query().group("k", {"v": ("median",)})
    with pytest.raises(chain.ChainError):
        t.query().sort("zz")


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from numfast_b200 import NativeUnavailable, executor
    jobs = [ir.ir_series("k", [1, 2], "int32"), ir.ir_series("v", [1, 2], "int32"),
            ir.ir_groupby_multi("g", "v", "k", ("sum",))]
    with pytest.raises(NativeUnavailable):
        executor.execute(jobs)


# ---------------------------------------------------------------- batched group-by host side

def test_batch_layout_distribution():
    from numfast_b200 import batch as B
    lay = B.config4_layout()
    rows, card = lay["rows"], lay["card"]
    assert rows.size == 4096
    assert rows.min() >= 1000 and rows.max() <= 4_000_000
    assert (card >= 1).all() and (card <= rows).all()
    assert 1.5e9 < lay["row_offsets"][-1] < 2.5e9
    assert 0.4 < lay["zipf"].mean() < 0.6
    assert (lay["s"] >= 0.5).all() and (lay["s"] <= 2.0).all() and (np.abs(lay["s"] - 1) >= 1e-3).all()
    again = B.config4_layout()
    assert np.array_equal(again["row_offsets"], lay["row_offsets"])
    sig = B.layout_signature(lay["row_offsets"])
    assert sig.startswith("nq4096-rows%d-" % lay["row_offsets"][-1])


def test_batch_create_rejects_bad_arguments():
    """Tuning and layout checks run on the host before any CUDA call."""
    from numfast_b200 import _lib
    from numfast_b200 import batch as B
    lib = _lib.load()
    ro = np.array([0, 10, 20], dtype=np.int64)
    t = B.default_tuning()
    t.chunk_rows = 1000  # not a multiple of 8192
    assert not lib.nfc_batch_create(2, ro.ctypes.data, ctypes.byref(t))
    assert "invalid tuning" in _lib.last_error()
    t = B.default_tuning()
    t.ctas_per_sm = 2
    t.smem_slots = 24576  # two CTAs cannot hold 2 x 192 KiB
    assert not lib.nfc_batch_create(2, ro.ctypes.data, ctypes.byref(t))
    bad = np.array([0, 10, 5], dtype=np.int64)
    assert not lib.nfc_batch_create(2, bad.ctypes.data, None)
    assert "rows" in _lib.last_error()
    assert not lib.nfc_batch_create(0, ro.ctypes.data, None)
    d = B.default_tuning().as_dict()
    assert d["chunk_rows"] % 8192 == 0 and d["smem_slots"] % 1024 == 0
    for _, options in B.SEARCH_SPACE:
        for opt in options:
            for k in opt:
                assert k in d
