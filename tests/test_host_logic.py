"""Host-side logic that needs no GPU: IR constructors, ColumnCarry shapes, chain
validation, validity packing, and the loud failure without a device."""

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
