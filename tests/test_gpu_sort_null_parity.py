"""Sort with NULL keys against pandas, the way the reference pins its own sort
(tests/fast/test_consumer_sort_null_parity.py): the permutation equals pandas'
`sort_values(kind="stable", na_position="last")` index order, in both
directions, on its numeric fixtures (text columns are off this path)."""

import numpy as np
import pandas as pd
import pytest

from numfast_b200 import device as dev
from tests.gpu_util import bitmap, to_dev

pytestmark = pytest.mark.gpu

_FIXTURES = [
    ("i64_null_mid", pd.array([1, 2, None, 1, 3], dtype="Int64")),
    ("f64_null_mid", pd.array([1.5, 2.5, None, 1.5, 3.5], dtype="Float64")),
    ("all_null_i64", pd.array([None, None, None], dtype="Int64")),
    ("null_free_i32", np.array([3, 1, 2, 1, 0], np.int32)),
    ("null_free_f64", np.array([3.0, 1.0, 2.0], np.float64)),
    ("null_extremes", pd.array([None, 5, 1, None, -3, 0], dtype="Int64")),
    ("null_among_negatives", pd.array([-1, None, -5, 0, None], dtype="Int64")),
    ("null_next_to_a_real_zero", pd.array([0, None, 0, 1], dtype="Int64")),
    ("two_nulls_same_value", pd.array([2, None, 1, None], dtype="Int64")),
    ("null_in_float_key", pd.array([9.0, None, 2.0, None, 1.0], dtype="Float64")),
    ("i32_8_4null", pd.array([3, None, 3, 1, None, None, 2, None], dtype="Int32")),
    ("i64_extremes", pd.array([2 ** 63 - 1, None, -2 ** 63, 0, -2 ** 63], dtype="Int64")),
]


def _device_column(col):
    s = pd.Series(col)
    valid = ~s.isna().to_numpy()
    if s.dtype in ("Int64", "Int32"):
        vals = s.fillna(0).to_numpy().astype(np.int64 if s.dtype == "Int64" else np.int32)
    elif s.dtype == "Float64":
        vals = s.fillna(0.0).to_numpy().astype(np.float64)
    else:
        vals = s.to_numpy()
    return vals, (None if valid.all() else valid)


@pytest.mark.parametrize("name,col", _FIXTURES, ids=[f[0] for f in _FIXTURES])
@pytest.mark.parametrize("desc", [False, True], ids=["asc", "desc"])
def test_sort_null_key_matches_pandas(cuda, name, col, desc):
    vals, valid = _device_column(col)
    perm = dev.sort_perm(to_dev(vals), desc, bitmap(valid)).cpu().numpy()
    want = pd.Series(col).sort_values(ascending=not desc, kind="stable", na_position="last").index.to_numpy()
    np.testing.assert_array_equal(perm, want, err_msg=name)
