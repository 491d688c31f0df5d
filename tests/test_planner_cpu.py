"""Planner pieces that need no GPU: the fixed rule against the reference's own
decisions, and the CPU oracle of the MLP (finite-difference gradient check)."""

import ctypes
import json
import os

import numpy as np
import pytest

from numfast_b200 import _lib
from oracle import planner_oracle as P

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden_cases():
    with open(os.path.join(HERE, "golden", "plan_fixed.json")) as f:
        d = json.load(f)
    return [dict(zip(d["fields"], c)) for c in d["cases"]]


def test_oracle_fixed_rule_matches_reference_decisions():
    for c in _golden_cases():
        want = {"dense_by_code": "dense", "dense": "dense", "hash": "hash", "sorted": "sorted"}[c["strategy"]]
        got = P.plan_fixed_class(c["n"], c["span"], c["kmin"], c["naggs"], c["sorted"])
        assert got == want, c


def test_library_fixed_rule_matches_reference_decisions():
    lib = _lib.load()
    for c in _golden_cases():
        pr = _lib.Probe()
        pr.n_valid = c["n"]
        pr.kmin = c["kmin"]
        pr.kmax = c["kmin"] + c["span"] - 1
        pr.sorted = 1 if c["sorted"] else 0
        s = lib.nfc_plan_fixed(ctypes.byref(pr), c["naggs"])
        got = {_lib.STRAT_SORTED: "sorted", _lib.STRAT_SORT: "hash"}.get(s, "dense")
        want = {"dense_by_code": "dense", "dense": "dense", "hash": "hash", "sorted": "sorted"}[c["strategy"]]
        assert got == want, (c, s)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-30], dtype=np.float32)
    r = P.bf16(x)
    # Exactly representable values stay; others land on a bf16 grid point.
    assert r[0] == 1.0
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)
    # Ties go to even: 1 + 2^-8 is halfway between 1 and 1 + 2^-7.
    assert r[1] == 1.0


def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    params = P.init_params(1)
    x = rng.normal(size=(6, P.IN)).astype(np.float32)
    y = rng.uniform(0, 1, 6)
    lab = np.array([0, 3, -1, 2, 1, 0])

    def loss_at(p):
        _, _, _, out = P.mlp_forward(x, p)
        return P.mlp_loss(out, y, lab, 1.0, 0.5)[0]

    _, _, _, out = P.mlp_forward(x, params)
    _, dout = P.mlp_loss(out, y, lab, 1.0, 0.5)
    g = P.mlp_backward(x, params, dout)
    # Biases are float32 (no bf16 rounding), so central differences apply directly.
    offs = P.offsets()
    for name in ("b1", "b2", "b3"):
        o, s = offs[name]
        for j in range(0, s[0], max(1, s[0] // 8)):
            e = np.zeros(P.NPARAMS, np.float64)
            e[o + j] = 1e-3
            fd = (loss_at(params + e) - loss_at(params - e)) / 2e-3
            assert abs(fd - g[o + j]) <= 1e-4 + 1e-3 * abs(fd), (name, j, fd, g[o + j])


def test_sketch_oracle_basic_properties():
    rng = np.random.default_rng(0)
    k = rng.integers(0, 1000, 100_000).astype(np.int32)
    f = P.sketch(k)
    assert f.shape == (P.IN,) and f.dtype == np.float32
    est = 2 ** (f[256 + 3] * 32) - 1
    assert 850 < est < 1150  # HLL-256 on 1000 distinct: a few percent error
    runs = np.repeat(np.arange(50, dtype=np.int32), 2000)
    g = P.sketch(runs)
    assert g[256 + 5] > 0.99  # adjacent equal pairs
