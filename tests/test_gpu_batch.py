"""Batched group-by (nfc_batch_*): every query bit-exact against the oracle.

Each query of a batch is one executor groupby_multi node with ops ("sum", "count")
(src/Drivers/CPU/_lib/cpu.py:3435-3704).  The cases cover every plan the kernel can
take (solo, shared-memory, global, empty, deferred), NULL bitmaps, the graph and the
plain launch, every tuning option the autotuner can pick, unaligned inputs, deferral by
value magnitude and by output capacity, and the full-size 4,096-query workload through
size-independent properties.
"""

import numpy as np
import pytest
import torch

from numfast_b200 import _lib
from numfast_b200 import batch as B
from numfast_b200 import device as dev
from oracle import nf_oracle as O

pytestmark = pytest.mark.gpu


def _small_layout(nq, seed, max_rows=200_000):
    lay = B.config4_layout(nq=nq, seed=seed, min_rows=1, max_rows=max_rows)
    return lay


def _unpack(bm_u8, n):
    return np.unpackbits(bm_u8.cpu().numpy(), bitorder="little")[:n].astype(bool)


_REF = {}


def _reference(keys, vals, ro, kv=None, vv=None):
    key = (keys.data_ptr(), vals.data_ptr(), keys.numel(), kv is not None, vv is not None)
    if key not in _REF:
        hk, hv = keys.cpu().numpy(), vals.cpu().numpy()
        n = hk.size
        kmask = _unpack(kv, n) if kv is not None else None
        vmask = _unpack(vv, n) if vv is not None else None
        _REF[key] = O.batch_sum_count(hk, hv, ro, kmask, vmask)
    return _REF[key]


def _check(res, keys, vals, ro, kv=None, vv=None):
    ref = _reference(keys, vals, ro, kv, vv)
    offs = res.group_offsets.cpu().numpy()
    ngs = res.ngroups.cpu().numpy()
    uk, su, co = res.ukeys.cpu().numpy(), res.sums.cpu().numpy(), res.counts.cpu().numpy()
    for q, (rk, rs, rc) in enumerate(ref):
        ng = int(ngs[q])
        assert ng == rk.size, (q, ng, rk.size)
        sl = slice(int(offs[q]), int(offs[q]) + ng)
        np.testing.assert_array_equal(uk[sl], rk, err_msg="ukeys q=%d" % q)
        np.testing.assert_array_equal(co[sl], rc, err_msg="counts q=%d" % q)
        np.testing.assert_array_equal(su[sl], rs, err_msg="sums q=%d" % q)


@pytest.fixture(scope="module")
def mixed():
    """300 queries of 1..200K rows with 5% NULL keys and values, plus special queries:
    an empty one, an all-NULL one, one with sparse keys (deferred) and one sorted."""
    lay = _small_layout(300, 7)
    keys, vals = B.make_config4(lay)
    ro = lay["row_offsets"].copy()
    n = int(ro[-1])
    extra = [np.zeros(0, np.int32), np.arange(5000, dtype=np.int32), np.array([-2 ** 31, 2 ** 31 - 1] * 3000,
                                                                              dtype=np.int32),
             np.sort(np.random.default_rng(3).integers(-50, 50, 70_000)).astype(np.int32)]
    ek = np.concatenate(extra)
    ev = np.random.default_rng(4).integers(-1000, 1001, ek.size).astype(np.int32)
    keys = torch.cat([keys, torch.from_numpy(ek).cuda()])
    vals = torch.cat([vals, torch.from_numpy(ev).cuda()])
    sizes = [e.size for e in extra]
    ro = np.concatenate([ro, n + np.cumsum(sizes)])
    total = int(ro[-1])
    kv = dev.gen_validity(total, 42, 100, 0.05)
    vv = dev.gen_validity(total, 42, 101, 0.05)
    # The second special query (rows 5000) has every key NULL.
    a = int(ro[-4])
    km = _unpack(kv, total)
    km[a:a + 5000] = False
    kv = torch.from_numpy(np.packbits(km, bitorder="little")).cuda()
    return keys, vals, ro, kv, vv


def test_batch_mixed_default_tuning(mixed):
    keys, vals, ro, kv, vv = mixed
    b = B.BatchGroupby(ro)
    for graph in (False, True):
        res = b.run(keys, vals, kv, vv, graph=graph)
        _check(res, keys, vals, ro, kv, vv)
    plans = b.plans()
    assert {"solo", "smem", "global", "empty", "deferred"} <= set(plans), sorted(set(plans))
    assert res.deferred >= 1
    b.close()


def test_batch_without_validity_and_repeat(mixed):
    keys, vals, ro, _, _ = mixed
    b = B.BatchGroupby(ro)
    first = None
    for _ in range(3):  # state arena must come back clean after every run
        res = b.run(keys, vals, graph=True)
        cur = (res.ukeys.clone(), res.sums.clone(), res.counts.clone(), res.group_offsets.clone(),
               res.ngroups.clone())
        _check(res, keys, vals, ro)
        if first is not None:
            # Reservation order may differ between runs; per-query content may not.
            for q in range(len(ro) - 1):
                o0, n0 = int(first[3][q]), int(first[4][q])
                o1, n1 = int(cur[3][q]), int(cur[4][q])
                assert n0 == n1
                for i in range(3):
                    assert torch.equal(first[i][o0:o0 + n0], cur[i][o1:o1 + n1])
        first = cur
    b.close()


@pytest.mark.parametrize("knob", [name for name, _ in B.SEARCH_SPACE])
def test_batch_every_tuning_option(mixed, knob):
    keys, vals, ro, kv, vv = mixed
    options = dict(B.SEARCH_SPACE)[knob]
    for opt in options:
        t = B.tuning_from_dict(dict(B.default_tuning().as_dict(), **opt))
        b = B.BatchGroupby(ro, t)
        res = b.run(keys, vals, kv, vv, graph=True)
        _check(res, keys, vals, ro, kv, vv)
        b.close()


def test_batch_unaligned_inputs(mixed):
    keys, vals, ro, _, _ = mixed
    k1 = torch.empty(keys.numel() + 1, dtype=torch.int32, device="cuda")
    v1 = torch.empty_like(k1)
    k1[1:] = keys
    v1[1:] = vals
    b = B.BatchGroupby(ro)
    res = b.run(k1[1:], v1[1:], graph=False)
    _check(res, keys, vals, ro)
    b.close()


def test_batch_large_values_are_deferred_exactly():
    """|value| * rows beyond the packed 64-bit state's bound: such queries go to the
    single-query path and stay exact; small ones still run in the kernel."""
    lay = _small_layout(40, 11, max_rows=300_000)
    keys, _ = B.make_config4(lay)
    n = keys.numel()
    vals = dev.rng_fill_i32(n, 42, 500, -2 ** 31, 2 ** 31)
    ro = lay["row_offsets"]
    b = B.BatchGroupby(ro)
    res = b.run(keys, vals)
    _check(res, keys, vals, ro)
    assert res.deferred >= 1
    b.close()


def test_batch_small_output_capacity_defers():
    """A query whose reservation min(rows, span) does not fit is deferred without using
    up the capacity; the host-side path then places its groups in what is left."""
    k0 = dev.rng_fill_i32(200_000, 42, 600, 1000, 51_000)  # span 50,000, about 49,000 groups
    k1 = dev.rng_fill_i32(3_000, 42, 601, 0, 100)
    keys = torch.cat([k0, k1])
    vals = dev.rng_fill_i32(keys.numel(), 42, 602, -1000, 1001)
    ro = np.array([0, 200_000, 203_000], dtype=np.int64)
    ref = _reference(keys, vals, ro)
    need = sum(r[0].size for r in ref)
    assert need < 50_000
    b = B.BatchGroupby(ro)
    res = b.run(keys, vals, out_cap=need + 8)
    _check(res, keys, vals, ro)
    assert res.deferred == 1
    assert b.plans()[0] == "deferred"
    # Too small even for the groups themselves: a clean overflow error.
    with pytest.raises(_lib.NativeError) as ei:
        b.run(keys, vals, out_cap=need // 2)
    assert ei.value.code == _lib.ERR_OVERFLOW
    b.close()


def test_batch_full_size_properties():
    """The 4,096-query workload (rows 1K..4M, about 1.9e9 rows): no deferred query,
    per-query counts and sums equal to the per-query valid rows and value sums, and
    keys strictly ascending inside every query."""
    lay = B.config4_layout()
    keys, vals = B.make_config4(lay)
    ro = lay["row_offsets"]
    nq = ro.size - 1
    n = int(ro[-1])
    b = B.BatchGroupby(ro)
    res = b.run(keys, vals, out_cap=n // 4, graph=True)
    assert res.deferred == 0
    ng = res.ngroups
    off = res.group_offsets
    total = int(ng.sum())
    qid = torch.repeat_interleave(torch.arange(nq, device="cuda"), ng)
    start = torch.cumsum(ng, 0) - ng
    pos = torch.repeat_interleave(off, ng) + torch.arange(total, device="cuda") - torch.repeat_interleave(start, ng)
    uk, su, co = res.ukeys[pos], res.sums[pos], res.counts[pos]
    cnt_q = torch.zeros(nq, dtype=torch.int64, device="cuda").index_add_(0, qid, co)
    sum_q = torch.zeros(nq, dtype=torch.int64, device="cuda").index_add_(0, qid, su)
    rows_q = torch.from_numpy(np.diff(ro)).cuda()
    assert torch.equal(cnt_q, rows_q)
    row_q = torch.repeat_interleave(torch.arange(nq, device="cuda"), rows_q)
    vsum_q = torch.zeros(nq, dtype=torch.int64, device="cuda").index_add_(0, row_q, vals.long())
    assert torch.equal(sum_q, vsum_q)
    same = qid[1:] == qid[:-1]
    assert bool(((uk[1:] > uk[:-1]) | ~same).all())
    assert bool((co > 0).all())
    # Spot-check a few queries bit-exact against the oracle.
    hk, hv = keys.cpu().numpy(), vals.cpu().numpy()
    for q in (0, 1, nq // 2, nq - 1):
        a, e = int(ro[q]), int(ro[q + 1])
        ((rk, rs, rc),) = O.batch_sum_count(hk[a:e], hv[a:e], np.array([0, e - a]))
        gk, gs, gc = res.query(q)
        np.testing.assert_array_equal(gk, rk)
        np.testing.assert_array_equal(gs, rs)
        np.testing.assert_array_equal(gc, rc)
    b.close()
