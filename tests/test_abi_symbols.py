"""The C-ABI library loads and exports every symbol include/numfast_cuda.h declares
(no GPU needed: nothing here calls into a kernel)."""

import ctypes
import os
import re
import subprocess

import pytest

from numfast_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "numfast_cuda.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nfc?_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def libpath():
    from numfast_b200 import native_build
    return native_build.build()


def test_header_declares_reference_loader_symbols():
    syms = declared_symbols()
    # native_cpu._probe() requires these 8 (native_cpu.py:125-141).
    for s in ["nf_group_sum_count", "nf_group_multi_sum_count", "nf_pack_i32_direct", "nf_pattern_encode",
              "nf_sorted_run_i64", "nf_sorted_run_f64", "nf_carry_build_i64", "nf_carry_build_f64"]:
        assert s in syms


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (nfc?_\w+)", out))
    assert set(declared_symbols()) <= exported


def test_python_binding_covers_header(libpath):
    assert set(declared_symbols()) == set(_lib.SIGNATURES)
    lib = _lib.load()
    assert lib.nfc_version() >= 1
    assert isinstance(lib.nfc_last_error(), bytes)


def test_host_validation_without_gpu(libpath):
    """Argument checks run on the host before any CUDA call."""
    lib = _lib.load()
    assert lib.nf_group_sum_count(None, None, 0, None, None, 0) == _lib.ERR_NULL
    assert lib.nf_sort_perm_i32(None, 0, 0, None, None, None, None) == _lib.OK  # n == 0: no deref
    assert lib.nf_sorted_run_i64(None, None, 0, None, None, None) == 0
    assert lib.nf_carry_build_f64(None, None, 5, None, None, None) == _lib.ERR_RANGE
    assert lib.nfc_rng_fill_i32(10, 42, 0, 0, 5, 5, None, None) == _lib.ERR_RANGE
    assert lib.nfc_groupby(None, 0, None, None) == _lib.ERR_NULL


def test_pack_and_pattern_host_symbols(libpath):
    import numpy as np
    lib = _lib.load()
    k1 = np.array([0, 1, 2], dtype=np.int32)
    k2 = np.array([3, 4, 5], dtype=np.int32)
    out = np.zeros(3, dtype=np.int32)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)
    assert lib.nf_pack_i32_direct(vp(k1), vp(k2), 10, 3, vp(out)) == 0
    assert out.tolist() == [3, 14, 25]
    k1[0] = -1
    assert lib.nf_pack_i32_direct(vp(k1), vp(k2), 10, 3, vp(out)) == _lib.ERR_RANGE
    rows = [b"id-12", b"id--7", b"x9", b"id-", b"id-2147483648"]
    data = np.frombuffer(b"".join(rows), dtype=np.uint8).copy()
    offs = np.cumsum([0] + [len(r) for r in rows]).astype(np.int32)
    pre = np.frombuffer(b"id-", dtype=np.uint8).copy()
    codes = np.zeros(len(rows), dtype=np.int32)
    valid = np.zeros(len(rows), dtype=np.uint8)
    w = np.zeros(1, dtype=np.int32)
    e = np.zeros(1, dtype=np.int32)
    rc = lib.nf_pattern_encode(vp(data), data.size, vp(offs), len(rows) - 1, vp(pre), pre.size, vp(codes),
                               vp(valid), vp(w), vp(e))
    assert rc == 0
    assert codes[:4].tolist() == [12, -7, 0, 0] and valid[:4].tolist() == [1, 1, 0, 0] and w[0] == 2
    rc = lib.nf_pattern_encode(vp(data), data.size, vp(offs), len(rows), vp(pre), pre.size, vp(codes),
                               vp(valid), vp(w), vp(e))
    assert rc == _lib.ERR_RANGE and e[0] == 4
