"""The two loader-required symbols that run on the host (off the group-by path):
nf_pattern_encode (prefix + integer string encode) and nf_pack_i32_direct, checked
against the contract of the reference's transform/pattern.rs and lib.rs:262 (no GPU
needed: neither calls a kernel)."""

import ctypes

import numpy as np
import pytest



def vp(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.fixture(scope="module")
def lib():
    from numfast_b200 import native_build
    return ctypes.CDLL(native_build.build())


def encode(lib, rows, prefix):
    blob = b"".join(rows)
    offs = np.zeros(len(rows) + 1, dtype=np.int32)
    offs[1:] = np.cumsum([len(r) for r in rows])
    data = np.frombuffer(blob or b"\0", dtype=np.uint8).copy()
    pre = np.frombuffer(prefix or b"\0", dtype=np.uint8).copy()
    codes = np.full(len(rows), 7, dtype=np.int32)
    valid = np.full(len(rows), 9, dtype=np.uint8)
    width = ctypes.c_int32(0)
    err = ctypes.c_int32(0)
    rc = lib.nf_pattern_encode(vp(data), ctypes.c_size_t(len(blob)), vp(offs), ctypes.c_size_t(len(rows)),
                               vp(pre), ctypes.c_size_t(len(prefix)), vp(codes), vp(valid),
                               ctypes.byref(width), ctypes.byref(err))
    return rc, codes, valid, width.value, err.value


def test_pattern_encode_rows(lib):
    rows = [b"id007", b"id-12", b"id", b"x12", b"id1a", b"id2147483647", b"id-2147483648", b"id0000000000042"]
    rc, codes, valid, width, err = encode(lib, rows, b"id")
    assert rc == 0 and err == -1
    # non-matching prefix, empty body and non-digits are invalid rows (code 0), never errors
    assert valid.tolist() == [1, 1, 0, 0, 0, 1, 1, 1]
    assert codes.tolist() == [7, -12, 0, 0, 0, 2147483647, -2147483648, 42]
    assert width == 13  # widest digit core over valid rows, leading zeros included


def test_pattern_encode_overflow_and_malformed(lib):
    rc, codes, valid, width, err = encode(lib, [b"k1", b"k2147483648", b"k3"], b"k")
    assert rc == -2 and err == 1                       # value-based int32 overflow is an error
    assert codes[:2].tolist() == [1, 0] and valid[:2].tolist() == [1, 0]
    rc, *_ = encode(lib, [b"k00000000000000000000000005"], b"k")
    assert rc == 0                                     # leading zeros never fake an overflow
    data = np.frombuffer(b"k1k2", dtype=np.uint8).copy()
    offs = np.array([0, 3, 2], dtype=np.int32)         # regressing offsets
    out = np.zeros(2, dtype=np.int32)
    val = np.zeros(2, dtype=np.uint8)
    w, e = ctypes.c_int32(0), ctypes.c_int32(0)
    pre = np.frombuffer(b"k", dtype=np.uint8).copy()
    assert lib.nf_pattern_encode(vp(data), ctypes.c_size_t(4), vp(offs), ctypes.c_size_t(2), vp(pre),
                                 ctypes.c_size_t(1), vp(out), vp(val), ctypes.byref(w), ctypes.byref(e)) == -3


def test_pack_i32_direct(lib):
    k1 = np.array([0, 3, 7], dtype=np.int32)
    k2 = np.array([5, 0, 9], dtype=np.int32)
    out = np.zeros(3, dtype=np.int32)
    assert lib.nf_pack_i32_direct(vp(k1), vp(k2), ctypes.c_int32(10), ctypes.c_size_t(3), vp(out)) == 0
    assert out.tolist() == [5, 30, 79]
    neg = np.array([1, -1, 2], dtype=np.int32)
    assert lib.nf_pack_i32_direct(vp(neg), vp(k2), ctypes.c_int32(10), ctypes.c_size_t(3), vp(out)) == -2
    big = np.array([2 ** 30, 0, 0], dtype=np.int32)
    assert lib.nf_pack_i32_direct(vp(big), vp(k2), ctypes.c_int32(4), ctypes.c_size_t(3), vp(out)) == -2
