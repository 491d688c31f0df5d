"""ctypes binding of libnumfast_cuda.so (the library's C ABI, include/numfast_cuda.h).

Loading mirrors the reference's native loader (src/Drivers/CPU/_lib/native_cpu.py:93-143):
``NUMFAST_CUDA_LIB`` (or ``NUMFAST_NATIVE_DLL`` when it names this library) overrides the
in-tree path.  There is no fallback: if the library cannot be loaded every entry point
raises ``NativeUnavailable`` -- the group-by path never silently runs on the CPU.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(HERE, "libnumfast_cuda.so")

# Return codes (numfast-native/src/core/errors.rs:13-38 + CUDA-specific ones).
OK = 0
ERR_NULL = -1
ERR_RANGE = -2
ERR_MALFORMED = -3
ERR_OVERFLOW = -4
ERR_UNSORTED = -5
ERR_CUDA = -6
ERR_TIMEOUT = -7
ERR_NOMEM = -8
ERR_UNSUPPORTED = -9

ERR_NAMES = {
    ERR_NULL: "null pointer / unsorted abort",
    ERR_RANGE: "out-of-range key / null state",
    ERR_MALFORMED: "malformed arguments",
    ERR_OVERFLOW: "integer overflow",
    ERR_UNSORTED: "unsorted input",
    ERR_CUDA: "CUDA error",
    ERR_TIMEOUT: "bounded device wait expired",
    ERR_NOMEM: "device allocation failed",
    ERR_UNSUPPORTED: "unsupported argument combination",
}

I32, I64, F64 = 0, 1, 2
AGG_SUM, AGG_MIN, AGG_MAX = 1, 2, 4
(STRAT_AUTO, STRAT_SORTED, STRAT_DENSE_SMEM, STRAT_DENSE_GLOBAL, STRAT_PARTITION, STRAT_HASH,
 STRAT_SHARED_HASH, STRAT_SORT) = range(8)
STRATEGY_NAMES = {
    STRAT_AUTO: "auto", STRAT_SORTED: "sorted", STRAT_DENSE_SMEM: "dense_smem",
    STRAT_DENSE_GLOBAL: "dense_global", STRAT_PARTITION: "partition", STRAT_HASH: "hash",
    STRAT_SHARED_HASH: "shared_hash", STRAT_SORT: "sort",
}
MAX_COLS = 4
MAX_KEY_COLS = 8  # NFC_MAX_KEY_COLS: columns of a bit-packed tuple key
NOALLOC_MAX_ROWS = 1 << 25
NOALLOC_STATE_BYTES = 24 << 20


class NativeUnavailable(RuntimeError):
    """libnumfast_cuda.so is missing or failed to load."""


class NativeError(RuntimeError):
    """A libnumfast_cuda entry point returned a negative code."""

    def __init__(self, where, code, detail=""):
        self.code = code
        msg = "%s failed: %d (%s)" % (where, code, ERR_NAMES.get(code, "unknown"))
        if detail:
            msg += ": " + detail
        super().__init__(msg)


class ValueCol(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int32),
        ("aggs", ctypes.c_int32),
        ("data", ctypes.c_void_p),
        ("validity", ctypes.c_void_p),
        ("sum_out", ctypes.c_void_p),
        ("min_out", ctypes.c_void_p),
        ("max_out", ctypes.c_void_p),
    ]


class GroupbyArgs(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64),
        ("keys", ctypes.c_void_p),
        ("key_validity", ctypes.c_void_p),
        ("ncols", ctypes.c_int32),
        ("cols", ctypes.POINTER(ValueCol)),
        ("out_cap", ctypes.c_int64),
        ("ukeys_out", ctypes.c_void_p),
        ("counts_out", ctypes.c_void_p),
        ("row_filter", ctypes.c_void_p),
    ]


class Probe(ctypes.Structure):
    _fields_ = [
        ("n_valid", ctypes.c_int64),
        ("kmin", ctypes.c_int64),
        ("kmax", ctypes.c_int64),
        ("sorted", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


class GroupbyStats(ctypes.Structure):
    _fields_ = [
        ("strategy", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("ng", ctypes.c_int64),
        ("probe", Probe),
        ("buckets", ctypes.c_int64),
        ("timing", ctypes.c_int32),
        ("launches", ctypes.c_int32),
        ("nstages", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("stage_ms", ctypes.c_float * 8),
        ("distinct_hint", ctypes.c_int64),
        ("overflowed", ctypes.c_int32),
        ("planner_used", ctypes.c_int32),
        ("predicted_distinct", ctypes.c_int64),
        ("learned_pick", ctypes.c_int32),
        ("fixed_pick", ctypes.c_int32),
    ]


class BatchTuning(ctypes.Structure):
    """nfc_batch_tuning: tile sizes and item schedule of the batched group-by."""
    _fields_ = [
        ("solo_rows", ctypes.c_int32),
        ("chunk_rows", ctypes.c_int32),
        ("probe_rows", ctypes.c_int32),
        ("emit_slice", ctypes.c_int32),
        ("emit_max_items", ctypes.c_int32),
        ("smem_slots", ctypes.c_int32),
        ("smem_span_div", ctypes.c_int32),
        ("warp_agg", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("agg_split", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("arena_bytes", ctypes.c_int64),
    ]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_ if not name.startswith("pad")}


MLP_IN, MLP_H, MLP_OUT = 280, 128, 5
MLP_NPARAMS, MLP_NWEIGHTS = 53125, 52864
PLANNER_AUTO, PLANNER_FIXED, PLANNER_LEARNED = 0, 1, 2
PICK_NAMES = ["dense", "shared_hash", "global_hash", "sort"]

BATCH_GRAPH = 1
BATCH_NO_SYNC = 2
BATCH_PLAN_NAMES = {0: "none", 1: "empty", 2: "smem", 3: "global", 4: "deferred", 5: "solo"}

_VP = ctypes.c_void_p
_SZ = ctypes.c_size_t
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_U64 = ctypes.c_uint64

# name -> (restype, argtypes); every symbol include/numfast_cuda.h declares.
SIGNATURES = {
    # numfast-native ABI (host pointers)
    "nf_group_sum_count": (_I32, [_VP, _VP, _SZ, _VP, _VP, _SZ]),
    "nf_group_multi_sum_count": (_I32, [_VP, _VP, _SZ, _SZ, _VP, _VP, _SZ]),
    "nf_group_mixed_sum_only": (_I32, [_VP, _VP, _VP, _SZ, _SZ, _SZ, _VP, _VP, _SZ]),
    "nf_group_count_only": (_I32, [_VP, _SZ, _VP, _SZ]),
    "nf_group_owner_2i32_1f64": (_I32, [_VP, _VP, _VP, _VP, _SZ, _SZ, _SZ, _VP, _VP, _VP, _VP, _SZ]),
    "nf_pack_i32_direct": (_I32, [_VP, _VP, _I32, _SZ, _VP]),
    "nf_pack_sum_count_i32": (_I32, [_VP, _VP, _I32, _VP, _SZ, _VP, _VP, _SZ]),
    "nf_pack_sum_count_f64": (_I32, [_VP, _VP, _I32, _VP, _SZ, _VP, _VP, _SZ]),
    "nf_pattern_encode": (_I32, [_VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP, _VP, _VP]),
    "nf_sorted_run_i64": (_I64, [_VP, _VP, _SZ, _VP, _VP, _VP]),
    "nf_sorted_run_f64": (_I64, [_VP, _VP, _SZ, _VP, _VP, _VP]),
    "nf_carry_build_i64": (_I64, [_VP, _VP, _SZ, _VP, _VP, _VP]),
    "nf_carry_build_f64": (_I64, [_VP, _VP, _SZ, _VP, _VP, _VP]),
    "nf_group_variant_f64": (_I32, [_VP, _VP, _SZ, ctypes.c_uint32, _VP, _VP, _SZ]),
    "nf_group_variant_i64": (_I32, [_VP, _VP, _SZ, ctypes.c_uint32, _VP, _VP, _SZ]),
    "nf_group_variant_i32": (_I32, [_VP, _VP, _SZ, ctypes.c_uint32, _VP, _VP, _SZ]),
    "nf_sort_perm_i32": (_I32, [_VP, _SZ, ctypes.c_uint8, _VP, _VP, _VP, _VP]),
    "nf_sort_perm_i64": (_I32, [_VP, _SZ, ctypes.c_uint8, _VP, _VP, _VP, _VP]),
    "nf_unique_inverse_i32": (_I64, [_VP, _SZ, _VP, _VP, _VP, _VP, _VP, _VP]),
    "nf_unique_inverse_i64": (_I64, [_VP, _SZ, _VP, _VP, _VP, _VP, _VP, _VP]),
    # nfc_* device extension
    "nfc_groupby": (_I64, [ctypes.POINTER(GroupbyArgs), _I32, _VP, ctypes.POINTER(GroupbyStats)]),
    "nfc_plan_strategy": (_I32, [ctypes.POINTER(GroupbyArgs), ctypes.POINTER(Probe)]),
    "nfc_sort_perm": (_I32, [_I32, _VP, _VP, _I64, _I32, _VP, _VP]),
    "nfc_sort_topk": (_I32, [_I32, _VP, _VP, _I64, _I32, _I64, _VP, _VP]),
    "nfc_gather": (_I32, [_I32, _VP, _I64, _VP, _I64, _VP, _VP]),
    "nfc_unique": (_I64, [_VP, _I64, _VP, _VP, _VP, _VP, _VP]),
    "nfc_group_count_distinct": (_I64, [_VP, _VP, _VP, _VP, _I64, _I64, _VP, _VP, _VP]),
    "nfc_composite_codes": (_I64, [_VP, ctypes.c_uint32, _VP, ctypes.c_uint32, _VP, _I64, _VP, _VP, _VP, _VP]),
    "nfc_key_ranges": (_I64, [_VP, _VP, _I32, _VP, _I64, _VP, _VP, _VP]),
    "nfc_pack_key_bits": (_I32, [_VP, _VP, _VP, _VP, _I32, _I64, _VP, _VP]),
    "nfc_unpack_key_bits": (_I32, [_VP, _I64, _VP, _VP, _VP, _I32, _VP, _VP]),
    "nfc_rng_fill_i32": (_I32, [_I64, _U64, _U64, _U64, _I64, _I64, _VP, _VP]),
    "nfc_rng_fill_f64": (_I32, [_I64, _U64, _U64, _U64, ctypes.c_double, ctypes.c_double, _VP, _VP]),
    "nfc_gen_lognormal": (_I32, [_I64, _U64, _U64, _U64, ctypes.c_double, ctypes.c_double, _VP, _VP]),
    "nfc_gen_zipf": (_I32, [_I64, _U64, _U64, ctypes.c_double, _I64, _VP, _VP]),
    "nfc_gen_validity": (_I32, [_I64, _U64, _U64, ctypes.c_double, _VP, _VP]),
    "nfc_groupby_dense_noalloc": (_I64, [ctypes.POINTER(GroupbyArgs), _VP]),
    "nfc_sketch": (_I32, [_VP, _VP, _I64, _VP, _VP]),
    "nfc_mlp_forward": (_I32, [_VP, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "nfc_mlp_backward": (_I32, [_VP, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "nfc_mlp_loss": (_I32, [_VP, _VP, _VP, _VP, _I64, ctypes.c_float, ctypes.c_float, _VP, _VP, _VP]),
    "nfc_mlp_adam": (_I32, [_VP, _VP, _VP, _VP, _VP, _I64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                            ctypes.c_float, ctypes.c_float, _VP]),
    "nfc_mlp_to_bf16": (_I32, [_VP, _VP, _VP]),
    "nfc_planner_create": (_VP, [_VP, _VP, _VP, ctypes.c_float]),
    "nfc_planner_destroy": (None, [_VP]),
    "nfc_plan_fixed": (_I32, [ctypes.POINTER(Probe), _I32]),
    "nfc_groupby_planned": (_I64, [ctypes.POINTER(GroupbyArgs), _I32, _VP, _VP, ctypes.POINTER(GroupbyStats)]),
    "nfc_batch_default_tuning": (None, [ctypes.POINTER(BatchTuning)]),
    "nfc_batch_create": (_VP, [_I64, _VP, ctypes.POINTER(BatchTuning)]),
    "nfc_batch_run": (_I64, [_VP, _VP, _VP, _VP, _VP, _I64, _VP, _VP, _VP, _VP, _VP, _I32, _VP]),
    "nfc_batch_finish": (_I64, [_VP, _VP]),
    "nfc_batch_query_plans": (_I32, [_VP, _VP, _VP]),
    "nfc_batch_profile": (_I32, [_VP, _VP, _VP]),
    "nfc_batch_info": (_I32, [_VP, _VP, _I32]),
    "nfc_batch_destroy": (None, [_VP]),
    "nfc_last_error": (ctypes.c_char_p, []),
    "nfc_version": (_I32, []),
    "nfc_selftest_bounded_waits": (_I32, [ctypes.c_uint32, _VP, _VP]),
    "nfc_debug_fail_alloc": (_I32, [_I64]),
}

_lib = None
_why = "unprobed"


def lib_path():
    p = os.environ.get("NUMFAST_CUDA_LIB")
    if p:
        return p
    p = os.environ.get("NUMFAST_NATIVE_DLL", "")
    if p.endswith("libnumfast_cuda.so"):
        return p
    return DEFAULT_LIB


def load():
    """Load and argtype the library (memoised); raises NativeUnavailable."""
    global _lib, _why
    if _lib is not None:
        return _lib
    path = lib_path()
    try:
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    except (OSError, AttributeError) as e:
        _why = "unavailable: %s" % e
        raise NativeUnavailable("libnumfast_cuda could not be loaded from %s: %s" % (path, e)) from e
    _lib, _why = lib, "loaded:" + path
    return lib


def last_error():
    return load().nfc_last_error().decode("utf-8", "replace")


def check(where, rc):
    """Raise NativeError on a negative return code; pass through otherwise."""
    if rc < 0:
        raise NativeError(where, int(rc), last_error())
    return rc
