"""numfast_b200: NumFast's group-by hot path on B200 (sm_100a).

Layers:
  libnumfast_cuda.so   hand-written CUDA kernels behind a C ABI (include/numfast_cuda.h):
                       the numfast-native nf_* symbols (host buffers) and the nfc_*
                       device extension (device buffers, validity bitmaps, streams)
  _lib                 ctypes binding (loud failure when the library is missing)
  device               torch-tensor front end of the nfc_* entry points
  executor / ir        IR nodes series / groupby_multi / sort / gather / unique_inverse
  chain                Table.query().filter().group().sort().compile()
  carry                ColumnCarry result object
"""

from ._lib import NativeError, NativeUnavailable  # noqa: F401
from .carry import ColumnCarry  # noqa: F401
from .chain import Table, from_numpy  # noqa: F401
from .ir import ir_filter, ir_gather, ir_groupby_multi, ir_series, ir_sort, ir_unique_inverse  # noqa: F401

__version__ = "0.1.0"


def build_native(force=False):
    """Compile libnumfast_cuda.so in-tree (nvcc, sm_100a)."""
    from .native_build import build as _b
    return _b(force=force)


def execute(jobs, bufs=None):
    from .executor import execute as _e
    return _e(jobs, bufs)
