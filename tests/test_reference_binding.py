"""The reference's own native loader binds libnumfast_cuda.so as its native library.

The reference host loads its native backend with ctypes from NUMFAST_NATIVE_DLL
(src/Drivers/CPU/_lib/native_cpu.py:93-143) and probes each optional hot-path group
separately (variant :324-352, mixed :503-533, owner :548-575, fused :621-651,
unique :1399-1431, sort :1546-1576).  This test runs that loader, unmodified, from a
reference checkout against the library built here, in a fresh interpreter, and checks
that every group binds.  Binding sets argtypes only, so no GPU is needed.  Skipped when
no reference checkout is available (NUMFAST_REFERENCE or the default location).
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("NUMFAST_REFERENCE", "/root/reference")

PROBE = r"""
import importlib, json
nc = importlib.import_module("Drivers.CPU._lib.native_cpu")
out = {"available": nc.available(), "why": nc.why()}
for name in ("variant_available", "mixed_available", "owner_available", "fused_available",
             "unique_available", "sort_available"):
    out[name] = bool(getattr(nc, name)())
print(json.dumps(out))
"""


@pytest.fixture(scope="module")
def libpath():
    from numfast_b200 import native_build
    return native_build.build()


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src", "Drivers", "CPU", "_lib")),
                    reason="no reference checkout")
def test_reference_loader_binds_every_group(libpath, tmp_path):
    env = dict(os.environ, NUMFAST_NATIVE_DLL=libpath, PYTHONPATH=os.path.join(REF, "src"),
               PYTHONDONTWRITEBYTECODE="1")
    env.pop("NUMFAST_NATIVE_DISABLE", None)
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=str(tmp_path), env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got["available"], got["why"]
    assert got["why"] == "loaded:" + libpath
    for name in ("variant_available", "mixed_available", "owner_available", "fused_available",
                 "unique_available", "sort_available"):
        assert got[name], name
