"""The drop-in headers' error exit, on the CPU.

The reference checks no status; the void drop-in functions (dropin/vie_dropin.h)
print the library's message to stderr and exit the process with status 1 when
a library call fails.  Here the first call that needs a context
(Green_Function_Compute through the drop-in harness) is given a device ordinal
that no machine has (VIE_DEVICE=999), so vie_create fails before any GPU work
on every machine; the child process must exit with status 1 and name the
failing call.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "dropin", "_build", "libvie_dropin_harness.so")

CHILD = r"""
import ctypes, sys
import numpy as np
L = ctypes.CDLL(sys.argv[1])
dp = ctypes.POINTER(ctypes.c_double)
L.dh_setup.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [dp, dp] + [ctypes.c_double] * 3
L.dh_green.argtypes = [dp]
re = np.array([1.1, 2.0, -4.42, 3.8]); im = np.array([0.0, 0.0, -0.21, -0.6])
assert L.dh_setup(8, 8, 8, 0.01, 0.01, 0.01, 12.0, re.ctypes.data_as(dp), im.ctypes.data_as(dp), 0.0, 0.0, 0.0) == 0
L.dh_green(None)
print("returned")
"""


def test_failed_library_call_exits_with_status_1():
    if not os.path.exists(HARNESS):
        pytest.skip("drop-in harness not built (needs the reference sources: make -C dropin)")
    env = dict(os.environ, VIE_DEVICE="999")
    run = subprocess.run([sys.executable, "-c", CHILD, HARNESS], env=env, stdout=subprocess.PIPE,
                         stderr=subprocess.PIPE, text=True, timeout=300)
    assert run.returncode == 1, (run.returncode, run.stdout, run.stderr)
    assert "returned" not in run.stdout
    assert "vie_b200: vie_create failed:" in run.stderr, run.stderr
