"""The C-ABI library loads and exports every entry point include/*.h declares.
No compute calls: these run on machines without a GPU."""
import ctypes
import glob
import os
import re

import pytest

import vie_fft_b200 as V

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"^VIE_API\s+[\w\s\*]+?\b(vie_\w+)\s*\(", src, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ["vie_create", "vie_destroy", "vie_green", "vie_incident", "vie_matvec", "vie_solve"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(V.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_library_exports_nothing_undeclared():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", V.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l and l.split()[-1].startswith("vie_")}
    assert exported == set(declared_symbols())


def test_status_strings_and_version():
    L = V.lib()
    assert L.vie_status_string(0) == b"ok"
    assert L.vie_status_string(V.VIE_ERR_MAXIT) == b"iteration cap reached"
    assert b"sm_100a" in L.vie_version()


def test_create_rejects_bad_grids_before_touching_a_device():
    L = V.lib()
    h = ctypes.c_void_p()
    for bad in [(1, 4, 4, 0.01), (4, 4, 4, -0.01), (4, 4, 4, 0.0)]:
        g = V.VieGrid(bad[0], bad[1], bad[2], bad[3], 0.01, 0.01, 1.0, 0)
        assert L.vie_create(ctypes.byref(g), ctypes.byref(h)) == V.VIE_ERR_ARG
        assert not h.value


def test_create_without_gpu_reports_no_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(V.VieError) as e:
        V.Context(4, 4, 4, 0.01, 0.01, 0.01, 1.0)
    assert e.value.status == V.VIE_ERR_NODEVICE
