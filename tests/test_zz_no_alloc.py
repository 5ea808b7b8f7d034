"""vie_matvec_static: the operator application that allocates no device memory.

It exists for callers that must not allocate while they apply the operator
(a loop that cannot take the device-wide synchronisation of a cudaFree per
call, or a process whose free device memory belongs to another allocator).
Its scratch is one static device array shared by every call, so this test
calls it twice in a row, with different inputs and with A and A^H, and checks
each result against the allocating entry point vie_matvec.  The file is named
to be collected last.
"""
import ctypes

import numpy as np
import pytest

import vie_fft_b200 as V
from vie_fft_b200 import geometry as GEO

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-12  # the operator tolerance of tests/test_operator_gpu.py


def static_matvec(ctx, x, conj):
    lib = V.lib()
    fn = lib.vie_matvec_static
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    fn.restype = ctypes.c_int
    x = np.ascontiguousarray(x, np.complex128)
    y = np.empty_like(x)
    rc = fn(ctx.handle, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(conj))
    return rc, y


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_static_scratch_matvec_matches_allocating_matvec_twice():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    w = GEO.single_sphere()  # 32^3: 12.6 MB of the 64 MiB scratch
    rng = np.random.default_rng(21)
    with V.Context(*w.shape, *w.d, w.k0) as c:
        c.set_flags(w.flags)
        c.set_material(w.material, w.eps_table)
        c.green()
        for call, conj in enumerate((False, True)):
            x = rng.standard_normal((3,) + w.shape) + 1j * rng.standard_normal((3,) + w.shape)
            # the second call is warm (kernels loaded, scratch address known):
            # the device's free memory must not move across it
            free0 = torch.cuda.mem_get_info(c.device)[0]
            rc, y = static_matvec(c, x, conj)
            free1 = torch.cuda.mem_get_info(c.device)[0]
            assert rc == V.VIE_OK, (call, V.lib().vie_last_error(c.handle))
            if call:
                assert free1 == free0
            assert rel(y, c.matvec(x, conj=conj)) < FP64_TOL


def test_static_scratch_rejects_grids_beyond_its_size():
    n = 64  # 262144 voxels > 174762
    rng = np.random.default_rng(22)
    with V.Context(n, n, n, 0.01, 0.01, 0.01, 1.0) as c:
        c.set_flags(np.ones((3, n, n, n), np.uint8))
        c.set_material(np.full((n, n, n), 1, np.uint8), [1.1, 2.0])
        c.green()
        rc, _ = static_matvec(c, rng.standard_normal((3, n, n, n)) + 0j, False)
        assert rc == V.VIE_ERR_ARG
        assert b"static scratch" in V.lib().vie_last_error(c.handle)
