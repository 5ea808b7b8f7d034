"""The bounded waits of the staged passes: when a tile's wait runs out, the
call returns VIE_ERR_TIMEOUT and the device stays usable.

VIE_WAIT_TEST=1 makes every staged tile's first wait poll an mbarrier that
nothing completes (a short limit), so the timeout path runs without any fault:
the block records the timeout in the status word, waits for its real copy to
land and leaves its tile undone.  A context made afterwards without the switch
computes the operator as before.
"""
import ctypes

import numpy as np
import pytest

import vie_fft_b200 as V
from oracle import oracle as O
from vie_fft_b200 import geometry as GEO

pytestmark = pytest.mark.gpu


def _static_matvec(c, x):
    """vie_matvec_static through the C ABI: (status, y)."""
    fn = V.lib().vie_matvec_static
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    fn.restype = ctypes.c_int
    x = np.ascontiguousarray(x, np.complex128)
    y = np.zeros_like(x)
    dp = ctypes.POINTER(ctypes.c_double)
    return fn(c.handle, x.ctypes.data_as(dp), y.ctypes.data_as(dp), 0), y


def _ctx(shape, mat, flags, table):
    c = V.Context(*shape, 0.01, 0.01, 0.01, GEO.k0_of(500.0))
    c.set_flags(flags)
    c.set_material(mat, table)
    c.green()
    return c


def test_wait_timeout_is_reported_and_device_stays_usable(monkeypatch):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    shape = (16, 16, 16)  # every axis on the register kernels (staged y tiles and z rows)
    rng = np.random.default_rng(3)
    table = np.array([1.1, 2.4 - 0.05j, -4.4 - 0.2j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)

    monkeypatch.setenv("VIE_WAIT_TEST", "1")
    with _ctx(shape, mat, flags, table) as c:
        with pytest.raises(V.VieError) as e:
            c.matvec(x)
        assert e.value.status == V.VIE_ERR_TIMEOUT
        xt = torch.from_numpy(x.astype(np.complex64)).cuda()
        yt = torch.zeros_like(xt)
        torch.cuda.synchronize()
        c.matvec_dev(xt.data_ptr(), yt.data_ptr(), precision=V.PREC_MIXED)
        with pytest.raises(V.VieError) as e:
            c.sync()
        assert e.value.status == V.VIE_ERR_TIMEOUT
        c.incident()
        with pytest.raises(V.VieError) as e:
            c.solve("bicgstab", tol=1e-8, max_iter=2, allow_maxit=True)
        assert e.value.status == V.VIE_ERR_TIMEOUT
        # the operator that allocates nothing stages the same z rows
        rc, _ = _static_matvec(c, x)
        assert rc == V.VIE_ERR_TIMEOUT
        # the words were cleared by that call: the next call reports its own status only
        assert V.lib().vie_sync(c.handle) == V.VIE_OK
    monkeypatch.delenv("VIE_WAIT_TEST")

    g = O.Grid(*shape, 0.01, 0.01, 0.01, GEO.k0_of(500.0))
    ref = O.matvec(g, O.green(g), table[mat], flags, x)
    with _ctx(shape, mat, flags, table) as c:
        y = c.matvec(x)
        rc, ys = _static_matvec(c, x)
    assert np.abs(y - ref).max() < 1e-12 * np.abs(ref).max()
    assert rc == V.VIE_OK and np.abs(ys - ref).max() < 1e-12 * np.abs(ref).max()
