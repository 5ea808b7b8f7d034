"""FFT schedule autotuner (vie_autotune): the tuned operators still match the
oracle, other contexts of the same grid reuse the choice, and the choice
survives in the VIE_TUNE_CACHE file for a new process."""
import os
import subprocess
import sys

import numpy as np
import pytest

import vie_fft_b200 as V
from oracle import oracle as O
from vie_fft_b200 import geometry as GEO

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def setup(shape, seed=3):
    rng = np.random.default_rng(seed)
    d = (0.01, 0.01, 0.01)
    k0 = GEO.k0_of(520.0)
    table = np.array([1.1, 2.4 - 0.05j, -6.0 - 0.4j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    return d, k0, table, mat, flags, x


@pytest.mark.parametrize("shape", [(30, 28, 20), (48, 40, 33)])
def test_tuned_operator_matches_oracle(shape):
    torch = pytest.importorskip("torch")
    d, k0, table, mat, flags, x = setup(shape)
    g = O.Grid(*shape, *d, k0)
    ref = O.matvec(g, O.green(g), table[mat], flags, x, False)
    with V.Context(*shape, *d, k0) as c:
        c.set_flags(flags)
        c.set_material(mat, table)
        c.green()
        rep = c.autotune(force=True)
        assert rep.startswith("fp64") and "fp32" in rep and "x=" in rep
        assert rel(c.matvec(x), ref) < 1e-12
        xt = torch.from_numpy(x.astype(np.complex64)).cuda()
        yt = torch.zeros_like(xt)
        torch.cuda.synchronize()
        c.matvec_dev(xt.data_ptr(), yt.data_ptr(), conj=False, precision=V.PREC_MIXED)
        c.sync()
        assert rel(yt.cpu().numpy(), ref) < 2e-5
        # a second context of the same grid takes the cached schedule
        with V.Context(*shape, *d, k0) as c2:
            c2.set_flags(flags)
            c2.set_material(mat, table)
            c2.green()
            assert "cached" in c2.autotune()
            assert rel(c2.matvec(x), ref) < 1e-12


def test_cache_file_is_read_by_a_new_process(tmp_path):
    path = str(tmp_path / "tune.txt")
    code = (
        "import numpy as np, vie_fft_b200 as V\n"
        "c = V.Context(24, 30, 18, 0.01, 0.01, 0.01, 10.0)\n"
        "c.set_flags(np.ones((3, 24, 30, 18), np.uint8))\n"
        "c.set_eps(np.full((24, 30, 18), 2.0 - 0.1j))\n"
        "print(c.autotune())\n"
    )
    env = dict(os.environ, VIE_TUNE_CACHE=path, PYTHONPATH=ROOT)
    r1 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r1.returncode == 0, r1.stderr
    assert "cached" not in r1.stdout and os.path.getsize(path) > 0
    r2 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r2.returncode == 0, r2.stderr
    assert r2.stdout.count("cached") == 2
