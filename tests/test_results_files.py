"""Result files in the reference's formats (vie_fft_b200/results.py): every
number formatted exactly as C's printf("%.15lf") formats it (checked against
the C library here), the file layout of NearFar.h and the merge of main.cpp."""
import ctypes
import math
import os

import numpy as np

from vie_fft_b200 import results as RF

libc = ctypes.CDLL(None)


def c_fmt(v):
    buf = ctypes.create_string_buffer(512)
    libc.snprintf(buf, 512, b"%.15lf", ctypes.c_double(v))
    return buf.value.decode()


def test_number_format_matches_c():
    rng = np.random.default_rng(0)
    vals = list(rng.standard_normal(200) * 10.0 ** rng.integers(-12, 12, 200))
    vals += [0.0, -0.0, 1e-16, -2.5e-300, 123456789.123456789, -59.63328705123, math.inf, -math.inf]
    for v in vals:
        assert RF._f(v) == c_fmt(v), v
    # the NaN of 0/0 (empty active volume), computed by the C library
    nan00 = RF._ratio(0.0, 0.0)
    with np.errstate(invalid="ignore"):
        c_nan = float(np.float64(-np.inf) * 0.0)
    assert RF._f(nan00) == "-nan" == c_fmt(c_nan)


def test_point_files_and_merge(tmp_path):
    rng = np.random.default_rng(1)
    shape, d = (6, 5, 4), (0.0125, 0.0125, 0.0125)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    rt, rp = rng.standard_normal(181), rng.standard_normal(181)
    for m in range(3):
        RF.write_point(str(tmp_path), m, shape, d, x, 0.5 + m, 0.37, 1e-3 * m, 0.0, 0.0, rt, rp)
    lines = open(tmp_path / "Ene_Metal1.txt").read().splitlines()
    assert lines == [f"410 {c_fmt(1.5 / 0.37)} {c_fmt(1e-3 * RF.Z0 / 0.37)}"]
    assert open(tmp_path / "Ene_Active2.txt").read() == "420 -nan\n"
    assert open(tmp_path / "Grid0.txt").read() == f"0 6 5 4 {c_fmt(0.0125)} {c_fmt(0.0125)} {c_fmt(0.0125)}\n"
    rcs = np.loadtxt(tmp_path / "RCS0.txt")
    assert rcs.shape == (181, 2) and np.allclose(rcs[:, 0], rt, atol=1e-14)
    # plane dumps: k = Nz/2 of the core, C loop order (i, j)
    lf = np.loadtxt(tmp_path / "LField0.txt")
    core = x[:, :5, :4, 2]
    assert lf.shape == (20, 6) and np.allclose(lf[:, 0], core[0].real.ravel(), atol=1e-14)
    assert np.allclose(lf[:, 5], core[2].imag.ravel(), atol=1e-14)
    vf = np.loadtxt(tmp_path / "VField0.txt")
    assert vf.shape == (12, 6) and np.allclose(vf[:, 2], x[1, 3, :4, :3].real.ravel(), atol=1e-14)
    RF.merge_points(str(tmp_path), 3)
    merged = open(tmp_path / "Ene_Metal.txt").read().splitlines()
    assert [l.split()[0] for l in merged] == ["400", "410", "420"]
    assert not os.path.exists(tmp_path / "Ene_Metal0.txt") and os.path.exists(tmp_path / "RCS0.txt")
    g = np.loadtxt(tmp_path / "Grid.txt")
    assert g.shape == (3, 7) and list(g[:, 0]) == [0, 1, 2]
