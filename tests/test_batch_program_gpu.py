"""The reference program's 41-wavelength run (CG_FFT_VIE.cpp: 32^3 sphere,
Dia = 60 nm, BiCGSTAB to CG_THR = 1e-3, synthetic material tables of
tests/golden/make_golden.py) done the batched way: one vie_solve_batch over
all wavelengths, FarField1 / FarField2 / NearField on the GPU, the result
files written by vie_fft_b200.results and merged as main.cpp does.  The files
must agree with the reference program's own (dropin_program.npz)."""
import os
import sys

import numpy as np
import pytest

import vie_fft_b200 as V
from vie_fft_b200 import geometry as GEO
from vie_fft_b200 import results as RF

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from make_golden import program_tables  # noqa: E402

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def test_batched_program(tmp_path):
    gold = np.load(os.path.join(ROOT, "tests", "golden", "dropin_program.npz"))
    tabs = program_tables()
    base = GEO.single_sphere(n=32, voxel_nm=2.0, diameter_nm=60.0, box_nm=60.0)
    ws, ctxs = [], []
    try:
        for m in range(41):
            lam = 400.0 + 10.0 * m
            t = [complex(*tabs[f][m]) for f in ("PEDOT_epr.txt", "Au_epr.txt", "P3HT_PCBM_epr.txt")]
            w = GEO.Workload("program", base.shape, base.d, GEO.k0_of(lam), base.material, base.flags,
                             np.array([1.1, t[0], t[1], t[2]]), cross_section=base.cross_section)
            c = V.Context(*w.shape, *w.d, w.k0)
            c.set_flags(w.flags)
            c.set_material(w.material, w.eps_table)
            c.green()
            c.incident(0.0, 0.0, 0.0, copy=False)
            ws.append(w)
            ctxs.append(c)
        res = V.solve_batch(ctxs, "bicgstab", tol=1e-3, copy=False)
        steps = np.array([r.info["steps"] for r in res])
        assert res[0].info["graph_loops"] == 1
        assert np.max(np.abs(steps - gold["steps"])) <= 1
        for m, (c, w) in enumerate(zip(ctxs, ws)):
            RF.write_from_context(str(tmp_path), m, c, w, planes=(m == 0))
        RF.merge_points(str(tmp_path), 41)
    finally:
        for c in ctxs:
            c.close()
    metal = np.loadtxt(tmp_path / "Ene_Metal.txt")
    grid = np.loadtxt(tmp_path / "Grid.txt")
    active = np.loadtxt(tmp_path / "Ene_Active.txt")
    np.testing.assert_array_equal(grid, gold["grid"])
    np.testing.assert_array_equal(metal[:, 0], gold["metal"][:, 0])
    assert np.isnan(active[:, 1]).all() and np.isnan(gold["active"][:, 1]).all()
    for m in range(41):
        tol = 1e-8 if steps[m] == gold["steps"][m] else 3e-3
        assert _rel(metal[m, 1:], gold["metal"][m, 1:]) < tol, m
        rcs = np.loadtxt(tmp_path / f"RCS{m}.txt")
        lin, glin = 10.0 ** (rcs / 10.0), 10.0 ** (gold["rcs"][m] / 10.0)
        assert _rel(lin, glin) < 10 * tol, m
    assert os.path.getsize(tmp_path / "LField0.txt") > 0
