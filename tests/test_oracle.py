"""The oracle (CPU restatement of the reference hot path) pinned against the
reference's own code: golden fixtures generated from oracle/_ref by
tests/golden/make_golden.py, and the live reference build where present."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import pruned_model
from tests.golden import make_golden as MG

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("shape", [(64, 64, 64), (62, 6, 22), (2, 3, 5), (26, 14, 34), (7, 11, 13), (1, 1, 8),
                                   (96, 48, 10), (31, 37, 2)])
def test_fft_matches_numpy(shape):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert rel(O.fft3d(x, -1), np.fft.fftn(x)) < 2e-15
    assert rel(O.fft3d(x, +1), np.fft.ifftn(x) * x.size) < 2e-15


@pytest.mark.parametrize("idx", range(len(MG.SMALL)))
def test_restatement_matches_reference_ops(idx):
    gold = np.load(os.path.join(GOLD, "small_ops.npz"))
    shape, d, k0, ang, mat, flags, x = MG.small_inputs(idx)
    g = O.Grid(*shape, *d, k0)
    G = O.green(g)
    assert rel(G, gold[f"green{idx}"]) < 1e-14
    assert rel(O.incident(g, *ang), gold[f"inc{idx}"]) < 1e-14
    eps = MG.EPS_TABLE[mat]
    assert rel(O.matvec(g, G, eps, flags, x, False), gold[f"ax{idx}"]) < 1e-13
    assert rel(O.matvec(g, G, eps, flags, x, True), gold[f"ahx{idx}"]) < 1e-13


@pytest.mark.parametrize("solver", ["bicgstab", "cors", "bicorstab", "bicg", "cg"])
def test_restatement_matches_reference_solvers(solver):
    gold = np.load(os.path.join(GOLD, "small_solves.npz"))
    w = MG.solve_case()
    g = O.Grid(*w.shape, *w.d, w.k0)
    G = O.green(g)
    e = O.incident(g, w.theta, w.phi, w.psi)
    x, steps, err = O.solve(g, G, w.eps, w.flags, e, solver, float(gold[f"{solver}_thr"]))
    assert steps == int(gold[f"{solver}_steps"])
    xr = gold[f"{solver}_x"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-12


def test_restatement_c1_sphere_matches_reference():
    from vie_fft_b200 import geometry as GEO
    gold = np.load(os.path.join(GOLD, "c1_sphere.npz"))
    w = GEO.single_sphere()
    g = O.Grid(*w.shape, *w.d, w.k0)
    G = O.green(g)
    e = O.incident(g)
    x, steps, err = O.solve(g, G, w.eps, w.flags, e, "bicgstab", 1e-6)
    assert steps == int(gold["steps"])
    xr = gold["x_flagged"]
    xs = x[w.flags.astype(bool)]
    assert np.linalg.norm(xs - xr) / np.linalg.norm(xr) < 1e-12
    # the solution vanishes off the flagged edges
    assert np.abs(x[~w.flags.astype(bool)]).max() == 0.0
    fwd = O.farfield1(g, x)
    assert abs(fwd - float(gold["forward_rcs"])) < 1e-12 * abs(fwd)
    metal, _, _ = O.absorption(g, x, w.eps, w.material)
    assert abs(metal * GEO.Z0 / w.cross_section - float(gold["metal_abs_over_cs"])) < 1e-10


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref not present")
def test_restatement_matches_live_reference_random():
    rng = np.random.default_rng(7)
    shape = (9, 5, 7)
    g = O.Grid(*shape, 0.012, 0.013, 0.0125, 2 * np.pi / 5.5)
    table = np.array([1.1, 3.0 - 0.2j, -6.0 - 0.4j, 2.2 - 0.1j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    R = O.Reference(g, table, 15.0, 25.0, 35.0)
    R.set_geometry(mat, flags)
    Gr = R.green()
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    yr = R.matvec(x, False)
    R.release()
    assert rel(O.green(g), Gr) < 1e-14
    assert rel(O.matvec(g, Gr, table[mat], flags, x, False), yr) < 1e-13


@pytest.mark.parametrize("shape,d", [((4, 6, 5), (0.0125, 0.0125, 0.0125)), ((6, 8, 3), (0.0125, 0.011, 0.014)),
                                     ((8, 4, 12), (0.01, 0.01, 0.01)), ((5, 7, 9), (0.0125, 0.011, 0.014))])
def test_pruned_schedule_model_matches_oracle(shape, d):
    """The five-pass pruned schedule the CUDA kernels implement (split padded
    axes, digit-reversed spectra, charge-form symbol, folded octant) equals
    the reference's nine padded FFT pairs."""
    rng = np.random.default_rng(3)
    g = O.Grid(*shape, *d, 2 * np.pi / 4.0)
    table = np.array([1.1, 2.0 - 0.1j, -4.42 - 0.21j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    G = O.green(g)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    for conj in (0, 1):
        yo = O.matvec(g, G, table[mat], flags, x, conj)
        ye = pruned_model.emulate(g, G, table[mat], flags, x, conj)
        assert rel(ye, yo) < 1e-14
