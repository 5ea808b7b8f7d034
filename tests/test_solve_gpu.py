"""CUDA Krylov drivers against the reference.

BiCGSTAB and BiCORSTAB amplify rounding differences on metallic scatterers:
the reference itself, fed a right-hand side perturbed by 2e-16 relative,
changes its converged step count by several steps and its field by ~1e-6
at tolerance 1e-6 (test_oracle_sensitivity.py measures this with the
oracle).  Their parity is therefore asserted on fields converged to a tight
tolerance (relative field difference <= 1e-10), and their step counts at
the configured tolerance within that measured envelope.  CORS, BiCG and CG
do not amplify rounding on these cases: steps within +-1 and fields within
1e-10 at the configured tolerance.
"""
import os

import numpy as np
import pytest

import vie_fft_b200 as V
from oracle import oracle as O
from tests.golden import make_golden as MG
from vie_fft_b200 import geometry as GEO

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIELD_TOL = 1e-10


def relnorm(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def ctx_for(w):
    c = V.Context(*w.shape, *w.d, w.k0)
    c.set_flags(w.flags)
    if w.eps_voxel is not None:
        c.set_eps(w.eps_voxel)
    else:
        c.set_material(w.material, w.eps_table)
    c.green()
    c.incident(w.theta, w.phi, w.psi, copy=False)
    return c


@pytest.mark.parametrize("solver", ["cors", "bicg", "cg"])
def test_stable_solvers_match_reference(solver):
    gold = np.load(os.path.join(GOLD, "small_solves.npz"))
    w = MG.solve_case()
    with ctx_for(w) as c:
        r = c.solve(solver, tol=float(gold[f"{solver}_thr"]))
    assert abs(r.info["steps"] - int(gold[f"{solver}_steps"])) <= 1
    # CG stops on the unrooted ||r||^2/||b||^2 (CG_Iteration.h:323), so at 1e-12
    # its field is converged only to a 1e-6 residual; the reference's own spread
    # under 2e-16 perturbations is up to 1.3e-9 there.
    tol = 5e-9 if solver == "cg" else FIELD_TOL
    assert relnorm(r.x, gold[f"{solver}_x"]) < tol


def test_cg_fields_at_tight_tolerance():
    w = MG.solve_case()
    g = O.Grid(*w.shape, *w.d, w.k0)
    xo, so, _ = O.solve(g, O.green(g), w.eps, w.flags, O.incident(g, w.theta, w.phi, w.psi), "cg", 1e-22)
    with ctx_for(w) as c:
        r = c.solve("cg", tol=1e-22)
    assert abs(r.info["steps"] - so) <= 1
    assert relnorm(r.x, xo) < FIELD_TOL


@pytest.mark.parametrize("solver", ["bicgstab", "bicorstab"])
def test_sensitive_solvers_fields_at_tight_tolerance(solver):
    w = MG.solve_case()
    g = O.Grid(*w.shape, *w.d, w.k0)
    xo, so, _ = O.solve(g, O.green(g), w.eps, w.flags, O.incident(g, w.theta, w.phi, w.psi), solver, 1e-12)
    with ctx_for(w) as c:
        r = c.solve(solver, tol=1e-12)
    assert relnorm(r.x, xo) < FIELD_TOL
    assert r.info["true_relres"] < 1e-11


@pytest.mark.parametrize("solver", ["bicgstab", "bicorstab"])
def test_sensitive_solvers_steps_within_reference_envelope(solver):
    gold = np.load(os.path.join(GOLD, "small_solves.npz"))
    w = MG.solve_case()
    with ctx_for(w) as c:
        r = c.solve(solver, tol=float(gold[f"{solver}_thr"]))
    # the reference's own spread under 2e-16 perturbations is up to 8 steps here
    assert abs(r.info["steps"] - int(gold[f"{solver}_steps"])) <= 10
    assert relnorm(r.x, gold[f"{solver}_x"]) < 1e-6
    assert r.info["true_relres"] < 2e-8


def test_c1_silver_sphere_against_reference():
    """32^3 silver sphere, BiCGSTAB to 1e-6 (the reference's CPU case)."""
    gold = np.load(os.path.join(GOLD, "c1_sphere.npz"))
    w = GEO.single_sphere()
    g = O.Grid(*w.shape, *w.d, w.k0)
    with ctx_for(w) as c:
        r = c.solve("bicgstab", tol=1e-6)
    assert abs(r.info["steps"] - int(gold["steps"])) <= 6
    xs = r.x[w.flags.astype(bool)]
    assert relnorm(xs, gold["x_flagged"]) < 1e-5
    fwd = O.farfield1(g, r.x)
    assert abs(fwd - float(gold["forward_rcs"])) < 1e-5 * abs(fwd)
    metal, _, _ = O.absorption(g, r.x, w.eps, w.material)
    q_abs = metal * GEO.Z0 / w.cross_section
    assert abs(q_abs - float(gold["metal_abs_over_cs"])) < 1e-5 * abs(q_abs)


def test_c1_fields_at_tight_tolerance():
    w = GEO.single_sphere()
    g = O.Grid(*w.shape, *w.d, w.k0)
    xo, so, _ = O.solve(g, O.green(g), w.eps, w.flags, O.incident(g), "bicgstab", 1e-10)
    with ctx_for(w) as c:
        r = c.solve("bicgstab", tol=1e-10)
    assert relnorm(r.x, xo) < 1e-9


def test_mixed_precision_matches_fp64():
    w = GEO.single_sphere()
    g = O.Grid(*w.shape, *w.d, w.k0)
    with ctx_for(w) as c:
        r64 = c.solve("bicgstab", tol=1e-10)
        rmx = c.solve("bicgstab", tol=1e-8, precision=V.PREC_MIXED)
    assert rmx.info["true_relres"] < 1e-8
    assert rmx.info["matvecs_fp32"] > 0 and rmx.info["outer"] >= 1
    assert relnorm(rmx.x, r64.x) < 1e-6
    q64 = O.absorption(g, r64.x, w.eps, w.material)[0]
    qmx = O.absorption(g, rmx.x, w.eps, w.material)[0]
    assert abs(qmx - q64) < 1e-6 * abs(q64)
    e64, emx = O.farfield1(g, r64.x), O.farfield1(g, rmx.x)
    assert abs(emx - e64) < 1e-6 * abs(e64)


def test_iteration_cap_and_errors():
    w = MG.solve_case()
    with ctx_for(w) as c:
        r = c.solve("bicgstab", tol=1e-14, max_iter=3, allow_maxit=True)
        assert r.status == V.VIE_ERR_MAXIT and r.info["iterations"] == 3
        with pytest.raises(V.VieError) as e:
            c.solve("bicgstab", tol=-1.0)
        assert e.value.status == V.VIE_ERR_ARG
        c.set_rhs(np.zeros((3,) + w.shape))
        with pytest.raises(V.VieError) as e:
            c.solve("bicgstab", tol=1e-6)
        assert e.value.status == V.VIE_ERR_ARG
    with V.Context(*w.shape, *w.d, w.k0) as c:
        c.set_flags(w.flags)
        c.set_material(w.material, w.eps_table)
        with pytest.raises(V.VieError) as e:
            c.solve("bicgstab", tol=1e-6)
        assert e.value.status == V.VIE_ERR_STATE


@pytest.mark.parametrize("solver,precision", [("bicgstab", V.PREC_FP64), ("cors", V.PREC_FP64), ("cg", V.PREC_FP64),
                                              ("bicg", V.PREC_FP64), ("bicorstab", V.PREC_FP64),
                                              ("bicgstab", V.PREC_MIXED), ("cors", V.PREC_MIXED)])
def test_graph_loop_matches_host_loop(solver, precision, monkeypatch):
    """The iteration captured once and looped on the device (conditional WHILE
    node, reliable updates under an IF node) computes exactly what the same
    kernels launched from a host loop compute."""
    w = MG.solve_case()
    tol = 1e-8
    with ctx_for(w) as c:
        rg = c.solve(solver, tol=tol, precision=precision)
    monkeypatch.setenv("VIE_GRAPH", "0")
    with ctx_for(w) as c:
        rh = c.solve(solver, tol=tol, precision=precision)
    assert rg.info["graph_loops"] >= 1 and rh.info["graph_loops"] == 0
    if precision == V.PREC_FP64 or solver == "bicgstab":
        assert rg.info["graph_loops"] == 1
    for k in ("steps", "iterations", "outer", "matvecs_fp32", "matvecs_fp64"):
        assert rg.info[k] == rh.info[k], k
    np.testing.assert_array_equal(rg.x, rh.x)


@pytest.mark.parametrize("precision", [V.PREC_FP64, V.PREC_MIXED])
def test_staged_z_prologues_match_element_loads(precision, monkeypatch):
    """BiCGSTAB with the forward z pass reading its prologue vectors (r, v)
    from rows staged by bulk copies gives the same iterates, bit for bit, as
    with element loads."""
    # 16^3: every axis on the register kernels
    w = GEO.single_sphere(n=16, voxel_nm=2.0, diameter_nm=24.0, eps_physics=-4.0 + 0.3j, wavelength_nm=500.0,
                          theta=20.0, phi=30.0, psi=40.0)
    with ctx_for(w) as c:
        rs = c.solve("bicgstab", tol=1e-8, precision=precision)
    monkeypatch.setenv("VIE_ZSTAGE", "0")
    with ctx_for(w) as c:
        re_ = c.solve("bicgstab", tol=1e-8, precision=precision)
    for k in ("steps", "iterations", "outer", "matvecs_fp32", "matvecs_fp64"):
        assert rs.info[k] == re_.info[k], k
    np.testing.assert_array_equal(rs.x, re_.x)
