"""Batched solves (vie_solve_batch): several contexts with different grids,
wavelengths, polarisations and materials solved in one CUDA graph launch.
Every instance must come out bit-identical to its own single solve (the
batch runs each instance's kernels in the same order; only the loop is
shared), with the instance's own step count."""
import numpy as np
import pytest

import vie_fft_b200 as V
from vie_fft_b200 import geometry as GEO

pytestmark = pytest.mark.gpu


def ctx_for(w):
    c = V.Context(*w.shape, *w.d, w.k0)
    c.set_flags(w.flags)
    c.set_material(w.material, w.eps_table)
    c.green()
    c.incident(w.theta, w.phi, w.psi, copy=False)
    return c


def instances():
    sweep = GEO.batch_sweep(shape=(24, 20, 12), n_wavelengths=3, spacer_nm=3.0, active_nm=6.0, nspheres=1,
                            radius_nm=3.0, sphere_z_nm=(6.0, 6.0))
    spheres = GEO.batch_spheres(count=4, edges=(8, 12, 16), seed=7)
    return sweep + spheres


@pytest.mark.parametrize("solver,precision", [("bicgstab", V.PREC_FP64), ("cors", V.PREC_FP64),
                                              ("bicgstab", V.PREC_MIXED)])
def test_batch_matches_single_solves(solver, precision):
    ws = instances()
    ctxs = [ctx_for(w) for w in ws]
    try:
        rb = V.solve_batch(ctxs, solver, tol=1e-8, precision=precision, raise_errors=False)
        assert len(rb) == len(ws)
        for c, r in zip(ctxs, rb):
            assert r.info["graph_loops"] == 1
            # the same instance alone: same status (a driver's breakdown on an
            # instance is that instance's own), same counts, same bits
            try:
                rs = c.solve(solver, tol=1e-8, precision=precision)
                status, info, x = rs.status, rs.info, rs.x
            except V.VieError as e:
                status, info, x = e.status, None, c.solution()
            assert r.status == status
            if info is not None:
                for k in ("steps", "iterations", "outer", "matvecs_fp32", "matvecs_fp64"):
                    assert r.info[k] == info[k], k
            np.testing.assert_array_equal(r.x, x)
        ok = [r for r in rb if r.status == V.VIE_OK]
        assert len(ok) >= len(rb) - 2
        # the instances converge at different steps: the loop masked the early ones
        assert len({r.info["steps"] for r in ok}) > 1
    finally:
        for c in ctxs:
            c.close()


def test_batch_host_loop_and_errors(monkeypatch):
    ws = instances()[:3]
    monkeypatch.setenv("VIE_GRAPH", "0")
    ctxs = [ctx_for(w) for w in ws]
    try:
        rb = V.solve_batch(ctxs, "bicgstab", tol=1e-8)
        for c, r in zip(ctxs, rb):
            assert r.info["graph_loops"] == 0
            np.testing.assert_array_equal(r.x, c.solve("bicgstab", tol=1e-8).x)
        with pytest.raises(V.VieError) as e:
            V.solve_batch([ctxs[0], ctxs[0]], "bicgstab", tol=1e-8)
        assert e.value.status == V.VIE_ERR_ARG
        with pytest.raises(V.VieError) as e:
            V.solve_batch(ctxs, "cors", tol=1e-8, precision=V.PREC_MIXED)
        assert e.value.status == V.VIE_ERR_ARG
        r = V.solve_batch(ctxs, "bicgstab", tol=1e-14, max_iter=2, allow_maxit=True)
        assert all(x.info["iterations"] == 2 for x in r) and r[0].status == V.VIE_ERR_MAXIT
    finally:
        for c in ctxs:
            c.close()


def register_instances():
    """Instances whose three axes all run on the register kernels, the batches
    the persistent multi-instance loop takes: a wavelength sweep on one 24x32x16
    stack (one size class) and spheres of edges 16 and 24 (two more)."""
    sweep = GEO.batch_sweep(shape=(24, 32, 16), n_wavelengths=3, spacer_nm=3.0, active_nm=8.0, nspheres=1,
                            radius_nm=3.0, sphere_z_nm=(6.0, 6.0))
    spheres = GEO.batch_spheres(count=5, edges=(16, 24), seed=7)
    return sweep + spheres


def test_persistent_batch_matches_single_solves(monkeypatch):
    """Mixed BiCGSTAB over size classes as persistent kernels per pass
    (VIE_BATCH_FUSED=1): every instance bit-identical to its single solve and
    to the per-instance graph branches (the default), with a fixed number of
    kernels per size class and pass."""
    ws = register_instances()
    ctxs = [ctx_for(w) for w in ws]
    try:
        monkeypatch.setenv("VIE_BATCH_FUSED", "1")
        n0 = V.launch_count()
        rb = V.solve_batch(ctxs, "bicgstab", tol=1e-8, precision=V.PREC_MIXED, raise_errors=False)
        fused = V.launch_count() - n0
        monkeypatch.delenv("VIE_BATCH_FUSED")
        n0 = V.launch_count()
        rb0 = V.solve_batch(ctxs, "bicgstab", tol=1e-8, precision=V.PREC_MIXED, raise_errors=False)
        branches = V.launch_count() - n0
        for c, r, r0 in zip(ctxs, rb, rb0):
            assert r.info["graph_loops"] == 1
            rs = c.solve("bicgstab", tol=1e-8, precision=V.PREC_MIXED)
            assert r.status == rs.status == r0.status
            for k in ("steps", "iterations", "outer", "matvecs_fp32", "matvecs_fp64"):
                assert r.info[k] == rs.info[k] == r0.info[k], k
            np.testing.assert_array_equal(r.x, rs.x)
            np.testing.assert_array_equal(r0.x, rs.x)
        assert len({r.info["steps"] for r in rb}) > 1
        # per pass a fixed set of kernels per size class (3 classes here), whatever
        # the number of instances in it; the branches launch per instance
        passes = max(r.info["iterations"] for r in rb) + 1
        assert fused <= 30 * 3 * passes < branches, (fused, passes, branches)
    finally:
        for c in ctxs:
            c.close()
