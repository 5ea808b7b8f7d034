"""Adjoint gradient of the absorbed power (vie_power_grad) and its
torch.autograd binding.

Objective: NearField's Ene_Active sum (NearFar.h:186-250) over the edges
whose two voxels are in the active layer.  Checked against
* the numpy restatement of the reference's formula on the forward field,
* FP64 central finite differences of P in Re and Im of eps at seeded voxels,
* the all-FP64 adjoint (for the mixed-precision adjoint),
* the operator's complex symmetry x^T A y = y^T A x that the adjoint relies on.
"""
import numpy as np
import pytest

import vie_fft_b200 as V
from vie_fft_b200 import geometry as GEO
from vie_fft_b200 import post

pytestmark = pytest.mark.gpu


def small_design(wavelength_nm=550.0):
    return GEO.design_stack(shape=(24, 24, 16), spacer_nm=4.0, active_top_nm=14.0,
                            region_nm=((6, 18), (6, 18), (5, 12)), wavelength_nm=wavelength_nm, seed=5)


def ctx_for(w):
    c = V.Context(*w.shape, *w.d, w.k0)
    c.set_flags(w.flags)
    c.set_eps(w.eps_voxel)
    c.green()
    c.incident(w.theta, w.phi, w.psi, copy=False)
    return c


def test_power_matches_reference_formula():
    w = small_design()
    mask = post.edge_mask(w.material, 3)
    with ctx_for(w) as c:
        p, _, fi, _ = c.power_grad(mask, tol=1e-12, grad=False)
        x = c.solution()
    _, ea, _ = post.absorption(w.shape, w.d, w.k0, x, w.eps, w.material)
    assert p > 0 and abs(p - ea) < 1e-12 * abs(ea)
    assert fi["steps"] >= 0


def test_operator_is_complex_symmetric():
    w = small_design()
    rng = np.random.default_rng(1)
    x = (rng.standard_normal((3,) + w.shape) + 1j * rng.standard_normal((3,) + w.shape)) * w.flags
    y = (rng.standard_normal((3,) + w.shape) + 1j * rng.standard_normal((3,) + w.shape)) * w.flags
    with ctx_for(w) as c:
        ax, ay = c.matvec(x), c.matvec(y)
    lhs, rhs = np.sum(x * ay), np.sum(y * ax)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


@pytest.mark.parametrize("wavelength_nm", [450.0, 650.0])
def test_gradient_matches_central_differences(wavelength_nm):
    w = small_design(wavelength_nm)
    mask = post.edge_mask(w.material, 3)
    region = np.argwhere(w.meta["region"])
    rng = np.random.default_rng(6)
    picks = [tuple(region[i]) for i in rng.choice(len(region), 6, replace=False)]
    h = 1e-5
    with ctx_for(w) as c:
        p0, g, fi, ai = c.power_grad(mask, tol=1e-13)
        assert ai["steps"] >= 0
        scale = np.abs(g[w.meta["region"]]).max()
        for v in picks:
            fd = []
            for dz in (h, 1j * h):
                vals = []
                for sgn in (1.0, -1.0):
                    eps = w.eps_voxel.copy()
                    eps[v] += sgn * dz
                    c.set_eps(eps)
                    vals.append(c.power_grad(mask, tol=1e-13, grad=False)[0])
                fd.append((vals[0] - vals[1]) / (2 * h))
            c.set_eps(w.eps_voxel)
            fdg = fd[0] + 1j * fd[1]
            assert abs(g[v] - fdg) < 1e-5 * scale, (v, g[v], fdg)


def test_mixed_adjoint_matches_fp64_adjoint():
    w = small_design()
    mask = post.edge_mask(w.material, 3)
    with ctx_for(w) as c:
        p64, g64, _, _ = c.power_grad(mask, tol=1e-10, precision=V.PREC_FP64)
        pmx, gmx, fi, ai = c.power_grad(mask, tol=1e-10, precision=V.PREC_MIXED)
    assert fi["matvecs_fp32"] > 0 and ai["matvecs_fp32"] > 0
    assert abs(pmx - p64) < 1e-8 * abs(p64)
    assert np.abs(gmx - g64).max() < 1e-7 * np.abs(g64).max()


def test_autograd_binding():
    torch = pytest.importorskip("torch")
    from vie_fft_b200.autograd import absorbed_power
    ws = [small_design(lam) for lam in (450.0, 550.0, 650.0)]
    mask = post.edge_mask(ws[0].material, 3)
    ctxs = [ctx_for(w) for w in ws]
    try:
        eps_phys = torch.tensor(np.conj(ws[0].eps_voxel), dtype=torch.complex128, requires_grad=True)
        total = sum(absorbed_power(eps_phys.conj(), c, mask, tol=1e-12) for c in ctxs)
        total.backward()
        ref_total, ref_grad = 0.0, 0.0
        for c in ctxs:
            p, g, _, _ = c.power_grad(mask, tol=1e-12)
            ref_total += p
            ref_grad = ref_grad + g
        assert abs(total.item() - ref_total) < 1e-12 * abs(ref_total)
        # d/d eps_phys = conj of the gradient in the reference convention
        got = eps_phys.grad.numpy()
        assert np.abs(got - np.conj(ref_grad)).max() < 1e-10 * np.abs(ref_grad).max()
    finally:
        for c in ctxs:
            c.close()


def test_power_grad_errors():
    w = small_design()
    with V.Context(*w.shape, 0.01, 0.01, 0.012, w.k0) as c:
        c.set_flags(w.flags)
        c.set_eps(w.eps_voxel)
        c.green()
        c.incident(0.0, 0.0, 0.0, copy=False)
        with pytest.raises(V.VieError) as e:
            c.power_grad(post.edge_mask(w.material, 3))
        assert e.value.status == V.VIE_ERR_ARG
