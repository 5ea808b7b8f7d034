"""Config C5 at full size: the adjoint gradient of the absorbed power in the
P3HT:PCBM layer (NearField's Ene_Active sum, NearFar.h:186-250) over the
64x64x32 design region of the 128x128x64 solar-cell stack, at 550 nm.

* FP64 central differences with the configured step h = 1e-6 in Re and Im of
  eps at 32 seeded design voxels (seed 6), each difference from two FP64
  solves to relative residual 1e-13.  At this step the difference quotient
  carries the solves' error in P divided by h: with eta the error of P in one
  solve, |FD_v - g_v| <= eta / h + O(h^2).  eta is measured here as the
  change of P between solves to 1e-12 and 1e-13 (an upper estimate of the
  1e-13 solve's error), and every voxel's error must lie under that bound.
  The errors relative to |g_v| are printed per voxel.
* the mixed-precision adjoint against the all-FP64 GPU adjoint.
"""
import numpy as np
import pytest

import vie_fft_b200 as V
from vie_fft_b200 import geometry as GEO
from vie_fft_b200 import post

pytestmark = pytest.mark.gpu
H = 1e-6
FD_TOL = 1e-13


@pytest.fixture(scope="module")
def c5():
    w = GEO.design_stack(wavelength_nm=550.0)
    c = V.Context(*w.shape, *w.d, w.k0)
    c.set_flags(w.flags)
    c.set_eps(w.eps_voxel)
    c.green()
    c.incident(w.theta, w.phi, w.psi, copy=False)
    yield w, c, post.edge_mask(w.material, 3)
    c.close()


def test_c5_gradient_against_central_differences(c5):
    w, c, mask = c5
    p0, g, _, _ = c.power_grad(mask, tol=FD_TOL, max_iter=5000)
    p12 = c.power_grad(mask, tol=1e-12, grad=False, max_iter=5000)[0]
    eta = max(abs(p12 - p0), 1e-16 * abs(p0))
    region = np.argwhere(w.meta["region"])
    rng = np.random.default_rng(6)
    picks = [tuple(region[i]) for i in rng.choice(len(region), 32, replace=False)]
    rows = []
    for v in picks:
        fd = []
        for dz in (H, 1j * H):
            vals = []
            for sgn in (1.0, -1.0):
                eps = w.eps_voxel.copy()
                eps[v] += sgn * dz
                c.set_eps(eps)
                vals.append(c.power_grad(mask, tol=FD_TOL, grad=False, max_iter=5000)[0])
            fd.append((vals[0] - vals[1]) / (2 * H))
        fdg = fd[0] + 1j * fd[1]
        rows.append((v, g[v], fdg, abs(fdg - g[v])))
    c.set_eps(w.eps_voxel)
    bound = eta / H
    print(f"\nP = {p0:.15e}, eta = {eta:.3e}, bound eta/h = {bound:.3e}, max|g| = {np.abs(g).max():.3e}")
    for v, gv, fdg, err in rows:
        print(f"voxel {v}: |g| {abs(gv):.3e}  |FD - g| {err:.3e}  rel {err / abs(gv):.2e}")
    for v, gv, fdg, err in rows:
        assert err <= 2.0 * bound + 1e-6 * abs(gv), (v, gv, fdg, err, bound)


def test_c5_mixed_adjoint_against_fp64_adjoint(c5):
    w, c, mask = c5
    p64, g64, _, _ = c.power_grad(mask, tol=1e-8, precision=V.PREC_FP64)
    pmx, gmx, fi, ai = c.power_grad(mask, tol=1e-8, precision=V.PREC_MIXED)
    assert fi["matvecs_fp32"] > 0 and ai["matvecs_fp32"] > 0
    assert abs(pmx - p64) < 1e-6 * abs(p64)
    assert np.abs(gmx - g64).max() < 1e-5 * np.abs(g64).max()
