"""Post-processing on the GPU against the reference's FarField1, FarField2
and NearField (golden fixture post_ops.npz, written by the reference built
here on seeded currents) and against the oracle on a solved field."""
import os

import numpy as np
import pytest

import vie_fft_b200 as V
from oracle import oracle as O
from tests.golden import make_golden as MG
from vie_fft_b200 import geometry as GEO

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
Z0 = 120 * np.pi


@pytest.mark.parametrize("idx", range(len(MG.SMALL)))
def test_post_matches_reference(idx):
    gold = np.load(os.path.join(GOLD, "post_ops.npz"))
    shape, d, k0, ang, mat, flags, x = MG.small_inputs(idx)
    with V.Context(*shape, *d, k0) as c:
        c.set_flags(flags)
        c.set_material(mat, MG.EPS_TABLE)
        c.set_solution(x)
        fwd = c.farfield1(*ang)
        scale = np.abs(x).sum() * np.prod(d) * Z0
        assert abs(fwd - gold[f"ff1_{idx}"]) < 1e-13 * scale
        rt, rp = c.farfield2(ang[1])
        np.testing.assert_allclose(rt, gold[f"rcs_theta{idx}"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(rp, gold[f"rcs_phi{idx}"], rtol=0, atol=1e-9)
        em, ea, av = c.nearfield(mat)
    ext, metal, active = gold[f"near{idx}"]
    assert abs(fwd / 0.37 - ext) < 1e-13 * scale / 0.37
    assert abs(em * Z0 / 0.37 - metal) < 1e-12 * abs(metal)
    if av > 0:
        assert abs(3 * ea / av - active) < 1e-12 * abs(active)
    else:
        assert np.isnan(active)


def test_post_of_solved_sphere_matches_oracle():
    w = GEO.single_sphere()
    g = O.Grid(*w.shape, *w.d, w.k0)
    with V.Context(*w.shape, *w.d, w.k0) as c:
        c.set_flags(w.flags)
        c.set_material(w.material, w.eps_table)
        c.green()
        c.incident(w.theta, w.phi, w.psi, copy=False)
        x = c.solve("bicgstab", tol=1e-8).x
        fwd = c.farfield1(w.theta, w.phi, w.psi)
        em, ea, av = c.nearfield(w.material)
    assert abs(fwd - O.farfield1(g, x, w.theta, w.phi, w.psi)) < 1e-12 * abs(fwd)
    em_o, ea_o, av_o = O.absorption(g, x, w.eps, w.material)
    assert abs(em - em_o) < 1e-12 * abs(em_o) and av == av_o == 0.0


def test_post_state_errors():
    with V.Context(8, 8, 8, 0.01, 0.01, 0.01, 10.0) as c:
        with pytest.raises(V.VieError) as e:
            c.farfield1()
        assert e.value.status == V.VIE_ERR_STATE
