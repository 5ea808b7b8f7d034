"""Host-side workload set-up: the reference's material / flag rule."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from vie_fft_b200 import geometry as G

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref not present")
@pytest.mark.parametrize("n,vox,dia", [(32, 1.25, 36.0), (31, 2.0, 60.0), (20, 2.0, 34.0)])
def test_single_sphere_equals_reference_getmaterial_getflag(n, vox, dia):
    w = G.single_sphere(n=n, voxel_nm=vox, diameter_nm=dia)
    R = O.Reference(O.Grid(*w.shape, *w.d, w.k0), w.eps_table)
    R.sphere_geometry(w.meta["diameter"], w.meta["box"], w.meta["box"], w.meta["box"])
    m, f = R.get_geometry()
    R.release()
    assert (m == w.material).all()
    assert (f == w.flags).all()


def test_c1_flags_match_golden_solution_support():
    gold = np.load(os.path.join(GOLD, "c1_sphere.npz"))
    w = G.single_sphere()
    assert int(w.flags.sum()) == gold["x_flagged"].size


def test_cluster_spheres_do_not_overlap():
    w = G.sphere_cluster(n=48, count=8, rmin_nm=3.0, rmax_nm=6.0, seed=2)
    cs, rs = w.meta["centres"], w.meta["radii"]
    for i in range(len(rs)):
        for j in range(i):
            assert np.linalg.norm(cs[i] - cs[j]) >= rs[i] + rs[j]
    assert (w.material == 2).sum() > 0


def test_reference_sign_convention_and_drude():
    e = G.drude_silver(550.0)
    assert e.imag > 0 and e.real < 0            # physics convention: lossy metal
    assert G.to_reference_eps(e).imag < 0       # reference convention (data/Au_epr.txt)


def test_solar_cell_layers_and_box_edges():
    w = G.solar_cell(shape=(32, 32, 24), nspheres=2, radius_nm=3.0, spacer_nm=5.0, active_nm=12.0,
                     sphere_z_nm=(8.0, 12.0))
    labels = set(np.unique(w.material).tolist())
    assert labels == {0, 1, 2, 3}
    # the layers stop at the box: no x unknown on the last x plane, no y unknown on the last y plane
    assert w.flags[0][-1].sum() == 0 and w.flags[1][:, -1].sum() == 0
