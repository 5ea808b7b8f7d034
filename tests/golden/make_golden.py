"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

Runs the reference's vie_fft functions (compiled in place by oracle/Makefile
into oracle/_ref/libvieref.so against the MKL shim) on seeded inputs and
stores their outputs as .npz files.  It needs the reference checkout, so it
runs in the development container only; the fixtures it writes travel with
the repository.

    python tests/golden/make_golden.py

Fixtures
  small_ops.npz      Green spectrum, incident field, A x and A^H x on small
                     seeded grids (non-cubic, odd and prime axis lengths)
  small_solves.npz   all five Krylov drivers on one small seeded problem
  c1_sphere.npz      the 32^3 silver-sphere BiCGSTAB solve to 1e-6: step
                     count, solution on the flagged edges, FarField1 and
                     NearField outputs
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from vie_fft_b200 import geometry as G  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# small cases: (shape, d, wavelength nm, angles)
SMALL = [
    ((4, 6, 5), (0.0125, 0.0125, 0.0125), 400.0, (0.0, 0.0, 0.0)),
    ((7, 3, 11), (0.0125, 0.011, 0.014), 450.0, (10.0, 20.0, 30.0)),
    ((8, 8, 8), (0.01, 0.01, 0.01), 550.0, (0.0, 0.0, 90.0)),
    ((6, 10, 12), (0.01, 0.01, 0.01), 700.0, (35.0, 50.0, 15.0)),
]
EPS_TABLE = np.array([1.1, 2.4 - 0.05j, -4.42 - 0.21j, 3.8 - 0.6j])


def small_inputs(idx):
    """Seeded inputs of small case idx (re-created identically by the tests)."""
    shape, d, lam, ang = SMALL[idx]
    rng = np.random.default_rng(100 + idx)
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    return shape, d, G.k0_of(lam), ang, mat, flags, x


def make_small_ops():
    out = {}
    for idx in range(len(SMALL)):
        shape, d, k0, ang, mat, flags, x = small_inputs(idx)
        g = O.Grid(*shape, *d, k0)
        R = O.Reference(g, EPS_TABLE, *ang)
        R.set_geometry(mat, flags)
        out[f"green{idx}"] = R.green()
        out[f"inc{idx}"] = R.incident()
        out[f"ax{idx}"] = R.matvec(x, conj=False)
        out[f"ahx{idx}"] = R.matvec(x, conj=True)
        R.release()
    np.savez_compressed(os.path.join(OUT, "small_ops.npz"), **out)


def solve_case():
    """A small seeded scattering problem every driver converges on."""
    w = G.single_sphere(n=12, voxel_nm=2.0, diameter_nm=20.0, eps_physics=-4.0 + 0.3j, wavelength_nm=500.0,
                        theta=20.0, phi=30.0, psi=40.0)
    return w


def make_small_solves():
    w = solve_case()
    g = O.Grid(*w.shape, *w.d, w.k0)
    out = {}
    for name, thr in [("bicgstab", 1e-8), ("cors", 1e-8), ("bicorstab", 1e-8), ("bicg", 1e-8), ("cg", 1e-12)]:
        R = O.Reference(g, w.eps_table, w.theta, w.phi, w.psi)
        R.set_geometry(w.material, w.flags)
        R.green()
        R.incident()
        x, steps, err = R.solve(name, thr)
        out[f"{name}_x"] = x
        out[f"{name}_steps"] = steps
        out[f"{name}_err"] = err
        out[f"{name}_thr"] = thr
        R.release()
    np.savez_compressed(os.path.join(OUT, "small_solves.npz"), **out)


def make_c1():
    w = G.single_sphere()
    g = O.Grid(*w.shape, *w.d, w.k0)
    R = O.Reference(g, w.eps_table, w.theta, w.phi, w.psi)
    R.sphere_geometry(w.meta["diameter"], w.meta["box"], w.meta["box"], w.meta["box"])
    m, f = R.get_geometry()
    assert (m == w.material).all() and (f == w.flags).all()
    R.green()
    R.incident()
    x, steps, err = R.solve("bicgstab", 1e-6)
    fwd = R.farfield1()
    ext, metal, active = R.nearfield()
    R.release()
    mask = w.flags.astype(bool)
    np.savez_compressed(os.path.join(OUT, "c1_sphere.npz"), steps=steps, err=err, x_flagged=x[mask],
                        forward_rcs=fwd, ext_over_cs=ext, metal_abs_over_cs=metal)


if __name__ == "__main__":
    make_small_ops()
    make_small_solves()
    make_c1()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
