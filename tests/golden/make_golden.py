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
  geometry.npz       the reference's GetMaterial / GetFlag of its one-sphere
                     model (Model_Identifier) on a cubic and a non-cubic grid
  post_ops.npz       FarField1, FarField2 (RCS) and NearField outputs of the
                     reference on seeded currents of the small cases
  dropin_blocks.npz  X/Y/Z_FFT rows, L_DC_Dq, L_Dq, L??_DO (and conjugate
                     twins) and Current_Reset on small seeded cases
  c2_<solver>.npz    the 128^3 cluster of 40 gold spheres (background eps 1.77
                     mapped to vacuum) solved by the reference's CORS_FFT and
                     BICGSTAB_FFT to 1e-8 and BICGSTAB_FFT to 1e-12: step
                     count, last error, the field at 8192 seeded entries, two
                     seeded random projections and the norm of the field,
                     FarField1's forward value and the metal absorption
  dropin_program.npz the reference's unchanged main program (CG_FFT_VIE.cpp,
                     41 wavelengths) on the synthetic material tables of
                     program_tables(): its Ene_Metal, Ene_Active, Grid and
                     RCS outputs and the step count of each solve
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


# C2: (driver, CG_THR) of each fixture
C2_RUNS = {"cors": ("cors", 1e-8), "bicgstab": ("bicgstab", 1e-8), "bicgstab_tight": ("bicgstab", 1e-12)}
C2_SAMPLES = 8192


def c2_probe(x):
    """Size-independent summary of a C2 field (shared with the tests): the
    field at seeded entries, two seeded random complex projections, the norm."""
    flat = np.ascontiguousarray(x, np.complex128).ravel()
    rng = np.random.default_rng(22)
    idx = np.sort(rng.choice(flat.size, size=C2_SAMPLES, replace=False))
    proj = []
    for _ in range(2):
        wv = rng.standard_normal(flat.size) + 1j * rng.standard_normal(flat.size)
        proj.append(np.vdot(wv, flat))
    return idx, flat[idx], np.array(proj), float(np.linalg.norm(flat))


def make_c2(which):
    """One C2 fixture (about 20-40 minutes of one host core for each run)."""
    import time
    solver, thr = C2_RUNS[which]
    w = G.sphere_cluster()
    g = O.Grid(*w.shape, *w.d, w.k0)
    R = O.Reference(g, w.eps_table, w.theta, w.phi, w.psi)
    R.set_geometry(w.material, w.flags)
    R.green()
    R.incident()
    t = time.perf_counter()
    x, steps, err = R.solve(solver, thr)
    secs = time.perf_counter() - t
    R.release()
    idx, samples, proj, norm = c2_probe(x)
    fwd = O.farfield1(g, x)
    metal, _, _ = O.absorption(g, x, w.eps, w.material)
    np.savez_compressed(os.path.join(OUT, f"c2_{which}.npz"), steps=steps, err=err, thr=thr, idx=idx,
                        samples=samples, proj=proj, norm=norm, forward_rcs=fwd, metal=metal,
                        reference_seconds=secs)
    print(f"c2 {which}: {steps} steps, err {err:.3e}, {secs:.0f} s")


GEOMETRY_CASES = [
    # (shape, d, dia, box)
    ((32, 32, 32), (0.0125, 0.0125, 0.0125), 0.36, (0.4, 0.4, 0.4)),
    ((20, 24, 16), (0.011, 0.01, 0.013), 0.18, (0.22, 0.24, 0.2)),
]


def make_geometry():
    out = {}
    for idx, (shape, d, dia, box) in enumerate(GEOMETRY_CASES):
        g = O.Grid(*shape, *d, G.k0_of(500.0))
        R = O.Reference(g, EPS_TABLE)
        R.sphere_geometry(dia, *box)
        m, f = R.get_geometry()
        out[f"material{idx}"], out[f"flags{idx}"] = m, f
        R.release()
    np.savez_compressed(os.path.join(OUT, "geometry.npz"), **out)


def make_post_ops():
    out = {}
    for idx in range(len(SMALL)):
        shape, d, k0, ang, mat, flags, x = small_inputs(idx)
        g = O.Grid(*shape, *d, k0)
        R = O.Reference(g, EPS_TABLE, *ang)
        R.set_geometry(mat, flags)
        R.set_cross_section(0.37)
        R.set_current(x)
        out[f"ff1_{idx}"] = R.farfield1()
        rt, rp = R.farfield2()
        out[f"rcs_theta{idx}"], out[f"rcs_phi{idx}"] = rt, rp
        out[f"near{idx}"] = np.array(R.nearfield())
        R.release()
    np.savez_compressed(os.path.join(OUT, "post_ops.npz"), **out)


def make_dropin_blocks():
    out = {}
    for idx in (0, 1, 3):
        shape, d, k0, ang, mat, flags, x = small_inputs(idx)
        g = O.Grid(*shape, *d, k0)
        R = O.Reference(g, EPS_TABLE, *ang)
        R.set_geometry(mat, flags)
        R.green()
        for which in range(6):
            out[f"row{idx}_{which}"] = R.row(which, x)
        for conj in (0, 1):
            for src in range(3):
                out[f"blk{idx}_0_{src}_{src}_{conj}"] = R.block(0, src, src, conj, x)
                out[f"blk{idx}_2_{src}_{src}_{conj}"] = R.block(2, src, src, conj, x)
                for fld in range(3):
                    if fld != src:
                        out[f"blk{idx}_1_{src}_{fld}_{conj}"] = R.block(1, src, fld, conj, x)
        for flag in range(3):
            out[f"reset{idx}_{flag}"] = R.reset(x[flag], flag)
        R.release()
    np.savez_compressed(os.path.join(OUT, "dropin_blocks.npz"), **out)


def program_tables():
    """Synthetic permittivity tables (41 rows, 400-800 nm, reference sign) for
    the files the main program reads: PEDOT_epr.txt, Au_epr.txt, P3HT_PCBM_epr.txt."""
    lam = 400.0 + 10.0 * np.arange(41)
    t = (lam - 400.0) / 400.0
    pedot = np.stack([2.4 + 0.1 * t, -0.05 - 0.02 * t], 1)
    metal = np.stack([-1.0 - 4.0 * t, -3.0 + 0.5 * t], 1)
    p3ht = np.stack([3.8 - 0.4 * t, -0.6 + 0.3 * t], 1)
    return {"PEDOT_epr.txt": pedot, "Au_epr.txt": metal, "P3HT_PCBM_epr.txt": p3ht}


def write_program_tree(root):
    """data/ with the tables, result/ for the outputs, run/ as the working directory."""
    for sub in ("data", "result", "run"):
        os.makedirs(os.path.join(root, sub), exist_ok=True)
    for name, tab in program_tables().items():
        with open(os.path.join(root, "data", name), "w") as f:
            for re_, im_ in tab:
                f.write(f" {re_:.16e}\t {im_:.16e}\n")


def read_program_results(root):
    res = os.path.join(root, "result")
    metal = np.array([np.loadtxt(os.path.join(res, f"Ene_Metal{m}.txt")) for m in range(41)])
    active = np.array([np.loadtxt(os.path.join(res, f"Ene_Active{m}.txt")) for m in range(41)])
    grid = np.array([np.loadtxt(os.path.join(res, f"Grid{m}.txt")) for m in range(41)])
    rcs = np.array([np.loadtxt(os.path.join(res, f"RCS{m}.txt")) for m in range(41)])
    return {"metal": metal, "active": active, "grid": grid, "rcs": rcs}


def program_steps(stdout):
    """Step count of every solve, from the drivers' "Steps: m" lines."""
    return [int(line.split(":")[1]) for line in stdout.splitlines() if line.startswith("Steps:")]


def make_dropin_program():
    import subprocess
    import tempfile
    exe = os.path.join(ROOT, "oracle", "_ref", "vie_fft_ref_main")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-main"], check=True)
    with tempfile.TemporaryDirectory() as tmp:
        write_program_tree(tmp)
        run = subprocess.run([exe], cwd=os.path.join(tmp, "run"), check=True, stdout=subprocess.PIPE,
                             encoding="latin-1")
        out = read_program_results(tmp)
    out["steps"] = np.array(program_steps(run.stdout))
    np.savez_compressed(os.path.join(OUT, "dropin_program.npz"), **out)


if __name__ == "__main__":
    import sys as _sys
    which = _sys.argv[1:] or ["ops", "solves", "c1", "geometry", "post", "blocks", "program"]
    if "ops" in which:
        make_small_ops()
    if "solves" in which:
        make_small_solves()
    if "c1" in which:
        make_c1()
    if "geometry" in which:
        make_geometry()
    if "post" in which:
        make_post_ops()
    if "blocks" in which:
        make_dropin_blocks()
    if "program" in which:
        make_dropin_program()
    for k in C2_RUNS:
        if f"c2_{k}" in which:
            make_c2(k)
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
