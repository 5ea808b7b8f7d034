"""Result files in the reference's formats, so that its MATLAB
post-processing (Postprocess1_NP.m, Postprocess2_SolarCell.m) reads the
output of batched GPU runs unchanged.

Per frequency point m (0-based, the reference's Fre_Point) in result_dir:
  Ene_Metal{m}.txt   "%d %.15lf %.15lf": wavelength label, Forward_RCS / Cross_Section,
                     Ene_Metal * Z0 / Cross_Section            (NearFar.h:276-278)
  Ene_Active{m}.txt  "%d %.15lf": wavelength label, 3 Ene_Active / Absorb_Volume (:280-281)
  Grid{m}.txt        "%d %d %d %d %.15lf %.15lf %.15lf": m, Nx, Ny, Nz, dx, dy, dz (:283)
  RCS{m}.txt         181 lines "%.15lf %.15lf": RCS_Theta, RCS_Phi in dB (:465-475)
  LField/HField/VField{m}.txt  the current on the planes k = Nz/2, j = Ny/2, i = Nx/2 of the
                     core i < Nx-1, j < Ny-1, k < Nz-1, six "%.15lf" per line (:252-270)
merge_points() combines the per-point Ene_Metal / Ene_Active / Grid files into
Ene_Metal.txt, Ene_Active.txt, Grid.txt and removes them, like main.cpp:53-109.
Numbers are formatted with C's rules: "%.15f", and the NaN of 0/0 (an empty
active volume) as glibc prints it, "-nan".
"""
from __future__ import annotations

import math
import os

import numpy as np

Z0 = 120.0 * math.pi
WBEGIN, WINTERVAL = 400, 10   # ReadFile.h:4-6


def _f(v: float) -> str:
    v = float(v)
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    if math.isinf(v):
        return "-inf" if v < 0 else "inf"
    return "%.15f" % v


def _ratio(a: float, b: float) -> float:
    """a / b with IEEE semantics; 0/0 gives the x86 default NaN (sign bit set),
    which is what the reference divides out for an empty active volume."""
    if b == 0.0:
        if a == 0.0 or math.isnan(a):
            return -math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)
    return a / b


def wavelength_label(fre_point: int) -> int:
    return WBEGIN + int(fre_point) * WINTERVAL


def write_point(result_dir, fre_point, shape, d, x, forward_rcs, cross_section, ene_metal, ene_active,
                absorb_volume, rcs_theta, rcs_phi, planes=True):
    """Write the files of one frequency point (see the module docstring).
    x: the current (3, nx, ny, nz) complex, only needed for the plane files."""
    os.makedirs(result_dir, exist_ok=True)
    m = int(fre_point)
    nx, ny, nz = shape
    lab = wavelength_label(m)
    with open(os.path.join(result_dir, f"Ene_Metal{m}.txt"), "w") as f:
        f.write(f"{lab} {_f(forward_rcs / cross_section)} {_f(ene_metal * Z0 / cross_section)}\n")
    with open(os.path.join(result_dir, f"Ene_Active{m}.txt"), "w") as f:
        f.write(f"{lab} {_f(_ratio(3.0 * ene_active, absorb_volume))}\n")
    with open(os.path.join(result_dir, f"Grid{m}.txt"), "w") as f:
        f.write(f"{m} {nx} {ny} {nz} {_f(d[0])} {_f(d[1])} {_f(d[2])}\n")
    with open(os.path.join(result_dir, f"RCS{m}.txt"), "w") as f:
        for a, b in zip(rcs_theta, rcs_phi):
            f.write(f"{_f(a)} {_f(b)}\n")
    if planes:
        x = np.asarray(x)
        core = x[:, : nx - 1, : ny - 1, : nz - 1]
        for name, sel in (("LField", core[:, :, :, int(nz / 2.0)] if int(nz / 2.0) < nz - 1 else None),
                          ("HField", core[:, :, int(ny / 2.0), :] if int(ny / 2.0) < ny - 1 else None),
                          ("VField", core[:, int(nx / 2.0), :, :] if int(nx / 2.0) < nx - 1 else None)):
            with open(os.path.join(result_dir, f"{name}{m}.txt"), "w") as f:
                if sel is None:
                    continue
                v = sel.reshape(3, -1)
                for q in range(v.shape[1]):
                    c = v[:, q]
                    f.write(" ".join(_f(t) for t in (c[0].real, c[0].imag, c[1].real, c[1].imag, c[2].real,
                                                      c[2].imag)) + "\n")


def merge_points(result_dir, count):
    """main.cpp:53-109: combine points 0..count-1 into Ene_Metal.txt,
    Ene_Active.txt and Grid.txt and remove the per-point files."""
    outs = {k: open(os.path.join(result_dir, f"{k}.txt"), "w") for k in ("Ene_Metal", "Ene_Active", "Grid")}
    try:
        for m in range(count):
            for k, fh in outs.items():
                p = os.path.join(result_dir, f"{k}{m}.txt")
                with open(p) as f:
                    t = f.read().split()
                if k == "Ene_Metal":
                    fh.write(f"{int(t[0])} {_f(float(t[1]))} {_f(float(t[2]))}\n")
                elif k == "Ene_Active":
                    fh.write(f"{int(t[0])} {_f(float(t[1]))}\n")
                else:
                    fh.write(f"{int(t[0])} {int(t[1])} {int(t[2])} {int(t[3])} {_f(float(t[4]))} "
                             f"{_f(float(t[5]))} {_f(float(t[6]))}\n")
                os.remove(p)
    finally:
        for fh in outs.values():
            fh.close()


def write_from_context(result_dir, fre_point, ctx, w, planes=True):
    """All files of one point from a solved context (post-processing on the GPU)."""
    fwd = ctx.farfield1(w.theta, w.phi, w.psi)
    em, ea, av = ctx.nearfield(w.material)
    rt, rp = ctx.farfield2(w.phi)
    x = ctx.solution() if planes else None
    write_point(result_dir, fre_point, w.shape, w.d, x, fwd, w.cross_section, em, ea, av, rt, rp, planes=planes)
