"""Cross sections from a solved current, restated in numpy on the host.

The reference computes these in NearFar.h after the solve: extinction from
the forward-scattering amplitude (FarField1, NearFar.h:16-109) and absorption
from the edge currents (NearField, NearFar.h:180-250).  The library computes
them on the GPU from the solution in device memory (vie_farfield1,
vie_farfield2, vie_nearfield; Context.farfield1 / farfield2 / nearfield).
This module is the host restatement: the edge masks of the adjoint objective
(edge_mask) and bench.py's comparison of the mixed and FP64 solves' cross
sections on fields copied to the host.
"""
from __future__ import annotations

import numpy as np

from .geometry import PI, Z0


def forward_scattering(shape, d, k0, x, theta=0.0, phi=0.0, psi=0.0) -> float:
    """Forward_RCS of FarField1 (NearFar.h:16-109)."""
    nx, ny, nz = shape
    dx, dy, dz = d
    v1, v2 = np.cos(PI * theta / 180.0), np.sin(PI * theta / 180.0)
    v3, v4 = np.cos(PI * phi / 180.0), np.sin(PI * phi / 180.0)
    vx, vy, vz = v2 * v3, v2 * v4, v1
    px = np.exp(1j * k0 * ((np.arange(nx) + 0.5) * dx) * vx)
    py = np.exp(1j * k0 * ((np.arange(ny) + 0.5) * dy) * vy)
    pz = np.exp(1j * k0 * ((np.arange(nz) + 0.5) * dz) * vz)
    vol = dx * dy * dz
    S = [np.einsum("i,j,k,ijk->", px, py, pz, x[c]) for c in range(3)]
    S[0] = np.exp(1j * k0 * 0.5 * dx * vx) * S[0] * vol
    S[1] = np.exp(1j * k0 * 0.5 * dy * vy) * S[1] * vol
    S[2] = np.exp(1j * k0 * 0.5 * dz * vz) * S[2] * vol
    tm = Z0 * (S[0].real * v1 * v3 + S[1].real * v1 * v4 - S[2].real * v2)
    te = Z0 * (S[0].real * v4 - S[1].real * v3)
    return float(np.cos(PI * psi / 180.0) * tm - np.sin(PI * psi / 180.0) * te)


def absorption(shape, d, k0, x, eps, material, metal_label=2, active_label=3):
    """(Ene_Metal, Ene_Active, Absorb_Volume) of NearField (NearFar.h:180-250)."""
    nx, ny, nz = shape
    dV = d[0] * d[1] * d[2]
    core = (slice(0, nx - 1), slice(0, ny - 1), slice(0, nz - 1))
    em = ea = av = 0.0
    for c in range(3):
        nb = [slice(0, nx - 1), slice(0, ny - 1), slice(0, nz - 1)]
        nb[c] = slice(1, [nx, ny, nz][c])
        nb = tuple(nb)
        V2 = 1.0 / (eps[nb] - 1.0) + 1.0 / (eps[core] - 1.0)
        V1 = V2 * (-0.5j * Z0 / k0)
        V4 = 2.0 / V2 + 1.0
        absE = np.abs(x[c][core]) * np.abs(V1)
        contrib = k0 / Z0 * (-V4.imag) * absE * absE * dV
        m2, m3 = material[nb], material[core]
        em += float(contrib[(m2 == metal_label) & (m3 == metal_label)].sum())
        act = (m2 == active_label) & (m3 == active_label)
        ea += float(contrib[act].sum())
        av += float(act.sum()) * dV
    return em, ea, av


def edge_mask(material, label=3):
    """Edge set of NearField's per-material sum (NearFar.h:186-250): bit f of voxel
    (i, j, k) is set when i, j, k < N - 1 and the voxel and its +f neighbour both
    hold ``label`` (3: Ene_Active, 2: Ene_Metal)."""
    m = np.asarray(material)
    nx, ny, nz = m.shape
    out = np.zeros(m.shape, np.uint8)
    core = (slice(0, nx - 1), slice(0, ny - 1), slice(0, nz - 1))
    for f in range(3):
        nb = [slice(0, nx - 1), slice(0, ny - 1), slice(0, nz - 1)]
        nb[f] = slice(1, m.shape[f])
        sel = (m[core] == label) & (m[tuple(nb)] == label)
        out[core] |= (sel.astype(np.uint8) << f)
    return out


def cross_sections(w, x) -> dict:
    """Extinction and absorption efficiencies of a Workload's solution."""
    fwd = forward_scattering(w.shape, w.d, w.k0, x, w.theta, w.phi, w.psi)
    em, ea, av = absorption(w.shape, w.d, w.k0, x, w.eps, w.material)
    return {"q_ext": fwd / w.cross_section, "q_abs_metal": em * Z0 / w.cross_section,
            "active_abs_per_volume": 3.0 * ea / av if av > 0 else 0.0}
