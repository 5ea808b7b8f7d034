"""Grids, materials and edge flags for the VIE workloads (host-side set-up).

The reference derives the voxel material and the edge-unknown flags from an
analytic geometry ``Model_Identifier(x, y, z)`` (Model.h:216-300):

* ``GetMaterial`` (Model.h:305-332) samples the voxel centre
  ``(i*dx + 0.5*dx, j*dy + 0.5*dy, k*dz + 0.5*dz)``;
* ``GetFlag`` (Model.h:335-398) keeps the x-directed unknown of edge
  ``(i, j, k)`` only if the face point ``((i+1)dx, (j+0.5)dy, (k+0.5)dz)`` and
  the two neighbouring voxel centres (face point -/+ dx/2) are all non-air;
  likewise for y and z.

This module evaluates the same rule, with the same floating-point
expressions, on label functions for the workloads below.  Lengths are in the
reference's unit of 100 nm (``WScale = 100``, ReadFile.h:7): ``nm(1.25)``
is 1.25 nm.  Permittivities are given in the physics convention (positive
imaginary part = loss) and converted with :func:`to_reference_eps`, because
the reference uses ``exp(+j omega t)`` (GreenFunction.h:65-67).

Workloads (sizes, materials and seeds as specified for each benchmark case;
box placements, layer heights and sphere counts the specification leaves open
are fixed here):

* :func:`single_sphere`     -- one sphere centred in a cubic box (the
  reference's own model, Model.h:51-56, 222-236)
* :func:`sphere_cluster`    -- non-overlapping random spheres
* :func:`solar_cell`        -- layered organic solar cell with embedded spheres
* :func:`design_stack`      -- solar-cell stack with a per-voxel design region
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

PI = 3.1415926535897932384626433832795  # common.h:17
Z0 = 120 * PI                            # common.h:18
WSCALE = 100.0                           # ReadFile.h:7
AIR_DUMMY = 1.1 + 0.0j                   # Model.h:82, avoids 1/(eps - 1) = 1/0


def nm(x):
    """Length in nanometres -> the reference's 100 nm unit."""
    return np.asarray(x, dtype=np.float64) / WSCALE


def k0_of(wavelength_nm: float) -> float:
    """Free-space wavenumber for a wavelength in nm (Model.h:105-106)."""
    return 2 * PI / (wavelength_nm / WSCALE)


def to_reference_eps(eps_physics):
    """Physics convention (exp(-i omega t), Im > 0 lossy) -> reference (exp(+j omega t))."""
    return np.conj(np.asarray(eps_physics, dtype=np.complex128))


def drude_silver(wavelength_nm, eps_inf=3.7, wp_ev=9.0, gamma_ev=0.018):
    """Drude permittivity eps(w) = eps_inf - wp^2 / (w^2 + i gamma w), physics convention."""
    w = 1239.84 / np.asarray(wavelength_nm, dtype=np.float64)
    return eps_inf - wp_ev ** 2 / (w ** 2 + 1j * gamma_ev * w)


def material_and_flags(label, shape, d):
    """GetMaterial + GetFlag on the label function ``label(x, y, z) -> uint8``."""
    nx, ny, nz = shape
    dx, dy, dz = d
    i = np.arange(nx, dtype=np.float64)[:, None, None]
    j = np.arange(ny, dtype=np.float64)[None, :, None]
    k = np.arange(nz, dtype=np.float64)[None, None, :]
    # GetMaterial, Model.h:319-324
    mat = label(i * dx + 0.5 * dx, j * dy + 0.5 * dy, k * dz + 0.5 * dz).astype(np.uint8)
    mat = np.broadcast_to(mat, shape).copy()
    flags = np.zeros((3,) + tuple(shape), np.uint8)
    # x rooftop, Model.h:352-364
    px, py, pz = (i + 1) * dx, (j + 0.5) * dy, (k + 0.5) * dz
    fx = (label(px, py, pz) != 0) & (label(px - 0.5 * dx, py, pz) != 0) & (label(px + 0.5 * dx, py, pz) != 0)
    # y rooftop, Model.h:367-379
    px, py, pz = (i + 0.5) * dx, (j + 1) * dy, (k + 0.5) * dz
    fy = (label(px, py, pz) != 0) & (label(px, py - 0.5 * dy, pz) != 0) & (label(px, py + 0.5 * dy, pz) != 0)
    # z rooftop, Model.h:382-394
    px, py, pz = (i + 0.5) * dx, (j + 0.5) * dy, (k + 1) * dz
    fz = (label(px, py, pz) != 0) & (label(px, py, pz - 0.5 * dz) != 0) & (label(px, py, pz + 0.5 * dz) != 0)
    flags[0] = np.broadcast_to(fx, shape)
    flags[1] = np.broadcast_to(fy, shape)
    flags[2] = np.broadcast_to(fz, shape)
    return mat, flags


@dataclass
class Workload:
    """Everything one solve needs, in the reference's conventions."""
    name: str
    shape: tuple
    d: tuple                      # (dx, dy, dz), 100 nm units
    k0: float
    material: np.ndarray          # uint8 labels (0 air, 1 spacer, 2 metal, 3 active)
    flags: np.ndarray             # (3, nx, ny, nz) uint8
    eps_table: np.ndarray         # reference-convention permittivity per label
    eps_voxel: np.ndarray | None = None  # per-voxel override (reference convention)
    theta: float = 0.0
    phi: float = 0.0
    psi: float = 0.0
    cross_section: float = 1.0    # geometric cross section used to normalise Q_ext / Q_abs
    meta: dict = field(default_factory=dict)

    @property
    def eps(self) -> np.ndarray:
        """Per-voxel permittivity (reference convention)."""
        if self.eps_voxel is not None:
            return self.eps_voxel
        return self.eps_table[self.material]

    @property
    def a(self) -> int:
        return int(np.prod(self.shape))


def _sphere_label(centres, radii, inside=2):
    centres = np.asarray(centres, np.float64)
    radii = np.asarray(radii, np.float64)

    def lab(x, y, z):
        shp = np.broadcast_shapes(np.shape(x), np.shape(y), np.shape(z))
        out = np.zeros(shp, np.uint8)
        axes = _axis_vectors(x, y, z, shp)
        for (cx, cy, cz), r in zip(centres, radii):
            if axes is not None:
                # only the bounding box of the sphere can be inside it
                sl = []
                for v, c in zip(axes, (cx, cy, cz)):
                    idx = np.nonzero(np.abs(v - c) <= r * (1 + 1e-12) + 1e-15)[0]
                    if idx.size == 0:
                        break
                    sl.append(slice(int(idx[0]), int(idx[-1]) + 1))
                if len(sl) < 3:
                    continue
                xs = np.asarray(x)[sl[0], :, :] if np.ndim(x) == 3 and np.shape(x)[0] > 1 else x
                ys = np.asarray(y)[:, sl[1], :] if np.ndim(y) == 3 and np.shape(y)[1] > 1 else y
                zs = np.asarray(z)[:, :, sl[2]] if np.ndim(z) == 3 and np.shape(z)[2] > 1 else z
                # distance from the centre as Model.h:227, inside when <= radius (:229)
                v = np.sqrt((xs - cx) ** 2 + (ys - cy) ** 2 + (zs - cz) ** 2)
                sub = out[sl[0], sl[1], sl[2]]
                out[sl[0], sl[1], sl[2]] = np.where(v <= r, np.uint8(inside), sub)
            else:
                v = np.sqrt((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2)
                out = np.where(v <= r, np.uint8(inside), out)
        return out
    return lab


def _axis_vectors(x, y, z, shp):
    """The 1-D coordinate vectors if x, y, z are per-axis arrays of shapes
    (n,1,1), (1,n,1), (1,1,n) (how material_and_flags calls the labels)."""
    try:
        if (len(shp) == 3 and np.shape(x) == (shp[0], 1, 1) and np.shape(y) == (1, shp[1], 1)
                and np.shape(z) == (1, 1, shp[2])):
            return np.ravel(x), np.ravel(y), np.ravel(z)
    except Exception:
        pass
    return None


def single_sphere(n=32, voxel_nm=1.25, diameter_nm=36.0, box_nm=None, eps_physics=-4.42 + 0.21j,
                  wavelength_nm=400.0, theta=0.0, phi=0.0, psi=0.0) -> Workload:
    """One sphere centred in a cubic box of n voxels (Model_Identifier, Model.h:222-236)."""
    d = float(nm(voxel_nm))
    box = float(nm(box_nm if box_nm is not None else n * voxel_nm))
    dia = float(nm(diameter_nm))
    lab = _sphere_label([(box / 2.0, box / 2.0, box / 2.0)], [0.5 * dia])
    mat, flags = material_and_flags(lab, (n, n, n), (d, d, d))
    table = np.array([AIR_DUMMY, 2.0, to_reference_eps(eps_physics), 2.0], np.complex128)
    return Workload("single_sphere", (n, n, n), (d, d, d), k0_of(wavelength_nm), mat, flags, table,
                    theta=theta, phi=phi, psi=psi, cross_section=PI * dia * dia / 4.0,
                    meta={"diameter": dia, "box": box, "wavelength_nm": wavelength_nm})


def _place_spheres(rng, count, rmin, rmax, lo, hi, max_tries=200000):
    """Random non-overlapping spheres: centre uniform in [lo + r, hi - r], reject overlaps."""
    cs, rs = [], []
    tries = 0
    while len(cs) < count and tries < max_tries:
        tries += 1
        r = rng.uniform(rmin, rmax) if rmax > rmin else rmin
        c = np.array([rng.uniform(lo[q] + r, hi[q] - r) for q in range(3)])
        if all(np.linalg.norm(c - c2) >= r + r2 for c2, r2 in zip(cs, rs)):
            cs.append(c)
            rs.append(r)
    if len(cs) < count:
        raise RuntimeError("could not place the requested spheres without overlap")
    return np.array(cs), np.array(rs)


def sphere_cluster(n=128, voxel_nm=1.0, count=40, rmin_nm=5.0, rmax_nm=15.0, eps_physics=-1.66 + 5.74j,
                   eps_background=1.77, wavelength_nm=500.0, seed=2) -> Workload:
    """Random cluster of non-overlapping spheres in a cubic grid.

    The reference has only a vacuum background (k0, Z0, common.h:18); a
    background eps_b is mapped to the equivalent vacuum problem
    lambda -> lambda / sqrt(eps_b), eps -> eps / eps_b.
    """
    rng = np.random.default_rng(seed)
    d = float(nm(voxel_nm))
    L = n * d
    cs, rs = _place_spheres(rng, count, float(nm(rmin_nm)), float(nm(rmax_nm)), [0, 0, 0], [L, L, L])
    lab = _sphere_label(cs, rs)
    mat, flags = material_and_flags(lab, (n, n, n), (d, d, d))
    table = np.array([AIR_DUMMY, 2.0, to_reference_eps(eps_physics / eps_background), 2.0], np.complex128)
    lam = wavelength_nm / np.sqrt(eps_background)
    return Workload("sphere_cluster", (n, n, n), (d, d, d), k0_of(lam), mat, flags, table,
                    cross_section=float(np.sum(PI * rs ** 2)),
                    meta={"centres": cs, "radii": rs, "wavelength_nm": wavelength_nm,
                          "eps_background": eps_background})


def _stack_label(L_xy, z_spacer, z_active, centres=(), radii=()):
    """Layered stack inside the box (0, L) in x and y (the reference's layer tests use
    |x - L/2| < L/2, Model.h:264-290): spacer z in [0, z_spacer), active layer
    [z_spacer, z_active), air above; spheres (label 2) override the layers."""
    sph = _sphere_label(centres, radii) if len(radii) else None

    def lab(x, y, z):
        shp = np.broadcast_shapes(np.shape(x), np.shape(y), np.shape(z))
        inbox = (np.abs(x - L_xy[0] / 2.0) < L_xy[0] / 2.0) & (np.abs(y - L_xy[1] / 2.0) < L_xy[1] / 2.0)
        out = np.zeros(shp, np.uint8)
        out = np.where(inbox & (z > 0) & (z < z_spacer), np.uint8(1), out)
        out = np.where(inbox & (z >= z_spacer) & (z < z_active), np.uint8(3), out)
        if sph is not None:
            s = sph(x, y, z)
            out = np.where(s != 0, s, out)
        return np.broadcast_to(out, shp)
    return lab


def solar_cell(shape=(256, 256, 256), voxel_nm=1.0, spacer_nm=40.0, active_nm=120.0, nspheres=16,
               radius_nm=20.0, eps_spacer=2.40 + 0.05j, eps_active=3.80 + 0.60j, eps_metal=-8.5 + 0.3j,
               wavelength_nm=550.0, sphere_z_nm=(60.0, 140.0), seed=3, psi=0.0) -> Workload:
    """Organic solar-cell stack with metal spheres embedded in the active layer."""
    rng = np.random.default_rng(seed)
    d = float(nm(voxel_nm))
    nx, ny, nz = shape
    Lx, Ly = nx * d, ny * d
    r = float(nm(radius_nm))
    z0, z1 = float(nm(sphere_z_nm[0])), float(nm(sphere_z_nm[1]))
    if nspheres:
        # centres: x, y in [r, L - r], z in [z0, z1] (the sphere may cross the layer boundary)
        cs, rs = _place_spheres(rng, nspheres, r, r, [0.0, 0.0, z0 - r], [Lx, Ly, z1 + r])
    else:
        cs, rs = np.zeros((0, 3)), np.zeros(0)
    zs, za = float(nm(spacer_nm)), float(nm(spacer_nm + active_nm))
    lab = _stack_label((Lx, Ly), zs, za, cs, rs)
    mat, flags = material_and_flags(lab, shape, (d, d, d))
    table = np.array([AIR_DUMMY, to_reference_eps(eps_spacer), to_reference_eps(eps_metal),
                      to_reference_eps(eps_active)], np.complex128)
    return Workload("solar_cell", tuple(shape), (d, d, d), k0_of(wavelength_nm), mat, flags, table, psi=psi,
                    cross_section=Lx * Ly,
                    meta={"centres": cs, "radii": rs, "wavelength_nm": wavelength_nm})


def design_stack(shape=(128, 128, 64), voxel_nm=1.0, spacer_nm=16.0, active_top_nm=64.0,
                 region_nm=((32, 96), (32, 96), (24, 56)), wavelength_nm=550.0, seed=5,
                 eps_spacer=2.40 + 0.05j, eps_active=3.80 + 0.60j) -> Workload:
    """Solar-cell stack whose design region carries a per-voxel permittivity
    Re in [1, 4], Im in [0, 0.5] (physics convention)."""
    rng = np.random.default_rng(seed)
    d = float(nm(voxel_nm))
    nx, ny, nz = shape
    lab = _stack_label((nx * d, ny * d), float(nm(spacer_nm)), float(nm(active_top_nm)))
    mat, flags = material_and_flags(lab, shape, (d, d, d))
    table = np.array([AIR_DUMMY, to_reference_eps(eps_spacer), 2.0, to_reference_eps(eps_active)], np.complex128)
    eps = table[mat].copy()
    (x0, x1), (y0, y1), (z0, z1) = [(int(a / voxel_nm), int(b / voxel_nm)) for a, b in region_nm]
    shp = (x1 - x0, y1 - y0, z1 - z0)
    design = rng.uniform(1.0, 4.0, shp) + 1j * rng.uniform(0.0, 0.5, shp)
    eps[x0:x1, y0:y1, z0:z1] = to_reference_eps(design)
    region = np.zeros(shape, bool)
    region[x0:x1, y0:y1, z0:z1] = True
    return Workload("design_stack", tuple(shape), (d, d, d), k0_of(wavelength_nm), mat, flags, table,
                    eps_voxel=eps, cross_section=nx * d * ny * d,
                    meta={"region": region, "wavelength_nm": wavelength_nm})


def batch_sweep(shape=(96, 96, 48), voxel_nm=1.0, n_wavelengths=64, wavelength_range_nm=(350.0, 800.0),
                psis=(0.0, 90.0), spacer_nm=8.0, active_nm=24.0, nspheres=4, radius_nm=8.0,
                sphere_z_nm=(16.0, 24.0), seed=4):
    """Wavelength x polarisation sweep over one solar-cell grid: the 256^3 stack
    scaled to a 48-voxel height (spacer 8 nm, active layer 24 nm, Ag spheres of
    radius 8 nm in the active layer), silver from the Drude model at each
    wavelength (drude_silver), the layers at their fixed permittivities;
    polarisation x (psi = 0) and y (psi = 90).  Returns the list of
    n_wavelengths * len(psis) workloads (all on the same grid)."""
    base = solar_cell(shape=shape, voxel_nm=voxel_nm, spacer_nm=spacer_nm, active_nm=active_nm, nspheres=nspheres,
                      radius_nm=radius_nm, sphere_z_nm=sphere_z_nm, seed=seed)
    out = []
    for lam in np.linspace(wavelength_range_nm[0], wavelength_range_nm[1], n_wavelengths):
        table = base.eps_table.copy()
        table[2] = to_reference_eps(drude_silver(lam))
        for psi in psis:
            out.append(Workload("batch_sweep", base.shape, base.d, k0_of(lam), base.material, base.flags, table,
                                psi=psi, cross_section=base.cross_section,
                                meta={"wavelength_nm": float(lam), "psi": psi}))
    return out


def batch_spheres(count=48, edges=tuple(range(16, 97, 8)), voxel_nm=1.0, wavelength_nm=550.0, seed=4):
    """Single spheres on uneven grids: edge n drawn from `edges`, diameter (n - 2)
    voxels, permittivity Re uniform in [-6, -1], Im uniform in [0.1, 1.0]
    (physics convention)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(np.asarray(edges)))
        eps = rng.uniform(-6.0, -1.0) + 1j * rng.uniform(0.1, 1.0)
        w = single_sphere(n=n, voxel_nm=voxel_nm, diameter_nm=(n - 2) * voxel_nm, eps_physics=eps,
                          wavelength_nm=wavelength_nm)
        w.meta["eps_physics"] = eps
        out.append(w)
    return out
