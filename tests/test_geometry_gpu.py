"""Geometry on the GPU (vie_set_geometry_scene) against the reference's own
GetMaterial / GetFlag (golden fixture geometry.npz, from the reference built
here) and, for the layered model, against a numpy evaluation of the same
primitive tests."""
import os

import numpy as np
import pytest

import vie_fft_b200 as V
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TABLE = np.array([1.1, 2.4 - 0.05j, -4.42 - 0.21j, 3.8 - 0.6j])


@pytest.mark.parametrize("idx", range(len(MG.GEOMETRY_CASES)))
def test_one_sphere_matches_reference(idx):
    gold = np.load(os.path.join(GOLD, "geometry.npz"))
    shape, d, dia, box = MG.GEOMETRY_CASES[idx]
    scene = [{"kind": V.PRIM_SPHERE, "label": 2, "c": tuple(b / 2 for b in box), "r": 0.5 * dia}]
    rng = np.random.default_rng(idx)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    with V.Context(*shape, *d, 10.0) as c:
        mat = c.set_scene(scene, TABLE)
        c.green()
        y_scene = c.matvec(x)
    np.testing.assert_array_equal(mat, gold[f"material{idx}"])
    # the flags: the operator of the scene context equals the one built from the reference's flags
    with V.Context(*shape, *d, 10.0) as c2:
        c2.set_flags(gold[f"flags{idx}"])
        c2.set_material(gold[f"material{idx}"], TABLE)
        c2.green()
        np.testing.assert_array_equal(y_scene, c2.matvec(x))


def _label_np(scene, x, y, z):
    def holds(p):
        dx, dy, dz = x - p["c"][0], y - p["c"][1], z - p["c"][2]
        if p["kind"] == V.PRIM_SPHERE:
            return np.sqrt(dx * dx + dy * dy + dz * dz) <= p["r"]
        if p["kind"] == V.PRIM_SPHERE_F32:
            return (dx * dx + dy * dy + dz * dz).astype(np.float32) < np.float32(p["r"] * p["r"])
        return (np.abs(dx) < p["h"][0]) & (np.abs(dy) < p["h"][1]) & (np.abs(dz) < p["h"][2])

    shp = np.broadcast_shapes(np.shape(x), np.shape(y), np.shape(z))
    out = np.zeros(shp, np.uint8)
    done = np.zeros(shp, bool)
    for p in scene:
        m = np.broadcast_to(holds(p), shp)
        if p.get("parent", -1) >= 0:
            m = m & np.broadcast_to(holds(scene[p["parent"]]), shp)
        out[m & ~done] = p["label"]
        done |= m
    return out


def test_layered_scene_matches_numpy():
    # the reference's layered solar-cell form (Model.h, commented model):
    # spheres only inside the spacer box, then the spacer, then the active layer
    shape, d = (40, 24, 22), (0.01, 0.01, 0.01)
    L, W, t1, t2 = 0.4, 0.24, 0.08, 0.12
    spacer = {"kind": V.PRIM_BOX, "label": 1, "c": (L / 2, W / 2, t1 / 2), "h": (L / 2, W / 2, t1 / 2)}
    active = {"kind": V.PRIM_BOX, "label": 3, "c": (L / 2, W / 2, t1 + t2 / 2), "h": (L / 2, W / 2, t2 / 2)}
    spheres = [{"kind": V.PRIM_SPHERE_F32, "label": 2, "c": (cx, W / 2, t1 / 2), "r": 0.04, "parent": 4}
               for cx in (0.06, 0.14, 0.22, 0.30)]
    scene = spheres + [spacer, active]
    nx, ny, nz = shape
    i = np.arange(nx)[:, None, None].astype(float)
    j = np.arange(ny)[None, :, None].astype(float)
    k = np.arange(nz)[None, None, :].astype(float)
    with V.Context(*shape, *d, 10.0) as c:
        mat = c.set_scene(scene, TABLE)
    ref = _label_np(scene, i * d[0] + 0.5 * d[0], j * d[1] + 0.5 * d[1], k * d[2] + 0.5 * d[2])
    np.testing.assert_array_equal(mat, ref)
    assert set(np.unique(mat)) == {0, 1, 2, 3}
    # edge flags: the three-point rule on the same label function
    px, py, pz = (i + 1) * d[0], (j + 0.5) * d[1], (k + 0.5) * d[2]
    fx = (_label_np(scene, px, py, pz) != 0) & (_label_np(scene, px - 0.005, py, pz) != 0) & \
         (_label_np(scene, px + 0.005, py, pz) != 0)
    with V.Context(*shape, *d, 10.0) as c1, V.Context(*shape, *d, 10.0) as c2:
        c1.set_scene(scene, TABLE)
        c1.green()
        flags = np.zeros((3,) + shape, np.uint8)
        flags[0] = fx
        for f, (a, b, cc) in ((1, ((i + 0.5) * d[0], (j + 1) * d[1], (k + 0.5) * d[2])),
                              (2, ((i + 0.5) * d[0], (j + 0.5) * d[1], (k + 1) * d[2]))):
            off = [0.0, 0.0, 0.0]
            off[f] = 0.5 * d[f]
            flags[f] = (_label_np(scene, a, b, cc) != 0) & \
                       (_label_np(scene, a - off[0], b - off[1], cc - off[2]) != 0) & \
                       (_label_np(scene, a + off[0], b + off[1], cc + off[2]) != 0)
        c2.set_flags(flags)
        c2.set_material(mat, TABLE)
        c2.green()
        rng = np.random.default_rng(3)
        x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
        np.testing.assert_array_equal(c1.matvec(x), c2.matvec(x))


def test_scene_errors():
    with V.Context(8, 8, 8, 0.01, 0.01, 0.01, 10.0) as c:
        with pytest.raises(V.VieError):
            c.set_scene([{"kind": 9, "label": 1}], TABLE)
        with pytest.raises(V.VieError):
            c.set_scene([{"kind": V.PRIM_BOX, "label": 1, "parent": 0, "h": (1, 1, 1)}], TABLE)
        with pytest.raises(V.VieError):
            c.set_scene([{"kind": V.PRIM_BOX, "label": 7, "h": (1, 1, 1)}], TABLE)
