"""ctypes bindings for the oracle (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module.  It loads

* ``oracle/_build/libvieoracle.so`` -- the C restatement of the reference hot
  path (``vie_oracle.c``).  If it is missing it is compiled here with ``make``
  (gcc only, no reference sources needed).
* ``oracle/_ref/libvieref.so`` -- the reference's own ``vie_fft`` headers
  compiled in place against the MKL shim (``ref_harness.cpp``).  It can only
  be built where the reference checkout exists; elsewhere ``ref_available()``
  returns False.

All arrays are numpy ``complex128`` / ``uint8`` in the reference layout
(C order, shape ``(nx, ny, nz)``; vectors of three components are shape
``(3, nx, ny, nz)``).  Permittivities use the reference sign convention
(lossy media have negative imaginary parts).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libvieoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvieref.so")

_lock = threading.Lock()
_oracle = None
_ref = None

_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_ubyte)


class VoGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("k0", ctypes.c_double)]


@dataclass
class Grid:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    k0: float

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    @property
    def a(self):
        return self.nx * self.ny * self.nz

    def c(self) -> VoGrid:
        return VoGrid(self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, self.k0)


def _p(arr, kind=_dp):
    return arr.ctypes.data_as(kind)


def _build(target: str) -> None:
    subprocess.run(["make", "-C", HERE, target], check=True, capture_output=True)


def lib():
    """The C restatement (compiled on demand with gcc)."""
    global _oracle
    with _lock:
        if _oracle is None:
            if not os.path.exists(ORACLE_SO):
                _build("all")
            L = ctypes.CDLL(ORACLE_SO)
            g = ctypes.POINTER(VoGrid)
            L.vo_green.argtypes = [g, _dp]
            L.vo_incident.argtypes = [g, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp]
            L.vo_matvec.argtypes = [g, _dp, _dp, _up, _dp, _dp, ctypes.c_int]
            L.vo_solve.argtypes = [g, _dp, _dp, _up, _dp, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int), _dp]
            L.vo_farfield1.argtypes = [g, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
            L.vo_farfield1.restype = ctypes.c_double
            L.vo_absorption.argtypes = [g, _dp, _dp, _up, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]
            L.vo_block.argtypes = [g, _dp, _dp, _dp]
            _oracle = L
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    """The reference's own code (oracle/_ref); raises if it was not built."""
    global _ref
    with _lock:
        if _ref is None:
            if not os.path.exists(REF_SO):
                raise FileNotFoundError(f"{REF_SO} not built (needs the reference checkout)")
            L = ctypes.CDLL(REF_SO)
            L.ref_setup.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [_dp, _dp] + [ctypes.c_double] * 3
            L.ref_set_geometry.argtypes = [_up] * 4
            L.ref_get_geometry.argtypes = [_up] * 4
            L.ref_sphere_geometry.argtypes = [ctypes.c_double] * 4
            L.ref_set_cross_section.argtypes = [ctypes.c_double]
            L.ref_green.argtypes = [_dp]
            L.ref_set_green.argtypes = [_dp]
            L.ref_incident.argtypes = [_dp, _dp, _dp]
            L.ref_set_incident.argtypes = [_dp, _dp, _dp]
            L.ref_matvec.argtypes = [_dp, _dp, ctypes.c_int]
            L.ref_time_block.argtypes = [_dp, _dp]
            L.ref_solve.argtypes = [ctypes.c_int, ctypes.c_double, _dp, ctypes.POINTER(ctypes.c_int), _dp]
            L.ref_set_current.argtypes = [_dp]
            L.ref_farfield1.argtypes = [_dp]
            L.ref_farfield2.argtypes = [_dp, _dp]
            L.ref_nearfield.argtypes = [_dp, _dp, _dp]
            L.ref_set_verbose.argtypes = [ctypes.c_int]
            L.ref_row.argtypes = [ctypes.c_int, _dp, _dp]
            L.ref_block.argtypes = [ctypes.c_int] * 4 + [_dp, _dp]
            L.ref_reset.argtypes = [_dp, ctypes.c_int]
            _ref = L
    return _ref


# ---------------------------------------------------------------------------
# restatement (vie_oracle.c)
# ---------------------------------------------------------------------------

def green(g: Grid) -> np.ndarray:
    out = np.zeros((2 * g.nx, 2 * g.ny, 2 * g.nz), np.complex128)
    rc = lib().vo_green(ctypes.byref(g.c()), _p(out))
    if rc:
        raise RuntimeError(f"vo_green failed ({rc})")
    return out


def incident(g: Grid, theta=0.0, phi=0.0, psi=0.0) -> np.ndarray:
    e = np.zeros((3,) + g.shape, np.complex128)
    lib().vo_incident(ctypes.byref(g.c()), theta, phi, psi, _p(e))
    return e


def matvec(g: Grid, green_full, eps, flags, x, conj=False) -> np.ndarray:
    green_full = np.ascontiguousarray(green_full, np.complex128)
    eps = np.ascontiguousarray(eps, np.complex128)
    flags = np.ascontiguousarray(flags, np.uint8)
    x = np.ascontiguousarray(x, np.complex128)
    out = np.zeros_like(x)
    rc = lib().vo_matvec(ctypes.byref(g.c()), _p(green_full), _p(eps), _p(flags, _up), _p(x), _p(out), int(conj))
    if rc:
        raise RuntimeError(f"vo_matvec failed ({rc})")
    return out


SOLVERS = {"cg": 1, "bicg": 2, "bicgstab": 3, "cors": 4, "bicorstab": 5}


def solve(g: Grid, green_full, eps, flags, einc, solver="bicgstab", thr=1e-3, maxit=0):
    green_full = np.ascontiguousarray(green_full, np.complex128)
    eps = np.ascontiguousarray(eps, np.complex128)
    flags = np.ascontiguousarray(flags, np.uint8)
    einc = np.ascontiguousarray(einc, np.complex128)
    x = np.zeros_like(einc)
    steps = ctypes.c_int(0)
    err = ctypes.c_double(0)
    rc = lib().vo_solve(ctypes.byref(g.c()), _p(green_full), _p(eps), _p(flags, _up), _p(einc),
                        SOLVERS[solver], thr, int(maxit), _p(x), ctypes.byref(steps), ctypes.byref(err))
    if rc:
        raise RuntimeError(f"vo_solve failed ({rc})")
    return x, steps.value, err.value


def farfield1(g: Grid, x, theta=0.0, phi=0.0, psi=0.0) -> float:
    x = np.ascontiguousarray(x, np.complex128)
    return lib().vo_farfield1(ctypes.byref(g.c()), _p(x), theta, phi, psi)


def absorption(g: Grid, x, eps, material, metal_label=2, active_label=3):
    x = np.ascontiguousarray(x, np.complex128)
    eps = np.ascontiguousarray(eps, np.complex128)
    material = np.ascontiguousarray(material, np.uint8)
    m = ctypes.c_double(0)
    a = ctypes.c_double(0)
    v = ctypes.c_double(0)
    lib().vo_absorption(ctypes.byref(g.c()), _p(x), _p(eps), _p(material, _up), metal_label, active_label,
                        ctypes.byref(m), ctypes.byref(a), ctypes.byref(v))
    return m.value, a.value, v.value


# ---------------------------------------------------------------------------
# reference build (oracle/_ref)
# ---------------------------------------------------------------------------

class Reference:
    """Drives the reference's own functions through the harness.

    ``eps_table`` holds the 4 entries of Real_EPR/Imag_EPR (Model.h:81-83),
    index 0 being the air dummy 1.1.
    """

    def __init__(self, g: Grid, eps_table, theta=0.0, phi=0.0, psi=0.0):
        self.g = g
        self.L = ref_lib()
        t = np.asarray(eps_table, np.complex128)
        assert t.shape == (4,)
        re = np.ascontiguousarray(t.real)
        im = np.ascontiguousarray(t.imag)
        rc = self.L.ref_setup(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.k0, _p(re), _p(im), theta, phi, psi)
        if rc:
            raise RuntimeError("ref_setup failed")

    def set_geometry(self, material, flags):
        m = np.ascontiguousarray(material, np.uint8)
        f = np.ascontiguousarray(flags, np.uint8)
        self.L.ref_set_geometry(_p(m, _up), _p(f[0], _up), _p(f[1], _up), _p(f[2], _up))

    def sphere_geometry(self, dia, box_l, box_w, box_h):
        self.L.ref_sphere_geometry(dia, box_l, box_w, box_h)

    def get_geometry(self):
        s = self.g.shape
        m = np.zeros(s, np.uint8)
        f = np.zeros((3,) + s, np.uint8)
        self.L.ref_get_geometry(_p(m, _up), _p(f[0], _up), _p(f[1], _up), _p(f[2], _up))
        return m, f

    def green(self):
        g = self.g
        out = np.zeros((2 * g.nx, 2 * g.ny, 2 * g.nz), np.complex128)
        self.L.ref_green(_p(out))
        return out

    def set_green(self, full):
        full = np.ascontiguousarray(full, np.complex128)
        self.L.ref_set_green(_p(full))

    def incident(self):
        e = np.zeros((3,) + self.g.shape, np.complex128)
        self.L.ref_incident(_p(e[0]), _p(e[1]), _p(e[2]))
        return e

    def set_incident(self, e):
        e = np.ascontiguousarray(e, np.complex128)
        self.L.ref_set_incident(_p(e[0]), _p(e[1]), _p(e[2]))

    def matvec(self, x, conj=False):
        x = np.ascontiguousarray(x, np.complex128)
        out = np.zeros_like(x)
        self.L.ref_matvec(_p(x), _p(out), int(conj))
        return out

    def solve(self, solver="bicgstab", thr=1e-3):
        x = np.zeros((3,) + self.g.shape, np.complex128)
        steps = ctypes.c_int(0)
        err = ctypes.c_double(0)
        rc = self.L.ref_solve(SOLVERS[solver], thr, _p(x), ctypes.byref(steps), ctypes.byref(err))
        if rc:
            raise RuntimeError(f"ref_solve failed ({rc})")
        return x, steps.value, err.value

    def set_current(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        self.L.ref_set_current(_p(x))

    def farfield1(self):
        v = ctypes.c_double(0)
        self.L.ref_farfield1(ctypes.byref(v))
        return v.value

    def farfield2(self):
        rt, rp = np.zeros(181), np.zeros(181)
        self.L.ref_farfield2(_p(rt), _p(rp))
        return rt, rp

    def nearfield(self):
        e = ctypes.c_double(0)
        m = ctypes.c_double(0)
        a = ctypes.c_double(0)
        self.L.ref_nearfield(ctypes.byref(e), ctypes.byref(m), ctypes.byref(a))
        return e.value, m.value, a.value

    def row(self, which, x):
        """X/Y/Z_FFT (which 0..2) or their _Conjugate twins (3..5), field from zero."""
        x = np.ascontiguousarray(x, np.complex128)
        out = np.zeros(self.g.shape, np.complex128)
        self.L.ref_row(int(which), _p(x), _p(out))
        return out

    def block(self, kind, src, fld, conj, x):
        """L_DC_Dq (kind 0), L_Dq (1) or L??_DO (2) on component src of x after Current_Expansion."""
        x = np.ascontiguousarray(x, np.complex128)
        out = np.zeros(self.g.shape, np.complex128)
        self.L.ref_block(int(kind), int(src), int(fld), int(conj), _p(x), _p(out))
        return out

    def reset(self, v, flag):
        v = np.array(v, dtype=np.complex128, order="C", copy=True)
        self.L.ref_reset(_p(v), int(flag))
        return v

    def set_cross_section(self, cs):
        self.L.ref_set_cross_section(cs)

    def release(self):
        self.L.ref_release()


def fft3d(x, sign=-1) -> np.ndarray:
    """The oracle's unnormalised 3D transform (sign -1 forward, +1 backward)."""
    L = lib()
    L.vo_fft3d.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    y = np.ascontiguousarray(x, np.complex128).copy()
    n0, n1, n2 = y.shape
    if L.vo_fft3d(_p(y), n0, n1, n2, int(sign)):
        raise RuntimeError("vo_fft3d failed")
    return y


def time_block(g: Grid, use_reference: bool = True) -> dict:
    """Seconds of one L_DC_Dq block (fft.h:41-127) at grid g: two (2N)^3 FFTs,
    the spectral multiply and the crop, on the reference build when present,
    else on the restatement.  The unit of the CPU baseline."""
    import time
    n = g.shape
    pad = np.zeros((2 * n[0], 2 * n[1], 2 * n[2]), np.complex128)
    pad[: n[0] - 1, : n[1], : n[2]] = 1.0 + 0.5j
    fld = np.zeros(n, np.complex128)
    if use_reference and ref_available():
        R = Reference(g, np.array([1.1, 2.0, 2.0, 2.0]))
        R.L.ref_green(None)
        t = time.perf_counter()
        R.L.ref_time_block(_p(pad), _p(fld))
        dt = time.perf_counter() - t
        R.release()
        return {"seconds": dt, "kind": "reference"}
    G = green(g)
    t = time.perf_counter()
    lib().vo_block(ctypes.byref(g.c()), _p(G), _p(pad), _p(fld))
    return {"seconds": time.perf_counter() - t, "kind": "port"}

