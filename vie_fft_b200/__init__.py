"""vie_fft_b200 -- B200-native VIE-FFT operator and Krylov solvers.

Python binding of the C ABI in ``include/vie_b200.h`` (``_lib/libvie_b200.so``).
The library is the product; this module only marshals arrays.  There is no
CPU fallback: if the CUDA library is missing or no GPU is present, every
compute call raises.

Arrays use the reference layout: numpy ``complex128`` of shape ``(3, nx, ny, nz)``
for current / field vectors, ``(nx, ny, nz)`` for per-voxel data, C order.
Permittivities use the reference sign convention (lossy media have negative
imaginary parts; see ``geometry.to_reference_eps``).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libvie_b200.so")

VIE_OK = 0
VIE_ERR_ARG = 1
VIE_ERR_ALLOC = 2
VIE_ERR_CUDA = 3
VIE_ERR_BREAKDOWN = 4
VIE_ERR_MAXIT = 5
VIE_ERR_NAN = 6
VIE_ERR_STATE = 7
VIE_ERR_TIMEOUT = 8
VIE_ERR_NODEVICE = 9

SOLVERS = {"cg": 1, "bicg": 2, "bicgstab": 3, "cors": 4, "bicorstab": 5}
PART_GREEN, PART_DIAG, PART_MASK, PART_ALL = 1, 2, 4, 7
PREC_FP64 = 0
PREC_MIXED = 1

_lib = None


class VieError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class VieGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("k0", ctypes.c_double), ("device", ctypes.c_int)]


class VieSolveParams(ctypes.Structure):
    _fields_ = [("solver", ctypes.c_int), ("precision", ctypes.c_int), ("tol", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("inner_tol", ctypes.c_double), ("max_outer", ctypes.c_int),
                ("verbose", ctypes.c_int), ("true_residual", ctypes.c_int)]


class ViePrimitive(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("label", ctypes.c_int), ("parent", ctypes.c_int), ("pad", ctypes.c_int),
                ("c", ctypes.c_double * 3), ("r", ctypes.c_double), ("h", ctypes.c_double * 3)]


PRIM_SPHERE, PRIM_SPHERE_F32, PRIM_BOX = 1, 2, 3


class VieSolveInfo(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int), ("iterations", ctypes.c_int), ("outer", ctypes.c_int),
                ("matvecs_fp64", ctypes.c_int), ("matvecs_fp32", ctypes.c_int), ("relres", ctypes.c_double),
                ("true_relres", ctypes.c_double), ("seconds", ctypes.c_double), ("graph_loops", ctypes.c_int),
                ("status", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_ubyte)
_vp = ctypes.c_void_p


def lib():
    """Load the CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m vie_fft_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        L.vie_create.argtypes = [P(VieGrid), P(_vp)]
        L.vie_destroy.argtypes = [_vp]
        L.vie_destroy.restype = None
        L.vie_last_error.argtypes = [_vp]
        L.vie_last_error.restype = ctypes.c_char_p
        L.vie_status_string.argtypes = [ctypes.c_int]
        L.vie_status_string.restype = ctypes.c_char_p
        L.vie_version.restype = ctypes.c_char_p
        L.vie_launch_count.restype = ctypes.c_longlong
        L.vie_set_material.argtypes = [_vp, _up, _dp, _dp, ctypes.c_int]
        L.vie_set_eps.argtypes = [_vp, _dp]
        L.vie_set_flags.argtypes = [_vp, _up, _up, _up]
        L.vie_set_geometry_scene.argtypes = [_vp, P(ViePrimitive), ctypes.c_int, _dp, _dp, ctypes.c_int, _up]
        L.vie_green.argtypes = [_vp]
        L.vie_green_spectrum.argtypes = [_vp, _dp]
        L.vie_incident.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp]
        L.vie_set_rhs.argtypes = [_vp, _dp]
        L.vie_matvec.argtypes = [_vp, _dp, _dp, ctypes.c_int]
        L.vie_apply.argtypes = [_vp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.vie_reset.argtypes = [_vp, _dp, ctypes.c_int]
        L.vie_matvec_dev.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int]
        L.vie_solve.argtypes = [_vp, P(VieSolveParams), _dp, P(VieSolveInfo)]
        L.vie_solve_batch.argtypes = [P(_vp), ctypes.c_int, P(VieSolveParams), P(VieSolveInfo)]
        L.vie_farfield1.argtypes = [_vp] + [ctypes.c_double] * 3 + [_dp]
        L.vie_farfield2.argtypes = [_vp, ctypes.c_double, _dp, _dp]
        L.vie_nearfield.argtypes = [_vp, _up, _dp, _dp, _dp]
        L.vie_autotune.argtypes = [_vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.vie_power_grad.argtypes = [_vp, _up, P(VieSolveParams), _dp, _dp, P(VieSolveInfo), P(VieSolveInfo)]
        L.vie_get_solution.argtypes = [_vp, _dp]
        L.vie_set_solution.argtypes = [_vp, _dp]
        L.vie_residual.argtypes = [_vp, _dp]
        L.vie_solution_device.argtypes = [_vp, P(_vp)]
        L.vie_rhs_device.argtypes = [_vp, P(_vp)]
        L.vie_sync.argtypes = [_vp]
        L.vie_stream.argtypes = [_vp, P(_vp)]
        _lib = L
    return _lib


def _p(arr, kind=_dp):
    return arr.ctypes.data_as(kind)


def _c128(x, shape=None):
    a = np.ascontiguousarray(x, dtype=np.complex128)
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"expected shape {tuple(shape)}, got {a.shape}")
    return a


@dataclass
class SolveResult:
    x: np.ndarray | None
    info: dict
    status: int


class Context:
    """One grid on one GPU (wraps ``vie_ctx``)."""

    def __init__(self, nx, ny, nz, dx, dy, dz, k0, device=0):
        self._L = lib()
        self.shape = (int(nx), int(ny), int(nz))
        self.a = int(nx) * int(ny) * int(nz)
        self.device = int(device)
        g = VieGrid(int(nx), int(ny), int(nz), float(dx), float(dy), float(dz), float(k0), int(device))
        h = _vp()
        rc = self._L.vie_create(ctypes.byref(g), ctypes.byref(h))
        if rc != VIE_OK:
            raise VieError(rc, self._L.vie_status_string(rc).decode())
        self._h = h

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.vie_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc, allow=()):
        if rc != VIE_OK and rc not in allow:
            raise VieError(rc, self._L.vie_last_error(self._h).decode())
        return rc

    # ------------------------------------------------------------------
    def set_material(self, material, eps_table):
        m = np.ascontiguousarray(material, np.uint8)
        t = np.asarray(eps_table, np.complex128)
        re = np.ascontiguousarray(t.real)
        im = np.ascontiguousarray(t.imag)
        self._check(self._L.vie_set_material(self._h, _p(m, _up), _p(re), _p(im), len(t)))

    def set_eps(self, eps):
        e = _c128(eps, self.shape)
        self._check(self._L.vie_set_eps(self._h, _p(e)))

    def set_scene(self, prims, eps_table):
        """Material labels and edge flags from an analytic scene, evaluated on the
        GPU (``vie_set_geometry_scene``).  prims: dicts with kind (PRIM_*), label,
        c (centre), r (sphere radius), h (box half-widths), parent (-1).
        Returns the material labels (nx, ny, nz) uint8."""
        arr = (ViePrimitive * max(len(prims), 1))()
        for q, p in enumerate(prims):
            arr[q].kind = int(p["kind"])
            arr[q].label = int(p["label"])
            arr[q].parent = int(p.get("parent", -1))
            for t in range(3):
                arr[q].c[t] = float(p.get("c", (0, 0, 0))[t])
                arr[q].h[t] = float(p.get("h", (0, 0, 0))[t])
            arr[q].r = float(p.get("r", 0.0))
        t = np.asarray(eps_table, np.complex128)
        re, im = np.ascontiguousarray(t.real), np.ascontiguousarray(t.imag)
        mat = np.zeros(self.shape, np.uint8)
        ptr = ctypes.cast(arr, ctypes.POINTER(ViePrimitive))
        self._check(self._L.vie_set_geometry_scene(self._h, ptr, len(prims), _p(re), _p(im), len(t), _p(mat, _up)))
        return mat

    def set_flags(self, flags):
        f = np.ascontiguousarray(flags, np.uint8)
        if f.shape != (3,) + self.shape:
            raise ValueError("flags must have shape (3, nx, ny, nz)")
        self._check(self._L.vie_set_flags(self._h, _p(f[0], _up), _p(f[1], _up), _p(f[2], _up)))

    def green(self):
        self._check(self._L.vie_green(self._h))

    def green_spectrum(self):
        nx, ny, nz = self.shape
        out = np.zeros((2 * nx, 2 * ny, 2 * nz), np.complex128)
        self._check(self._L.vie_green_spectrum(self._h, _p(out)))
        return out

    def incident(self, theta=0.0, phi=0.0, psi=0.0, copy=True):
        out = np.zeros((3,) + self.shape, np.complex128) if copy else None
        self._check(self._L.vie_incident(self._h, float(theta), float(phi), float(psi),
                                         _p(out) if copy else None))
        return out

    def set_rhs(self, e):
        e = _c128(e, (3,) + self.shape)
        self._check(self._L.vie_set_rhs(self._h, _p(e)))

    def matvec(self, x, conj=False):
        x = _c128(x, (3,) + self.shape)
        y = np.zeros_like(x)
        self._check(self._L.vie_matvec(self._h, _p(x), _p(y), int(bool(conj))))
        return y

    def apply(self, x, conj=False, parts=7):
        """Selected parts of the operator (PART_GREEN | PART_DIAG | PART_MASK)."""
        x = _c128(x, (3,) + self.shape)
        y = np.zeros_like(x)
        self._check(self._L.vie_apply(self._h, _p(x), _p(y), int(bool(conj)), int(parts)))
        return y

    def reset(self, v, comp):
        """Current_Reset of one component (in place on a copy, returned)."""
        v = np.array(v, dtype=np.complex128, order="C", copy=True)
        self._check(self._L.vie_reset(self._h, _p(v), int(comp)))
        return v

    def matvec_dev(self, x_ptr: int, y_ptr: int, conj=False, precision=PREC_FP64):
        """Device-pointer operator application (e.g. torch tensor data_ptr())."""
        self._check(self._L.vie_matvec_dev(self._h, _vp(x_ptr), _vp(y_ptr), int(bool(conj)), int(precision)))

    def solve(self, solver="bicgstab", tol=1e-3, precision=PREC_FP64, max_iter=0, inner_tol=0.0, max_outer=0,
              verbose=False, copy=True, allow_maxit=False, true_residual=True, out=None):
        prm = VieSolveParams(SOLVERS[solver] if isinstance(solver, str) else int(solver), int(precision),
                             float(tol), int(max_iter), float(inner_tol), int(max_outer), int(bool(verbose)),
                             int(bool(true_residual)))
        info = VieSolveInfo()
        x = out if out is not None else (np.zeros((3,) + self.shape, np.complex128) if copy else None)
        rc = self._L.vie_solve(self._h, ctypes.byref(prm), _p(x) if copy else None, ctypes.byref(info))
        self._check(rc, allow=(VIE_ERR_MAXIT,) if allow_maxit else ())
        return SolveResult(x, info.as_dict(), rc)

    def power_grad(self, edge_mask, solver="bicgstab", tol=1e-8, precision=PREC_FP64, grad=True, max_iter=0,
                   inner_tol=0.0):
        """Absorbed power P in the edges of ``edge_mask`` (uint8 per voxel, bit f =
        the f-edge; see post.edge_mask) and, with ``grad``, dP/dRe(eps) + i dP/dIm(eps)
        per voxel for the permittivity as given to set_eps / set_material
        (``vie_power_grad``: forward solve + one adjoint solve).
        Returns (P, grad (nx, ny, nz) complex or None, forward info, adjoint info)."""
        m = np.ascontiguousarray(edge_mask, np.uint8)
        if m.shape != self.shape:
            raise ValueError(f"edge_mask must have shape {self.shape}")
        prm = VieSolveParams(SOLVERS[solver] if isinstance(solver, str) else int(solver), int(precision), float(tol),
                             int(max_iter), float(inner_tol), 0, 0, 0)
        pw = ctypes.c_double(0.0)
        g = np.zeros(self.shape, np.complex128) if grad else None
        fi, ai = VieSolveInfo(), VieSolveInfo()
        self._check(self._L.vie_power_grad(self._h, _p(m, _up), ctypes.byref(prm), ctypes.byref(pw),
                                           _p(g) if grad else None, ctypes.byref(fi), ctypes.byref(ai)))
        return pw.value, g, fi.as_dict(), ai.as_dict()

    # -- post-processing of the last solution on the GPU ------------------
    def farfield1(self, theta=0.0, phi=0.0, psi=0.0) -> float:
        """Forward_RCS of FarField1 (NearFar.h:16-109)."""
        v = ctypes.c_double(0)
        self._check(self._L.vie_farfield1(self._h, float(theta), float(phi), float(psi), ctypes.byref(v)))
        return v.value

    def farfield2(self, phi=0.0):
        """(RCS_Theta[181], RCS_Phi[181]) in dB of FarField2 (NearFar.h:302-477)."""
        rt, rp = np.zeros(181), np.zeros(181)
        self._check(self._L.vie_farfield2(self._h, float(phi), _p(rt), _p(rp)))
        return rt, rp

    def nearfield(self, material):
        """(Ene_Metal, Ene_Active, Absorb_Volume) of NearField (NearFar.h:186-250)."""
        m = np.ascontiguousarray(material, np.uint8)
        if m.shape != self.shape:
            raise ValueError(f"material must have shape {self.shape}")
        out = [ctypes.c_double(0) for _ in range(3)]
        self._check(self._L.vie_nearfield(self._h, _p(m, _up), *[ctypes.byref(o) for o in out]))
        return tuple(o.value for o in out)

    def autotune(self, fp64=True, fp32=True, force=False) -> str:
        """Time the FFT schedules of this grid and rebuild the operators with the
        fastest (``vie_autotune``); returns the one-line report."""
        flags = (1 if fp64 else 0) | (2 if fp32 else 0) | (4 if force else 0)
        buf = ctypes.create_string_buffer(1024)
        self._check(self._L.vie_autotune(self._h, flags, buf, len(buf)))
        return buf.value.decode()

    def residual(self) -> float:
        """||b - A x|| / ||b|| of the last solution, in FP64."""
        v = ctypes.c_double(0)
        self._check(self._L.vie_residual(self._h, ctypes.byref(v)))
        return v.value

    def solution(self):
        x = np.zeros((3,) + self.shape, np.complex128)
        self._check(self._L.vie_get_solution(self._h, _p(x)))
        return x

    def set_solution(self, x):
        """Make x (3, nx, ny, nz) the context's solution (for post-processing)."""
        xx = _c128(x, (3,) + self.shape)
        self._check(self._L.vie_set_solution(self._h, _p(xx)))

    def solution_ptr(self) -> int:
        p = _vp()
        self._check(self._L.vie_solution_device(self._h, ctypes.byref(p)))
        return p.value

    def rhs_ptr(self) -> int:
        p = _vp()
        self._check(self._L.vie_rhs_device(self._h, ctypes.byref(p)))
        return p.value

    def stream_ptr(self) -> int:
        """The context's cudaStream_t as an integer (torch.cuda.ExternalStream)."""
        p = _vp()
        self._check(self._L.vie_stream(self._h, ctypes.byref(p)))
        return p.value

    def sync(self):
        self._check(self._L.vie_sync(self._h))


def solve_batch(contexts, solver="bicgstab", tol=1e-3, precision=PREC_FP64, max_iter=0, inner_tol=0.0,
                verbose=False, copy=True, allow_maxit=False, raise_errors=True):
    """Solve every context's system in one CUDA graph launch (``vie_solve_batch``).

    The contexts may have different grids, materials, wavelengths and
    right-hand sides; they must be distinct and on one GPU.  Returns one
    SolveResult per context (``x`` copied back when ``copy``; ``status`` the
    instance's own).  With ``raise_errors=False`` instance failures (cap,
    breakdown) are only reported in the results."""
    ctxs = list(contexts)
    n = len(ctxs)
    if n == 0:
        return []
    L = ctxs[0]._L
    prm = VieSolveParams(SOLVERS[solver] if isinstance(solver, str) else int(solver), int(precision), float(tol),
                         int(max_iter), float(inner_tol), 0, int(bool(verbose)), 0)
    infos = (VieSolveInfo * n)()
    handles = (_vp * n)(*[c._h for c in ctxs])
    rc = L.vie_solve_batch(handles, n, ctypes.byref(prm), infos)
    instance_failure = rc in (VIE_ERR_MAXIT, VIE_ERR_BREAKDOWN) and any(infos[i].status for i in range(n))
    if rc != VIE_OK and not (instance_failure and not raise_errors) and not (rc == VIE_ERR_MAXIT and allow_maxit):
        bad = next((c for c in ctxs if L.vie_last_error(c._h)), ctxs[0])
        raise VieError(rc, L.vie_last_error(bad._h).decode(errors="replace"))
    return [SolveResult(c.solution() if copy else None, infos[i].as_dict(), int(infos[i].status))
            for i, c in enumerate(ctxs)]


def launch_count() -> int:
    """Kernels launched by the library in this process so far."""
    return int(lib().vie_launch_count())


def version() -> str:
    return lib().vie_version().decode()
