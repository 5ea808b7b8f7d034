"""CUDA operator parity: Green spectrum, incident field, A x and A^H x in FP64
and FP32 against the reference's outputs (golden fixtures from oracle/_ref)
and the oracle restatement, plus size-independent properties at full sizes."""
import ctypes
import os

import numpy as np
import pytest

import vie_fft_b200 as V
from oracle import oracle as O
from tests.golden import make_golden as MG
from vie_fft_b200 import geometry as GEO

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

# tolerances: FP64 results are compared relative to the largest magnitude
FP64_TOL = 1e-12
FP32_TOL = 2e-5


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def make_ctx(shape, d, k0, material, flags, table=None, eps=None):
    c = V.Context(*shape, *d, k0)
    c.set_flags(flags)
    if eps is not None:
        c.set_eps(eps)
    else:
        c.set_material(material, table)
    c.green()
    return c


@pytest.mark.parametrize("idx", range(len(MG.SMALL)))
def test_small_cases_match_reference(idx):
    gold = np.load(os.path.join(GOLD, "small_ops.npz"))
    shape, d, k0, ang, mat, flags, x = MG.small_inputs(idx)
    with make_ctx(shape, d, k0, mat, flags, MG.EPS_TABLE) as c:
        assert rel(c.green_spectrum(), gold[f"green{idx}"]) < 1e-13
        assert rel(c.incident(*ang), gold[f"inc{idx}"]) < 1e-13
        assert rel(c.matvec(x, conj=False), gold[f"ax{idx}"]) < FP64_TOL
        assert rel(c.matvec(x, conj=True), gold[f"ahx{idx}"]) < FP64_TOL


# shapes cover the generic kernels (odd and prime lengths) and every length
# with register four-step kernels: 16..256 powers of two and the mixed-radix
# 24 (8x3), 40 (8x5), 48 (8x6), 56 (8x7), 72 (8x9), 80 (16x5), 88 (8x11), 96 (16x6),
# 112 (16x7), 120 (8x15), 144 (16x9), 160 (16x10), 176 (16x11), 192 (16x12)
@pytest.mark.parametrize("shape", [(24, 20, 16), (31, 17, 13), (48, 40, 56), (9, 7, 5), (2, 2, 2), (16, 3, 64),
                                   (72, 88, 16), (96, 24, 80), (32, 72, 40), (112, 120, 16), (144, 16, 160),
                                   (176, 16, 192)])
def test_matvec_fp64_matches_oracle(shape):
    rng = np.random.default_rng(sum(shape))
    d = (0.01, 0.012, 0.011)
    k0 = GEO.k0_of(530.0)
    table = np.array([1.1, 2.4 - 0.05j, -8.5 - 0.3j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    g = O.Grid(*shape, *d, k0)
    G = O.green(g)
    with make_ctx(shape, d, k0, mat, flags, table) as c:
        for conj in (False, True):
            assert rel(c.matvec(x, conj), O.matvec(g, G, table[mat], flags, x, conj)) < FP64_TOL


def _torch():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


@pytest.mark.parametrize("shape", [(24, 20, 16), (31, 17, 13), (48, 40, 56), (72, 88, 16), (96, 24, 80),
                                   (112, 120, 16), (176, 16, 192)])
def test_matvec_fp32_matches_oracle(shape):
    torch = _torch()
    rng = np.random.default_rng(5)
    d = (0.01, 0.01, 0.01)
    k0 = GEO.k0_of(450.0)
    table = np.array([1.1, 2.4 - 0.05j, -4.4 - 0.2j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    g = O.Grid(*shape, *d, k0)
    ref = O.matvec(g, O.green(g), table[mat], flags, x, False)
    with make_ctx(shape, d, k0, mat, flags, table) as c:
        xt = torch.from_numpy(x.astype(np.complex64)).cuda()
        yt = torch.zeros_like(xt)
        torch.cuda.synchronize()
        c.matvec_dev(xt.data_ptr(), yt.data_ptr(), conj=False, precision=V.PREC_MIXED)
        c.sync()
        assert rel(yt.cpu().numpy(), ref) < FP32_TOL
        refh = O.matvec(g, O.green(g), table[mat], flags, x, True)
        c.matvec_dev(xt.data_ptr(), yt.data_ptr(), conj=True, precision=V.PREC_MIXED)
        c.sync()
        assert rel(yt.cpu().numpy(), refh) < FP32_TOL


# the lengths the 128^3 and 256^3 grids run (register plans 16x8 and 16x16) in
# each axis position: the x pass (both pencil tiles), the y passes with their
# TMA-staged tiles (at 256 the inverse-y tile is two boxes of the maximum
# height, 256 rows) and the z row passes, each against the oracle
THIN = [(256, 6, 5), (5, 256, 6), (6, 5, 256), (128, 7, 9), (9, 128, 7), (7, 9, 128)]


@pytest.mark.parametrize("shape", THIN)
def test_lengths_128_256_match_oracle(shape, monkeypatch):
    """A x and A^H x in FP64 (1e-12) and FP32 (2e-5, default and half x tile)
    against the oracle (CG_Iteration.h:131-173, fft.h:41-127, 224-309)."""
    torch = _torch()
    rng = np.random.default_rng(sum(shape) + 7)
    d = (0.01, 0.012, 0.011)
    k0 = GEO.k0_of(530.0)
    table = np.array([1.1, 2.4 - 0.05j, -8.5 - 0.3j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    g = O.Grid(*shape, *d, k0)
    G = O.green(g)
    ref = [O.matvec(g, G, table[mat], flags, x, conj) for conj in (False, True)]
    for xtile in ("0", "1"):
        monkeypatch.setenv("VIE_XTILE", xtile)
        with make_ctx(shape, d, k0, mat, flags, table) as c:
            for conj in (False, True):
                assert rel(c.matvec(x, conj), ref[conj]) < FP64_TOL, (xtile, conj)
            xt = torch.from_numpy(x.astype(np.complex64)).cuda()
            for conj in (False, True):
                yt = torch.zeros_like(xt)
                torch.cuda.synchronize()
                c.matvec_dev(xt.data_ptr(), yt.data_ptr(), conj=conj, precision=V.PREC_MIXED)
                c.sync()
                assert rel(yt.cpu().numpy(), ref[conj]) < FP32_TOL, (xtile, conj)


def test_green_block_256_matches_reference():
    """One full-size self-term block, L_DC_Dq (fft.h:41-127) on the x current of
    a seeded 256^3 field (two 512^3 transforms), against the reference's own
    function built in place (oracle/_ref), else against the oracle restatement.
    The GPU computes the block as the Green part of the operator on a vector
    whose only non-zero component is x (the call dropin/fft.h makes).  On one
    host core the reference takes about a minute for its Green's function and
    the block; the GPU side takes under a second."""
    n = (256, 256, 256)
    d = (0.01, 0.01, 0.01)
    k0 = GEO.k0_of(550.0)
    table = np.array([1.1, 2.4 - 0.05j, 3.8 - 0.6j, -8.5 - 0.3j])
    rng = np.random.default_rng(256)
    x = np.zeros((3,) + n, np.complex128)
    x[0] = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    g = O.Grid(*n, *d, k0)
    if O.ref_available():
        R = O.Reference(g, table)
        R.L.ref_green(None)
        ref = np.zeros(n, np.complex128)
        assert R.L.ref_block(0, 0, 0, 0, O._p(x), O._p(ref)) == 0
        R.release()
    else:
        G = O.green(g)
        pad = np.zeros(tuple(2 * v for v in n), np.complex128)
        pad[: n[0] - 1, : n[1], : n[2]] = x[0, : n[0] - 1]
        ref = np.zeros(n, np.complex128)
        O.lib().vo_block(ctypes.byref(g.c()), O._p(G), O._p(pad), O._p(ref))
        del G, pad
    mat = np.ones(n, np.uint8)
    flags = np.ones((3,) + n, np.uint8)
    with make_ctx(n, d, k0, mat, flags, table) as c:
        y = c.apply(x, conj=False, parts=V.PART_GREEN)
    assert rel(y[0], ref) < FP64_TOL


# y lengths with register kernels; 2 nz not a multiple of the pencil tile width
# (16 columns FP32, 8 FP64) makes the last TMA box run past the row end
@pytest.mark.parametrize("shape", [(24, 40, 13), (8, 64, 20), (12, 120, 3), (6, 256, 9)])
def test_tma_staged_y_passes_match_plain_loads(shape, monkeypatch):
    """The y passes with their tiles staged by TMA compute exactly what the
    plain-load kernels compute: bit-identical A x and A^H x in FP64 and FP32."""
    torch = _torch()
    rng = np.random.default_rng(sum(shape))
    d = (0.01, 0.01, 0.01)
    k0 = GEO.k0_of(500.0)
    table = np.array([1.1, 2.4 - 0.05j, -4.4 - 0.2j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    out = {}
    for tma in ("1", "0"):
        monkeypatch.setenv("VIE_TMA", tma)
        with make_ctx(shape, d, k0, mat, flags, table) as c:
            r = [c.matvec(x, conj) for conj in (False, True)]
            xt = torch.from_numpy(x.astype(np.complex64)).cuda()
            for conj in (False, True):
                yt = torch.zeros_like(xt)
                torch.cuda.synchronize()
                c.matvec_dev(xt.data_ptr(), yt.data_ptr(), conj=conj, precision=V.PREC_MIXED)
                c.sync()
                r.append(yt.cpu().numpy())
        out[tma] = r
    for a, b in zip(out["1"], out["0"]):
        np.testing.assert_array_equal(a, b)


# fast z lengths; nx ny not a multiple of the rows per block (16 FP32, 8 FP64)
@pytest.mark.parametrize("shape", [(13, 7, 64), (5, 9, 24), (3, 11, 256)])
def test_bulk_staged_z_passes_match_element_loads(shape, monkeypatch):
    """The z passes with their rows staged by bulk copies compute exactly what
    the element-load kernels compute (FP64 and FP32, A x and A^H x), and a
    source vector that is not 16-byte aligned falls back to element loads."""
    torch = _torch()
    rng = np.random.default_rng(sum(shape) + 1)
    d = (0.01, 0.01, 0.01)
    k0 = GEO.k0_of(500.0)
    table = np.array([1.1, 2.4 - 0.05j, -4.4 - 0.2j, 3.8 - 0.6j])
    mat = rng.integers(0, 4, size=shape).astype(np.uint8)
    flags = rng.integers(0, 2, size=(3,) + shape).astype(np.uint8)
    x = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    n = x.size
    out = {}
    for zs in ("1", "0"):
        monkeypatch.setenv("VIE_ZSTAGE", zs)
        with make_ctx(shape, d, k0, mat, flags, table) as c:
            r = [c.matvec(x, conj) for conj in (False, True)]
            buf = torch.zeros(n + 1, dtype=torch.complex64, device="cuda")
            for off in (0, 1):  # offset 1: 8 bytes, not 16-byte aligned
                xt = buf[off:off + n]
                xt.copy_(torch.from_numpy(x.astype(np.complex64).ravel()))
                yt = torch.zeros(n, dtype=torch.complex64, device="cuda")
                torch.cuda.synchronize()
                c.matvec_dev(xt.data_ptr(), yt.data_ptr(), conj=False, precision=V.PREC_MIXED)
                c.sync()
                r.append(yt.cpu().numpy().reshape(x.shape))
        out[zs] = r
    for a, b in zip(out["1"], out["0"]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(out["1"][2], out["1"][3])


def test_adjoint_and_symmetry_identities_full_size():
    """<y, A x> = <A^H y, x> and, for cubic voxels on flagged edges, y^T A x = x^T A y."""
    w = GEO.solar_cell(shape=(96, 96, 48), nspheres=4, radius_nm=8.0, spacer_nm=8.0, active_nm=24.0,
                       sphere_z_nm=(16.0, 24.0))
    rng = np.random.default_rng(11)
    mask = w.flags.astype(bool)
    x = (rng.standard_normal((3,) + w.shape) + 1j * rng.standard_normal((3,) + w.shape)) * mask
    y = (rng.standard_normal((3,) + w.shape) + 1j * rng.standard_normal((3,) + w.shape)) * mask
    with make_ctx(w.shape, w.d, w.k0, w.material, w.flags, w.eps_table) as c:
        Ax, Ay, AHy = c.matvec(x), c.matvec(y), c.matvec(y, conj=True)
    lhs = np.vdot(y, Ax)
    assert abs(lhs - np.vdot(AHy, x)) < 1e-12 * np.linalg.norm(y) * np.linalg.norm(Ax)
    assert abs(np.sum(y * Ax) - np.sum(x * Ay)) < 1e-12 * np.linalg.norm(y) * np.linalg.norm(Ax)


def test_linearity_and_fp32_consistency_128():
    torch = _torch()
    w = GEO.sphere_cluster(n=128, count=40, seed=2)
    rng = np.random.default_rng(12)
    x = rng.standard_normal((3,) + w.shape) + 1j * rng.standard_normal((3,) + w.shape)
    y = rng.standard_normal((3,) + w.shape) + 1j * rng.standard_normal((3,) + w.shape)
    with make_ctx(w.shape, w.d, w.k0, w.material, w.flags, w.eps_table) as c:
        Ax, Ay = c.matvec(x), c.matvec(y)
        al, be = 0.3 - 1.2j, -0.7 + 0.4j
        assert rel(c.matvec(al * x + be * y), al * Ax + be * Ay) < 1e-12
        xt = torch.from_numpy(x.astype(np.complex64)).cuda()
        yt = torch.zeros_like(xt)
        torch.cuda.synchronize()
        c.matvec_dev(xt.data_ptr(), yt.data_ptr(), precision=V.PREC_MIXED)
        c.sync()
        assert rel(yt.cpu().numpy(), Ax) < FP32_TOL


def test_operator_state_errors():
    with V.Context(8, 8, 8, 0.01, 0.01, 0.01, 1.0) as c:
        with pytest.raises(V.VieError) as e:
            c.matvec(np.zeros((3, 8, 8, 8)))
        assert e.value.status == V.VIE_ERR_STATE
        with pytest.raises(V.VieError) as e:
            c.set_material(np.full((8, 8, 8), 5, np.uint8), [1.1, 2.0])
        assert e.value.status == V.VIE_ERR_ARG
        with pytest.raises(V.VieError) as e:
            c.set_eps(np.ones((8, 8, 8), complex))  # eps = 1 has no inverse contrast
        assert e.value.status == V.VIE_ERR_ARG
