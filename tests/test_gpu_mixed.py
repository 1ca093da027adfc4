"""Mixed precision through the C ABI: the int8-slice and split-TF32 tcgen05
complex GEMMs, the FP32 LU with FP64 residual refinement, and whole solves in
RCWA_PREC_MIXED against the FP64 form and the oracle.

Tolerances:
* int8-slice GEMM: d signed 7-bit digits per operand under power-of-two
  row / column scales, exact int32 accumulation: error ~ 2^(-7d) of
  max|A| max|B| sqrt(k) -- checked at 1e-7 / 1e-9 / 1e-11 for d = 4 / 5 / 6.
* split-TF32 GEMM: TF32 hi + lo per operand (2^-22), three products in the
  tensor core's FP32 accumulation -- checked at 1e-5 of max|A| max|B| k.
* LU: one FP64 refinement sweep after the FP32 solve leaves about
  (cond * 2^-24)^2 relative error -- checked at 1e-10 for well-conditioned
  systems; two sweeps reach FP64 rounding (1e-13).
* Solves: the mixed form must stay within |dR|, |dT| <= 1e-6 (absolute, per
  order and for the totals) of the FP64 form, which itself matches the oracle
  to 1e-10.
"""
import numpy as np
import pytest

from rcwa_b200 import configs as C
from helpers import oracle_solve

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6


@pytest.fixture(scope="module")
def ctx():
    from rcwa_b200 import lib as L
    c = L.Context(0)
    yield c
    c.close()


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


GEMM_SHAPES = [(1, 1, 1, 1), (8, 8, 8, 1), (64, 128, 16, 1), (70, 130, 50, 2), (128, 256, 100, 1),
               (450, 450, 450, 1), (300, 129, 1000, 1), (129, 49, 33, 3)]


@pytest.mark.parametrize("digits,tol", [(4, 1e-7), (5, 1e-9), (6, 1e-11)])
@pytest.mark.parametrize("m,n,k,b", GEMM_SHAPES)
def test_int8_slice_gemm_matches_fp64(ctx, m, n, k, b, digits, tol):
    from rcwa_b200 import lib as L
    rng = np.random.default_rng(m * 131 + n * 7 + k)
    A, B = _rand(rng, b, m, k), _rand(rng, b, k, n)
    ref = A @ B
    ctx.set_mixed(L.MIXED_LAYER_GEMM | L.MIXED_STAR_GEMM, 1, digits)
    try:
        got = ctx.gemm(A, B, precision=L.PREC_MIXED)
    finally:
        ctx.set_mixed(L.MIXED_LAYER_GEMM | L.MIXED_STAR_GEMM, 1, 5)
    scale = np.abs(A).max() * np.abs(B).max() * np.sqrt(k)
    err = np.abs(got - ref).max() / scale
    assert err < tol, err
    # it is not the FP64 kernel: the error is above FP64 rounding
    if k >= 16 and digits < 6:
        assert np.abs(got - ref).max() > 1e-15 * scale


def test_int8_slice_gemm_scaled_rows_and_nan(ctx):
    """Rows and columns of very different magnitude keep their relative
    accuracy (each has its own power-of-two scale); a NaN spreads over its
    row only, as in an FP64 product."""
    from rcwa_b200 import lib as L
    rng = np.random.default_rng(12)
    A = _rand(rng, 1, 90, 60) * np.logspace(-30, 30, 90)[None, :, None]
    B = _rand(rng, 1, 60, 70) * np.logspace(20, -20, 70)[None, None, :]
    ref = A @ B
    got = ctx.gemm(A, B, precision=L.PREC_MIXED)
    rel = np.abs(got - ref) / (np.abs(A).max(axis=2)[:, :, None] * np.abs(B).max(axis=1)[:, None, :])
    assert rel.max() < 1e-8
    A[0, 7, 3] = np.nan
    got = ctx.gemm(A, B, precision=L.PREC_MIXED)
    assert np.isnan(got[0, 7]).all() and np.isfinite(np.delete(got[0], 7, 0)).all()


@pytest.mark.parametrize("m,n,k,b", GEMM_SHAPES[:6])
def test_tf32_split_gemm_matches_fp64(ctx, m, n, k, b):
    from rcwa_b200 import lib as L
    rng = np.random.default_rng(m * 131 + n * 7 + k)
    A, B = _rand(rng, b, m, k), _rand(rng, b, k, n)
    ref = A @ B
    ctx.set_mixed(L.MIXED_LAYER_GEMM | L.MIXED_STAR_GEMM | L.MIXED_GEMM_TF32, 1, 5)
    try:
        got = ctx.gemm(A, B, precision=L.PREC_MIXED)
    finally:
        ctx.set_mixed(L.MIXED_LAYER_GEMM | L.MIXED_STAR_GEMM, 1, 5)
    scale = np.abs(A).max() * np.abs(B).max() * k
    err = np.abs(got - ref).max() / scale
    assert err < 1e-5, err
    if k >= 16:
        assert np.abs(got - ref).max() > 1e-14 * scale


@pytest.mark.parametrize("n,m,b", [(1, 1, 1), (33, 5, 2), (98, 98, 3), (130, 260, 2), (450, 900, 2),
                                   (450, 2, 4)])
def test_lu_fp32_refined_matches_fp64(ctx, n, m, b):
    """rcwa_lu_solve_ex(RCWA_PREC_MIXED): FP32 factors, FP64 residual
    refinement.  Diagonally weighted random systems (cond ~ 1e2..1e3)."""
    from rcwa_b200 import lib as L
    rng = np.random.default_rng(n * 17 + m + b)
    A = _rand(rng, b, n, n) + 2.0 * np.sqrt(n) * np.eye(n)[None]
    B = _rand(rng, b, n, m)
    X64, s64 = ctx.lu_solve(A, B)
    ref = np.linalg.solve(A, B)
    assert not s64.any()
    assert np.abs(X64 - ref).max() <= 1e-12 * np.abs(ref).max()
    for sweeps, tol in ((1, 1e-10), (2, 1e-13)):
        X, st = ctx.lu_solve(A, B, precision=L.PREC_MIXED, refine_sweeps=sweeps)
        assert not st.any(), st
        err = np.abs(X - ref).max() / np.abs(ref).max()
        assert err <= tol, (sweeps, err)
    # without refinement an FP32 solve would be ~1e-6 off: the result is not FP32
    X32 = np.linalg.solve(A.astype(np.complex64), B.astype(np.complex64))
    if n >= 33:
        assert np.abs(X32 - ref).max() / np.abs(ref).max() > 1e-9


def test_lu_refinement_too_slow_is_flagged(ctx):
    """cond(A) ~ 1e9: FP32 factors are useless (cond * 2^-24 > 1), one FP64
    sweep cannot converge, and the solve says so."""
    from rcwa_b200 import lib as L
    rng = np.random.default_rng(5)
    n = 64
    U, _ = np.linalg.qr(_rand(rng, n, n))
    V, _ = np.linalg.qr(_rand(rng, n, n))
    A = (U * np.logspace(0, -9, n)) @ V.conj().T
    B = _rand(rng, n, 3)
    X, st = ctx.lu_solve(A, B, precision=L.PREC_MIXED, refine_sweeps=1)
    assert st & L.STATUS_REFINE_SLOW
    X64, st64 = ctx.lu_solve(A, B)
    assert not (st64 & L.STATUS_REFINE_SLOW)


def _mixed_vs_fp64(ctx, pb, stages=None):
    from rcwa_b200 import lib as L
    r0 = ctx.solve_sweep(pb, precision=L.PREC_FP64)
    if stages is not None:
        ctx.set_mixed(stages, 1, 5)
    try:
        r1 = ctx.solve_sweep(pb, precision=L.PREC_MIXED)
    finally:
        ctx.set_mixed(L.MIXED_LAYER_GEMM | L.MIXED_STAR_GEMM, 1, 5)
    ok = r0[4] == 0
    assert np.array_equal(r0[4], r1[4])
    d = max(np.abs(r1[0][ok] - r0[0][ok]).max(), np.abs(r1[1][ok] - r0[1][ok]).max(),
            np.abs(r1[2][ok] - r0[2][ok]).max(), np.abs(r1[3][ok] - r0[3][ok]).max())
    return d, r0, r1


def test_mixed_c1_te_tm(ctx):
    """C1 (n = 98): every product is below the int8-slice kernel's size
    threshold (256), so the mixed form runs them in FP64 -- the same result."""
    d, r0, r1 = _mixed_vs_fp64(ctx, C.c1_pillars())
    assert d <= 1e-13, d


def test_mixed_c2_full_sweep(ctx):
    """All 201 wavelengths of the C2 sweep (n = 450), the two Rayleigh
    anomalies (status WOOD_ANOMALY in both forms) excluded."""
    d, r0, r1 = _mixed_vs_fp64(ctx, C.c2_sweep())
    assert d <= TOL_MIXED, d
    assert d > 1e-14, d
    # and the mixed results against the oracle on a few wavelengths
    pb = C.c2_sweep()
    for i in (3, 77, 150):
        ref = oracle_solve(pb, i)
        assert np.abs(r1[0][i] - ref.R).max() <= TOL_MIXED
        assert np.abs(r1[1][i] - ref.T).max() <= TOL_MIXED


@pytest.mark.parametrize("stages", [1, 2, 4, 8, 15])
def test_mixed_single_stage_c2(ctx, stages):
    """Each reduced-precision stage alone stays within the bound (the error
    attribution of the mixed form, on five C2 wavelengths)."""
    pb = C.c2_sweep(lambdas=[420.0, 452.0, 555.0, 690.0, 734.0])
    d, _, _ = _mixed_vs_fp64(ctx, pb, stages)
    assert d <= TOL_MIXED, (stages, d)


def test_mixed_c3_requests_m21(ctx):
    """C3 requests at the largest harmonic order (M = 21, n = 882) on 256^2
    grids: the FP64 form against the oracle, the mixed form against FP64."""
    rng = np.random.default_rng(2121)
    for _ in range(2):
        pb = C.c3_request(rng, grid=256, m_max=21, m_min=21)
        d, r0, r1 = _mixed_vs_fp64(ctx, pb)
        assert d <= TOL_MIXED, d
        ref = oracle_solve(pb)
        assert np.abs(r0[0][0] - ref.R).max() <= 1e-10
        assert np.abs(r0[1][0] - ref.T).max() <= 1e-10


@pytest.mark.parametrize("M,lams", [(23, [250.0, 610.0]), (31, [300.0, 700.0])])
def test_mixed_c4_precision_stress(ctx, M, lams):
    """The C4 stack (21 layers, n = 1058 and 1922): the mixed form within 1e-6
    of the FP64 form, which matches the committed oracle fixtures."""
    pb = C.c4_trapezoid(M=M, lambdas=lams)
    d, r0, r1 = _mixed_vs_fp64(ctx, pb)
    assert not r0[4].any()
    assert d <= TOL_MIXED, d
