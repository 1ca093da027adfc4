"""Mixed-precision building blocks: the split-TF32 tcgen05 complex GEMM
against FP64 (through the C ABI).  Tolerance: 3xTF32 with FP32 accumulation
keeps ~2^-21 relative per product, so errors are bounded by
2e-6 * sqrt(k) * max|A| * max|B| * k^(1/2) -- checked as a norm-relative 1e-5."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from rcwa_b200 import lib as L
    c = L.Context(0)
    yield c
    c.close()


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("m,n,k,b", [(1, 1, 1, 1), (8, 8, 8, 1), (64, 128, 16, 1), (70, 130, 50, 2),
                                     (128, 256, 100, 1), (450, 450, 450, 1)])
def test_tc_gemm_matches_fp64(ctx, m, n, k, b):
    from rcwa_b200 import lib as L
    rng = np.random.default_rng(m * 131 + n * 7 + k)
    A, B = _rand(rng, b, m, k), _rand(rng, b, k, n)
    ref = A @ B
    got = ctx.gemm(A, B, precision=L.PREC_MIXED)
    scale = np.abs(A).max() * np.abs(B).max() * k
    err = np.abs(got - ref).max() / scale
    assert err < 1e-5, err
    # it is not the FP64 kernel: the error is above FP64 rounding
    if k >= 16:
        assert np.abs(got - ref).max() > 1e-14 * scale


def test_mixed_sweep_against_fp64(ctx):
    """rcwa_solve_sweep with RCWA_PREC_MIXED (split-TF32 S-matrix algebra,
    FP64 Omega^2 and eigensolver) against the FP64 sweep on C1 (n = 98) and a
    5-wavelength slice of the C2 sweep (n = 450).  Measured on B200: C1
    |dR|,|dT| ~ 2e-6, C2 ~ 1.5e-5; the bound checked here is 1e-4, and the
    difference must exceed FP64 rounding (the tensor-core path really ran)."""
    from rcwa_b200 import lib as L, configs as Cf
    for pb in (Cf.c1_pillars(), Cf.c2_sweep(lambdas=[420.0, 452.0, 555.0, 690.0, 734.0])):
        R0, T0, Rt0, Tt0, st0 = ctx.solve_sweep(pb, precision=L.PREC_FP64)
        R1, T1, Rt1, Tt1, st1 = ctx.solve_sweep(pb, precision=L.PREC_MIXED)
        assert np.array_equal(st0, st1)
        d = max(np.abs(R1 - R0).max(), np.abs(T1 - T0).max(),
                np.abs(Rt1 - Rt0).max(), np.abs(Tt1 - Tt0).max())
        assert d < 1e-4, d
        assert d > 1e-13, d
