"""Failure reporting without a GPU fault, through the C ABI.

The reference abort()s when its eigensolver does not converge (rcwa.cpp:300);
here every bounded loop ends with a status the host reads, and the context
stays usable.  The failures are made on the host: a QR sweep cap of zero set
by rcwa_eig_set_sweep_cap, and a test hook that leaves out the first operand
copy of the int8-slice tensor-core GEMM and of the TMA-fed FP64 GEMM so that
their bounded mbarrier waits (about a second) run out.  Nothing here traps,
faults or hangs a GPU.
"""
import numpy as np
import pytest

from rcwa_b200 import configs as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from rcwa_b200 import lib as L
    c = L.Context(0)
    yield c
    c.close()


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_eig_sweep_cap_reports_noconv(ctx):
    from rcwa_b200 import lib as L
    lib = L.load()
    rng = np.random.default_rng(9)
    A = _rand(rng, 3, 64, 64)
    assert lib.rcwa_eig_set_sweep_cap(0) == L.RCWA_OK
    try:
        lam, W, st = ctx.eig(A)
        assert (st & L.STATUS_EIG_NOCONV).all(), st
        assert np.isnan(lam).any()
        # a whole solve carries the bit in its status word
        pb = C.c1_pillars(grid=64)
        R, T, Rt, Tt, s = ctx.solve_sweep(pb)
        assert (s & L.STATUS_EIG_NOCONV).all(), s
    finally:
        assert lib.rcwa_eig_set_sweep_cap(-1) == L.RCWA_OK
    assert lib.rcwa_eig_set_sweep_cap(-2) == L.RCWA_ERR_INVALID
    lam, W, st = ctx.eig(A)
    assert not st.any()
    for k in range(3):
        assert np.abs(A[k] @ W[k] - W[k] * lam[k][None, :]).max() <= 1e-10 * np.abs(A[k]).max() * 64


def test_int8_gemm_wait_timeout_is_reported(ctx):
    from rcwa_b200 import lib as L
    lib = L.load()
    rng = np.random.default_rng(10)
    A, B = _rand(rng, 1, 40, 70), _rand(rng, 1, 70, 30)
    assert lib.rcwa_debug_gemm_inject_timeout(1) == L.RCWA_OK
    try:
        with pytest.raises(L.RcwaError) as e:
            ctx.gemm(A, B, precision=L.PREC_MIXED)
        assert e.value.code == L.RCWA_ERR_CUDA
        assert "wait" in str(e.value)
    finally:
        lib.rcwa_debug_gemm_inject_timeout(0)
    # the context and the device are fine afterwards
    got = ctx.gemm(A, B, precision=L.PREC_MIXED)
    ref = A @ B
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_tma_dmma_gemm_wait_timeout_is_reported(ctx):
    """The FP64 kernel fed by the tensor memory accelerator: with its first
    k-tile copy left out, every warp's bounded wait runs out; the call
    reports the device flag, and the next product is exact again."""
    import ctypes
    from rcwa_b200 import lib as L
    lib = L.load()
    rng = np.random.default_rng(11)
    A, B = _rand(rng, 2, 100, 100), _rand(rng, 2, 100, 90)
    assert lib.rcwa_set_gemm_table((ctypes.c_int * 25)(*([2] * 25))) == L.RCWA_OK
    try:
        assert lib.rcwa_debug_gemm_inject_timeout(1) == L.RCWA_OK
        try:
            with pytest.raises(L.RcwaError) as e:
                ctx.gemm(A, B)
            assert e.value.code == L.RCWA_ERR_CUDA
            assert "wait" in str(e.value)
        finally:
            lib.rcwa_debug_gemm_inject_timeout(0)
        got = ctx.gemm(A, B)
        ref = A @ B
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    finally:
        if not L.apply_tuning():
            lib.rcwa_set_gemm_table(None)
