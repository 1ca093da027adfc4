"""The FP64 GEMM kernels behind every complex product, each forced for every
shape through the kernel table (rcwa_set_gemm_table): the DMMA kernel fed
by cp.async (0), the CUDA-core kernel (1), the DMMA kernel fed by the
tensor memory accelerator (2) and the cp.async-fed DMMA kernel on 32 x 64
tiles (3).  Each is checked against numpy on
the product form (alpha A B + beta C) and on the LU / Hessenberg update form
(C - A B), at shapes with ragged edges, thin strips and rank-32 updates, and
the TMA-fed kernel runs a whole solve against the FP64 oracle.  Tolerance as
for the other dense building blocks: 1e-13 sqrt(k) relative to the result.
"""
import ctypes
import math

import numpy as np
import pytest

from rcwa_b200 import configs as C
from helpers import oracle_solve

pytestmark = pytest.mark.gpu

SHAPES = [(37, 53, 29, 3), (450, 450, 450, 2), (66, 80, 100, 3), (140, 900, 130, 1), (64, 193, 65, 2),
          (79, 79, 300, 1), (418, 418, 32, 3), (200, 37, 64, 2), (129, 129, 129, 1), (8, 8, 8, 5),
          (1, 70, 9, 2)]


@pytest.fixture(scope="module")
def ctx():
    from rcwa_b200 import lib as L
    c = L.Context(0)
    yield c
    c.close()


@pytest.fixture
def force(ctx):
    from rcwa_b200 import lib as L
    lib = L.load()

    def set_choice(choice):
        arr = (ctypes.c_int * 25)(*([choice] * 25))
        assert lib.rcwa_set_gemm_table(arr) == L.RCWA_OK

    yield set_choice
    if not L.apply_tuning():
        lib.rcwa_set_gemm_table(None)


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("choice", [0, 1, 2, 3])
@pytest.mark.parametrize("m,n,k,b", SHAPES)
def test_product_and_update_forms(ctx, force, choice, m, n, k, b):
    force(choice)
    rng = np.random.default_rng(m + 3 * n + 7 * k + b)
    A, B, C0 = _rand(rng, b, m, k), _rand(rng, b, k, n), _rand(rng, b, m, n)
    tol = lambda ref: 1e-13 * math.sqrt(k) * np.abs(ref).max() + 1e-14
    ref = A @ B
    got = ctx.gemm(A, B)
    assert np.abs(got - ref).max() <= tol(ref)
    alpha, beta = 0.7 - 0.4j, -1.2 + 0.3j
    ref = alpha * (A @ B) + beta * C0
    got = ctx.gemm_ex(A, B, C0, 0, 0, alpha, beta)
    assert np.abs(got - ref).max() <= tol(ref)
    ref = C0 - A @ B
    got = ctx.gemm_ex(A, B, C0, 0, 0, -1.0, 1.0)
    assert np.abs(got - ref).max() <= tol(ref)


def test_solve_on_tma_fed_kernel(ctx, force):
    force(2)
    pb = C.c1_pillars(grid=128)
    R, T, Rt, Tt, st = ctx.solve_sweep(pb)
    for i in range(len(pb.sources)):
        assert st[i] == 0
        ref = oracle_solve(pb, i)
        assert np.abs(R[i] - ref.R).max() <= 1e-10
        assert np.abs(T[i] - ref.T).max() <= 1e-10
