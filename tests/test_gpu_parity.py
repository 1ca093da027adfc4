"""GPU parity tests: every call goes through the C ABI (librcwa_b200.so) and is
checked against the FP64 oracle restatement of the reference.

Tolerances: the plain FP64 path must reproduce the reference's R/T to
|dR|, |dT| <= 1e-10 (absolute, per order) and conserve energy to 1e-10 on
lossless stacks; dense building blocks are checked to 1e-11 relative to the
operand norms.
"""
import math

import numpy as np
import pytest

from oracle import rcwa_oracle as O
from rcwa_b200 import configs as C
from helpers import oracle_args, oracle_solve, oracle_sweep
from thinfilm import thin_film_rt

pytestmark = pytest.mark.gpu

TOL_RT = 1e-10


@pytest.fixture(scope="module")
def ctx():
    from rcwa_b200 import lib as L
    c = L.Context(0)
    yield c
    c.close()


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


# ---------------------------------------------------------------- building blocks
@pytest.mark.parametrize("m,n,k,b", [(1, 1, 1, 1), (37, 53, 29, 3), (98, 98, 98, 2), (130, 70, 200, 1)])
def test_gemm(ctx, m, n, k, b):
    rng = np.random.default_rng(m + n + k)
    A, B = _rand(rng, b, m, k), _rand(rng, b, k, n)
    Cg = ctx.gemm(A, B)
    ref = A @ B
    assert np.abs(Cg - ref).max() <= 1e-13 * math.sqrt(k) * np.abs(ref).max() + 1e-14


# sizes just above a multiple of 64 run their last rows / columns through the
# thin-strip CTAs beside the tensor-core tiles
@pytest.mark.parametrize("opa,opb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("m,n,k,b", [(450, 450, 450, 2), (66, 80, 100, 3), (140, 900, 130, 1),
                                     (64, 193, 65, 2), (79, 79, 300, 1)])
def test_gemm_ops_and_thin_edges(ctx, opa, opb, m, n, k, b):
    rng = np.random.default_rng(m * 3 + n + k + 7 * opa + 11 * opb)
    A = _rand(rng, b, k, m) if opa else _rand(rng, b, m, k)
    B = _rand(rng, b, n, k) if opb else _rand(rng, b, k, n)
    C0 = _rand(rng, b, m, n)
    alpha, beta = 0.7 - 0.4j, -1.2 + 0.3j
    Cg = ctx.gemm_ex(A, B, C0, opa, opb, alpha, beta)
    opA = np.conj(A.transpose(0, 2, 1)) if opa else A
    opB = np.conj(B.transpose(0, 2, 1)) if opb else B
    ref = alpha * (opA @ opB) + beta * C0
    assert np.abs(Cg - ref).max() <= 1e-13 * math.sqrt(k) * np.abs(ref).max() + 1e-14


@pytest.mark.parametrize("n,m,b", [(1, 1, 2), (7, 3, 4), (33, 5, 2), (98, 98, 3), (250, 17, 2)])
def test_lu_solve(ctx, n, m, b):
    rng = np.random.default_rng(n * 7 + m)
    A = _rand(rng, b, n, n) + 3 * np.eye(n)
    B = _rand(rng, b, n, m)
    X, st = ctx.lu_solve(A, B)
    assert not st.any()
    ref = np.linalg.solve(A, B)
    assert np.abs(X - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max())


def test_lu_pivoting_needed(ctx):
    # zero leading pivot: only partial pivoting solves this
    A = np.array([[0.0, 1.0, 2.0], [1.0, 0.0, 3.0], [4.0, -3.0, 8.0]], dtype=complex)
    b = np.array([1.0, 2.0, 3.0], dtype=complex)
    x, st = ctx.lu_solve(A, b[:, None])
    assert st == 0
    assert np.allclose(x[:, 0], np.linalg.solve(A, b), atol=1e-13)


def test_lu_singular_flagged(ctx):
    A = np.zeros((4, 4), complex)
    A[0, 0] = 1.0
    x, st = ctx.lu_solve(A, np.ones((4, 1), complex))
    from rcwa_b200 import lib as L
    assert st & L.STATUS_SINGULAR


def _eig_check(A, lam, W, tol=1e-10):
    n = A.shape[0]
    nrm = np.abs(A).max() * n
    res = np.abs(A @ W - W * lam[None, :]).max()
    assert res <= tol * nrm, res / nrm
    assert np.allclose(np.linalg.norm(W, axis=0), 1.0, atol=1e-12)
    ref = np.linalg.eigvals(A)
    # every GPU eigenvalue has a matching reference eigenvalue
    d = np.abs(lam[:, None] - ref[None, :]).min(axis=1)
    assert d.max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.parametrize("n", [1, 2, 3, 5, 18, 19, 20, 50, 98, 163])
def test_eig_random(ctx, n):
    rng = np.random.default_rng(n)
    A = _rand(rng, n, n)
    lam, W, st = ctx.eig(A)
    assert st == 0
    _eig_check(A, lam, W)


def test_eig_batched_and_structured(ctx):
    rng = np.random.default_rng(5)
    n = 40
    mats = [_rand(rng, n, n)]
    # degenerate but diagonalisable (uniform-layer-like): repeated eigenvalues
    Q = np.linalg.qr(_rand(rng, n, n))[0]
    d = np.repeat(_rand(rng, n // 2), 2)
    mats.append(Q @ np.diag(d) @ np.linalg.inv(Q))
    # upper Hessenberg input and a diagonal input
    H = np.triu(_rand(rng, n, n), -1)
    mats.append(H)
    mats.append(np.diag(_rand(rng, n)))
    A = np.stack(mats)
    lam, W, st = ctx.eig(A)
    assert not st.any()
    for i in (0, 2, 3):
        _eig_check(A[i], lam[i], W[i])
    # degenerate case: eigenvalues right, eigenvectors span (cond(W) finite)
    assert np.abs(np.sort_complex(lam[1]) - np.sort_complex(d)).max() < 1e-10 * np.abs(d).max()
    assert np.abs(A[1] @ W[1] - W[1] * lam[1][None, :]).max() < 1e-9 * np.abs(A[1]).max() * n


def test_eig_aed_paths(ctx):
    """Matrices large enough for aggressive early deflation (active blocks of
    30 or more): a random one, one with clusters of nearly equal eigenvalues
    (many window eigenvalues deflate at once), an exactly degenerate
    diagonalisable one, and an upper-triangular-plus-noise one whose
    eigenvalues are mostly converged on entry."""
    rng = np.random.default_rng(17)
    n = 160
    Q = np.linalg.qr(_rand(rng, n, n))[0]
    clus = np.repeat(_rand(rng, n // 8), 8) + 1e-9 * _rand(rng, n)
    degen = np.repeat(_rand(rng, n // 4), 4)
    T = np.diag(10.0 * _rand(rng, n)) + 0.1 * np.triu(_rand(rng, n, n), 1) + 1e-13 * _rand(rng, n, n)
    mats = [_rand(rng, n, n), Q @ np.diag(clus) @ Q.conj().T, Q @ np.diag(degen) @ Q.conj().T, T]
    A = np.stack(mats)
    lam, W, st = ctx.eig(A)
    assert not st.any()
    for i in (0, 1, 3):
        _eig_check(A[i], lam[i], W[i])
    ref = np.sort_complex(degen)
    assert np.abs(np.sort_complex(lam[2]) - ref).max() < 1e-9 * np.abs(ref).max()
    assert np.abs(A[2] @ W[2] - W[2] * lam[2][None, :]).max() < 1e-9 * np.abs(A[2]).max() * n


@pytest.mark.parametrize("cl", [2, 4, 8])
def test_eig_cluster_ctas_match_one_cta(ctx, cl):
    """The QR iteration with cl CTAs per matrix (a thread-block cluster whose
    helper CTAs share the far updates of each multishift sweep) applies the
    same reflectors to the same entries as one CTA: the eigen-decomposition
    is identical, and a true one."""
    from rcwa_b200 import lib as L
    lib = L.load()
    rng = np.random.default_rng(450 + cl)
    n = 450
    A = _rand(rng, 3, n, n)
    assert lib.rcwa_eig_set_cluster_size(1) == 0
    try:
        lam1, W1, st1 = ctx.eig(A)
        assert lib.rcwa_eig_set_cluster_size(cl) == 0
        lam2, W2, st2 = ctx.eig(A)
    finally:
        lib.rcwa_eig_set_cluster_size(0)
    assert not st1.any() and not st2.any()
    assert np.abs(lam2 - lam1).max() <= 1e-13 * np.abs(lam1).max()
    assert np.abs(W2 - W1).max() <= 1e-12
    _eig_check(A[0], lam2[0], W2[0])
    assert lib.rcwa_eig_set_cluster_size(3) == L.RCWA_ERR_INVALID


def test_cluster_eigensolver_in_a_solve(ctx):
    """A single large request (M = 25, n = 1250: few matrices, so the
    eigensolver runs its QR iteration on clusters of CTAs) gives the same R/T
    as with one CTA per matrix."""
    from rcwa_b200 import lib as L
    lib = L.load()
    rng = np.random.default_rng(4)
    pb = C.c3_request(rng, grid=128, m_max=25, m_min=25)
    a = ctx.solve_sweep(pb)
    assert lib.rcwa_eig_set_cluster_size(1) == 0
    try:
        b = ctx.solve_sweep(pb)
    finally:
        lib.rcwa_eig_set_cluster_size(0)
    assert a[4][0] == 0 and b[4][0] == 0
    assert np.abs(a[0] - b[0]).max() <= 1e-12 and np.abs(a[1] - b[1]).max() <= 1e-12


def test_eig_nonfinite_flagged(ctx):
    A = np.eye(6, dtype=complex)
    A[2, 3] = np.nan
    lam, W, st = ctx.eig(A)
    from rcwa_b200 import lib as L
    assert st & L.STATUS_NONFINITE


# ---------------------------------------------------------------- step functions
def _small_layer_problem():
    L = 480.0
    g = C.circle(64, 64, L, L, 130.0, 9.0 - 0.4j, 1.0)
    st = C.make_stack(L, L, [g], [140.0])
    src = C.SourceSpec(605.0, math.radians(23.0), math.radians(31.0), 0.8, 0.6)
    return C.Problem("small", st, [src], C.ParamSpec(2, 3, 1.0, 1.0, 2.25, 1.0))


def test_convmat_matches_oracle(ctx):
    rng = np.random.default_rng(3)
    Nx, Ny = 40, 34
    f = _rand(rng, 2 * Nx * Ny)
    for (hx, hy) in [(0, 0), (2, 3), (5, 4), (12, 11)]:   # last one exceeds Nx/4: zero fill
        ref = O.conv_mat(f, 1, Nx, Ny, hx, hy)
        got = ctx.convmat(f, 1, Nx, Ny, hx, hy)
        assert np.abs(got - ref).max() <= 1e-13


def test_wave_vectors_and_gap_match_oracle(ctx):
    pb = _small_layer_problem()
    S, src, par = oracle_args(pb)
    k_inc, Kx, Ky, Kzr, Kzt = O.compute_wave_vectors(S.Lx, S.Ly, src, par)
    gk, gx, gy, gzr, gzt = ctx.wave_vectors(S.Lx, S.Ly, pb.sources[0], pb.params)
    assert np.abs(gk - np.array(k_inc)).max() < 1e-14
    for a, b in ((gx, Kx), (gy, Ky), (gzr, Kzr), (gzt, Kzt)):
        assert np.abs(a - b).max() < 1e-13
    W0, V0 = O.gap_medium(Kx, Ky)
    gW0, gV0 = ctx.gap_medium(Kx, Ky)
    assert np.abs(gW0 - W0).max() == 0.0
    assert np.abs(gV0 - V0).max() < 1e-13 * np.abs(V0).max()


def test_smatrix_layer_and_ports_match_oracle(ctx):
    pb = _small_layer_problem()
    S, src, par = oracle_args(pb)
    erc, urc = O.conv_mats(S, par)
    k_inc, Kx, Ky, Kzr, Kzt = O.compute_wave_vectors(S.Lx, S.Ly, src, par)
    W0, V0 = O.gap_medium(Kx, Ky)
    ref = O.smatrix_layer(erc[0], urc[0], Kx, Ky, W0, V0, src.k0, 140.0)
    S11, S12, st = ctx.smatrix_layer(erc[0], urc[0], Kx, Ky, V0, src.k0, 140.0)
    assert st == 0
    assert np.abs(S11 - ref.S11).max() < 1e-11
    assert np.abs(S12 - ref.S12).max() < 1e-11
    for side, fn, kz in (("ref", O.smatrix_reflection, Kzr), ("trn", O.smatrix_transmission, Kzt)):
        Sref, _ = fn(par, Kx, Ky, kz, W0, V0)
        got = ctx.smatrix_port(side, pb.params, Kx, Ky, kz, V0)
        for a, b in zip(got, (Sref.S11, Sref.S12, Sref.S21, Sref.S22)):
            assert np.abs(a - b).max() < 1e-12 * max(1.0, np.abs(b).max())


def test_redheffer_matches_oracle(ctx):
    rng = np.random.default_rng(11)
    n = 30
    A = [0.3 * _rand(rng, n, n) / math.sqrt(n) for _ in range(4)]
    B = [0.3 * _rand(rng, n, n) / math.sqrt(n) for _ in range(4)]
    ref = O.redheffer_product(O.SMatrix(*A), O.SMatrix(*B))
    got, st = ctx.redheffer(A, B)
    assert st == 0
    for a, b in zip(got, (ref.S11, ref.S12, ref.S21, ref.S22)):
        assert np.abs(a - b).max() < 1e-12


def test_efficiencies_match_oracle(ctx):
    pb = _small_layer_problem()
    S, src, par = oracle_args(pb)
    k_inc, Kx, Ky, Kzr, Kzt = O.compute_wave_vectors(S.Lx, S.Ly, src, par)
    rng = np.random.default_rng(2)
    n = 2 * Kx.size
    S11, S21 = 0.1 * _rand(rng, n, n), 0.1 * _rand(rng, n, n)
    Sg = O.SMatrix(S11, None, S21, None)
    csrc = O.source_mode_coeff(src, par, k_inc, np.eye(n))
    r = O.reflected_field(Sg, csrc, Kx, Ky, Kzr, np.eye(n))
    t = O.transmitted_field(Sg, csrc, Kx, Ky, Kzt, np.eye(n))
    ref = O.diffraction_efficiencies(par, r, t, k_inc, Kzr, Kzt)
    R, T, Rt, Tt, st = ctx.efficiencies(pb.sources[0], pb.params, np.array(k_inc), Kx, Ky, Kzr, Kzt, S11, S21)
    assert np.abs(R - ref.R).max() < 1e-13 and np.abs(T - ref.T).max() < 1e-13
    assert abs(Rt - ref.R_tot) < 1e-12 and abs(Tt - ref.T_tot) < 1e-12


# ---------------------------------------------------------------- end to end
def _assert_parity(R, T, Rt, Tt, ref, tol=TOL_RT):
    assert np.abs(R - ref.R).max() <= tol, np.abs(R - ref.R).max()
    assert np.abs(T - ref.T).max() <= tol, np.abs(T - ref.T).max()
    assert abs(Rt - ref.R_tot) <= tol and abs(Tt - ref.T_tot) <= tol


def test_reference_demo_case(ctx):
    pb = C.demo_triangle(grid=256)
    R, T, Rt, Tt, st = ctx.solve_sweep(pb)
    assert st[0] == 0
    _assert_parity(R[0], T[0], Rt[0], Tt[0], oracle_solve(pb))
    assert abs(Rt[0] + Tt[0] - 1.0) < 1e-10


def test_c1_pillars_te_tm(ctx):
    pb = C.c1_pillars(grid=512)
    R, T, Rt, Tt, st = ctx.solve_sweep(pb)
    assert not st.any()
    refs = oracle_sweep(pb)
    for i, ref in enumerate(refs):
        _assert_parity(R[i], T[i], Rt[i], Tt[i], ref)
        assert abs(Rt[i] + Tt[i] - 1.0) < 1e-10


@pytest.mark.parametrize("pol", ["TE", "TM"])
def test_uniform_stack_thin_film(ctx, pol):
    eps = [4.0, 2.2 - 0.3j, 9.5 - 0.05j]
    d = [120.0, 75.0, 33.0]
    th = math.radians(35.0)
    grids = [C.uniform(8, 8, e) for e in eps]
    st = C.make_stack(700.0, 650.0, grids, d)
    pte, ptm = (1.0, 0.0) if pol == "TE" else (0.0, 1.0)
    pb = C.Problem("u", st, [C.SourceSpec(633.0, th, 0.0, pte, ptm)], C.ParamSpec(2, 2, 1.0, 1.0, 2.25, 1.0))
    R, T, Rt, Tt, s = ctx.solve_sweep(pb)
    Rf, Tf = thin_film_rt(eps, d, 1.0, 2.25, 633.0, th, pol)
    assert abs(Rt[0] - Rf) < 1e-11 and abs(Tt[0] - Tf) < 1e-11


def test_c2_subset_and_wood_anomaly(ctx):
    # the 201-point sweep contains two exact Rayleigh anomalies (400 and 600 nm)
    lams = [400.0, 452.0, 600.0, 734.0]
    pb = C.c2_sweep(lambdas=lams)
    R, T, Rt, Tt, st = ctx.solve_sweep(pb)
    from rcwa_b200 import lib as L
    assert st[0] & L.STATUS_WOOD_ANOMALY and st[2] & L.STATUS_WOOD_ANOMALY
    refs = oracle_sweep(pb, idx=[1, 3])
    for i, ref in zip((1, 3), refs):
        assert st[i] == 0
        _assert_parity(R[i], T[i], Rt[i], Tt[i], ref)


def test_c3_requests(ctx):
    rng = np.random.default_rng(33)
    for _ in range(4):
        pb = C.c3_request(rng, grid=128, m_max=9)
        R, T, Rt, Tt, st = ctx.solve_sweep(pb)
        assert st[0] == 0
        _assert_parity(R[0], T[0], Rt[0], Tt[0], oracle_solve(pb))


def test_zero_thickness_and_single_uniform(ctx):
    L = 450.0
    g = C.circle(64, 64, L, L, 120.0, 8.0, 1.0)
    src = [C.SourceSpec(610.0, math.radians(20.0), math.radians(40.0), 0.6, 0.8)]
    par = C.ParamSpec(2, 2, 1.0, 1.0, 2.25, 1.0)
    pa = C.Problem("a", C.make_stack(L, L, [g], [150.0]), src, par)
    pb = C.Problem("b", C.make_stack(L, L, [g, C.uniform(64, 64, 3.0)], [150.0, 0.0]), src, par)
    a = ctx.solve_sweep(pa)
    b = ctx.solve_sweep(pb)
    assert np.abs(a[0] - b[0]).max() < 1e-11 and np.abs(a[1] - b[1]).max() < 1e-11


@pytest.mark.parametrize("name", ["golden_small_c1", "golden_small_mixed", "golden_c4_m23", "golden_c4_m23_sweep",
                                  "golden_c4_m31", "golden_c3_full_0", "golden_c3_full_1", "golden_c3_full_2"])
def test_golden_fixtures(ctx, name):
    """The CUDA path reproduces the committed fixtures (generated by the
    oracle, tests/golden/make_golden.py) to 1e-10 per order: small cases, the
    C4 stack at M = 23 (n = 1058, four wavelengths) and M = 31 (n = 1922, two
    wavelengths), and full-size C3 requests (M = 15..21, 256^2 grids)."""
    import os
    from golden.make_golden import build_case
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    pb = build_case(name)
    R, T, Rt, Tt, st = ctx.solve_sweep(pb)
    assert not st.any()
    assert np.abs(R - z["R"]).max() <= TOL_RT
    assert np.abs(T - z["T"]).max() <= TOL_RT
    assert np.abs(Rt - z["R_tot"]).max() <= TOL_RT
    assert np.abs(Tt - z["T_tot"]).max() <= TOL_RT


def test_polarisation_variants_share_solves(ctx):
    """Sources that differ only in (pte, ptm) share one S-matrix solve; every
    source still gets its own efficiencies in its own output row."""
    import dataclasses
    pb0 = _small_layer_problem()
    mk = lambda lam, th, ph, te, tm: C.SourceSpec(lam, math.radians(th), math.radians(ph), te, tm)
    srcs = [mk(600.0, 17.0, 11.0, 1.0, 0.0), mk(650.0, 5.0, 0.0, 0.0, 1.0), mk(600.0, 17.0, 11.0, 0.0, 1.0),
            mk(600.0, 17.0, 11.0, 0.6, 0.8), mk(650.0, 5.0, 0.0, 1.0, 0.0)]
    pb = dataclasses.replace(pb0, sources=srcs)
    R, T, Rt, Tt, st = ctx.solve_sweep(pb)
    assert not st.any()
    for i in range(len(srcs)):
        ref = oracle_solve(pb, i)
        _assert_parity(R[i], T[i], Rt[i], Tt[i], ref)
        R1, T1, Rt1, Tt1, st1 = ctx.solve_sweep(pb, sources=[srcs[i]])
        assert np.abs(R1[0] - R[i]).max() <= 1e-13 and abs(Tt1[0] - Tt[i]) <= 1e-13
