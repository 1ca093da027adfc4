"""Pins for the CPU oracle: closed-form physics, conservation, symmetry,
eigen-basis invariance and the committed golden vectors (CPU only)."""
import math
import os

import numpy as np
import pytest

from oracle import rcwa_oracle as O
from rcwa_b200 import configs as C
from helpers import oracle_args, oracle_solve
from thinfilm import thin_film_rt

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _uniform_problem(eps_layers, d, eps_ref, eps_trn, lam, theta, phi, pol, h=2, grid=16):
    grids = [C.uniform(grid, grid, e) for e in eps_layers]
    st = C.make_stack(700.0, 650.0, grids, d)
    pte, ptm = (1.0, 0.0) if pol == "TE" else (0.0, 1.0)
    return C.Problem("uniform", st, [C.SourceSpec(lam, theta, phi, pte, ptm)],
                     C.ParamSpec(h, h, eps_ref, 1.0, eps_trn, 1.0))


@pytest.mark.parametrize("pol", ["TE", "TM"])
@pytest.mark.parametrize("theta_deg", [0.0, 20.0, 47.0])
def test_uniform_stack_matches_thin_film(pol, theta_deg):
    eps = [4.0 - 0.0j, 2.2 - 0.3j, 9.5 - 0.05j]   # reference convention: loss is Im < 0
    d = [120.0, 75.0, 33.0]
    th = math.radians(theta_deg)
    pb = _uniform_problem(eps, d, 1.0, 2.25, 633.0, th, 0.0, pol)
    res = oracle_solve(pb)
    R, T = thin_film_rt(eps, d, 1.0, 2.25, 633.0, th, pol)
    assert abs(res.R_tot - R) < 1e-11
    assert abs(res.T_tot - T) < 1e-11
    # only the specular order carries power
    P = res.R.copy()
    q0, p0 = P.shape[0] // 2, P.shape[1] // 2
    P[q0, p0] = 0.0
    assert np.abs(P).max() < 1e-20


def test_uniform_lossless_conserves_energy_oblique_phi():
    pb = _uniform_problem([6.0, 1.7], [210.0, 90.0], 1.0, 2.25, 555.0,
                          math.radians(33.0), math.radians(27.0), "TE")
    r = oracle_solve(pb)
    assert abs(r.R_tot + r.T_tot - 1.0) < 1e-12


def test_c1_energy_and_te_tm_symmetry():
    pb = C.c1_pillars(grid=128)
    te, tm = oracle_solve(pb, 0), oracle_solve(pb, 1)
    for r in (te, tm):
        assert abs(r.R_tot + r.T_tot - 1.0) < 1e-10
    # square lattice of discs at normal incidence: TE and TM see the same structure
    assert np.abs(te.R - tm.R.T).max() < 1e-10
    assert abs(te.R_tot - tm.R_tot) < 1e-10


def test_reference_demo_conserves_energy():
    r = oracle_solve(C.demo_triangle(grid=128))
    assert abs(r.R_tot + r.T_tot - 1.0) < 1e-10


def test_1d_grating_phi0_only_q0_orders():
    L = 500.0
    g = C.lines_x(64, 64, L, 0.4 * L, 11.0, 1.0)
    st = C.make_stack(L, L, [g], [180.0])
    pb = C.Problem("1d", st, [C.SourceSpec(480.0, math.radians(12.0), 0.0, 0.3, 0.8)],
                   C.ParamSpec(3, 2, 1.0, 1.0, 2.25, 1.0))
    r = oracle_solve(pb)
    q0 = r.R.shape[0] // 2
    mask = np.ones_like(r.R, dtype=bool)
    mask[q0, :] = False
    assert np.abs(r.R[mask]).max() < 1e-20 and np.abs(r.T[mask]).max() < 1e-20
    assert abs(r.R_tot + r.T_tot - 1.0) < 1e-10


def test_zero_thickness_layer_is_identity():
    L = 450.0
    g = C.circle(64, 64, L, L, 120.0, 8.0, 1.0)
    g2 = C.rect(64, 64, L, L, 200.0, 100.0, 3.0, 1.5)
    src = [C.SourceSpec(610.0, math.radians(20.0), math.radians(40.0), 0.6, 0.8)]
    par = C.ParamSpec(2, 2, 1.0, 1.0, 2.25, 1.0)
    a = oracle_solve(C.Problem("a", C.make_stack(L, L, [g], [150.0]), src, par))
    b = oracle_solve(C.Problem("b", C.make_stack(L, L, [g, g2], [150.0, 0.0]), src, par))
    assert np.abs(a.R - b.R).max() < 1e-11 and np.abs(a.T - b.T).max() < 1e-11


def test_eigenbasis_invariance():
    """S does not depend on eigenvector order or scaling (rcwa.cpp:335-348)."""
    import scipy.linalg as sla
    L = 450.0
    g = C.circle(32, 32, L, L, 140.0, 7.0 - 0.2j, 1.0)
    S, src, par = oracle_args(C.Problem("e", C.make_stack(L, L, [g], [130.0]),
                                        [C.SourceSpec(590.0, 0.3, 0.2, 1.0, 0.0)],
                                        C.ParamSpec(2, 2, 1.0, 1.0, 2.25, 1.0)))
    erc, urc = O.conv_mats(S, par)
    k_inc, Kx, Ky, Kzr, Kzt = O.compute_wave_vectors(S.Lx, S.Ly, src, par)
    W0, V0 = O.gap_medium(Kx, Ky)
    base = O.smatrix_layer(erc[0], urc[0], Kx, Ky, W0, V0, src.k0, 130.0)
    rng = np.random.default_rng(0)

    def scrambled(A):
        lam2, W = sla.eig(A)
        perm = rng.permutation(lam2.size)
        scale = rng.uniform(0.5, 2.0, lam2.size) * np.exp(1j * rng.uniform(0, 6.28, lam2.size))
        return lam2[perm], W[:, perm] * scale[None, :]

    alt = O.smatrix_layer(erc[0], urc[0], Kx, Ky, W0, V0, src.k0, 130.0, eig=scrambled)
    assert np.abs(base.S11 - alt.S11).max() < 1e-10
    assert np.abs(base.S12 - alt.S12).max() < 1e-10


def test_unsigned_sqrt_branch():
    z = np.array([-4.0 - 0.0j, -4.0 + 0.0j, complex(-4.0, -1e-300), 4.0 + 0j])
    w = O.unsigned_sqrt(z)
    assert w[0] == 2j and w[1] == 2j
    assert w[2].imag < 0
    assert w[3] == 2.0


def test_conv_mat_matches_direct_dft():
    rng = np.random.default_rng(1)
    Nx, Ny, hx, hy = 12, 10, 3, 2
    f = rng.standard_normal(2 * Nx * Ny) + 1j * rng.standard_normal(2 * Nx * Ny)
    C1 = O.conv_mat(f, 1, Nx, Ny, hx, hy)
    g = f[Nx * Ny:].reshape(Ny, Nx)
    P, Q = 2 * hx + 1, 2 * hy + 1
    ix, iy = np.arange(Nx), np.arange(Ny)
    for m in range(P * Q):
        for n in range(P * Q):
            dx = (m // Q - n // Q)
            dy = (m % Q - n % Q)
            if -(Nx // 2) <= dx < Nx - Nx // 2 and -(Ny // 2) <= dy < Ny - Ny // 2:
                ref = (g * np.exp(-2j * np.pi * (dx * ix[None, :] / Nx + dy * iy[:, None] / Ny))).sum() / (Nx * Ny)
            else:
                ref = 0.0
            assert abs(C1[m, n] - ref) < 1e-13


@pytest.mark.parametrize("name", ["golden_small_c1", "golden_small_mixed"])
def test_golden_fixtures_reproduce(name):
    """The committed fixtures (tests/golden/make_golden.py) are reproduced."""
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    from golden.make_golden import build_case
    z = np.load(path)
    pb = build_case(name)
    for i in range(len(pb.sources)):
        r = oracle_solve(pb, i)
        assert np.abs(r.R - z["R"][i]).max() < 1e-12
        assert np.abs(r.T - z["T"][i]).max() < 1e-12


@pytest.mark.parametrize("pol", ["TE", "TM"])
@pytest.mark.parametrize("theta_deg", [0.0, 20.0, 47.0])
def test_magnetic_uniform_stack_matches_thin_film(pol, theta_deg):
    """Permeability in the layers and in both half-spaces (rcwa.cpp:361-372,
    421-432, 579-582) against the characteristic-matrix formulas with mu."""
    eps = [4.0, 2.2 - 0.3j, 9.5 - 0.05j]
    mus = [1.7, 2.5 - 0.1j, 1.0]
    d = [120.0, 75.0, 33.0]
    st = C.make_stack(700.0, 650.0, [C.uniform(16, 16, e) for e in eps], d,
                      [C.uniform(16, 16, m) for m in mus])
    pte, ptm = (1.0, 0.0) if pol == "TE" else (0.0, 1.0)
    th = math.radians(theta_deg)
    pb = C.Problem("mu", st, [C.SourceSpec(633.0, th, 0.0, pte, ptm)], C.ParamSpec(2, 2, 1.0, 1.3, 2.25, 1.6))
    res = oracle_solve(pb)
    R, T = thin_film_rt(eps, d, 1.0, 2.25, 633.0, th, pol, mus, 1.3, 1.6)
    assert abs(res.R_tot - R) < 1e-11 and abs(res.T_tot - T) < 1e-11


@pytest.mark.parametrize("rule", ["laurent", "li"])
def test_lossless_magnetic_pattern_conserves_energy(rule):
    nx, ny, Lx, Ly = 72, 60, 520.0, 470.0
    er = [C.circle(nx, ny, Lx, Ly, 140.0, 7.5, 1.0), C.lines_x(nx, ny, Lx, 200.0, 3.1, 1.4)]
    ur = [C.rect(nx, ny, Lx, Ly, 260.0, 150.0, 2.2, 1.0), C.circle(nx, ny, Lx, Ly, 90.0, 1.8, 1.0)]
    st = C.make_stack(Lx, Ly, er, [110.0, 70.0], ur)
    pb = C.Problem("m", st, [C.SourceSpec(745.0, 0.35, 0.6, 0.6, 0.8)], C.ParamSpec(3, 2, 1.0, 1.2, 2.25, 1.0))
    S, src, par = oracle_args(pb, 0)
    res = O.solve(S, src, par, rule=rule)
    assert abs(res.R_tot + res.T_tot - 1.0) < 1e-10
