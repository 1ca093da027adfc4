"""Pins for the oracle's Li factorization rule (an option beside the
reference's Laurent-rule ConvMat, rcwa.cpp:6-82), CPU only: the limits in
which the rule must reduce to Laurent / to a 1-D inverse rule, TE invariance
of a lamellar grating and the faster TM convergence the rule exists for."""
import math

import numpy as np
import pytest

from oracle import rcwa_oracle as O
from rcwa_b200 import configs as C


def _toeplitz_1d(f, n, P):
    """1-D Toeplitz matrix (P x P) of the DFT coefficients of f (length n)."""
    a = np.fft.fft(f) / n
    d = np.arange(P)[:, None] - np.arange(P)[None, :]
    return a[d % n]


def test_x_grating_reduces_to_inverse_and_laurent_rules():
    Nx, Ny, h = 64, 8, (4, 2)
    g = C.lines_x(Nx, Ny, 500.0, 210.0, 9.0 - 0.4j, 1.5 + 0.0j).ravel()
    P, Q = 2 * h[0] + 1, 2 * h[1] + 1
    exx = O.li_conv_mat(g, 0, Nx, Ny, *h, "x")
    eyy = O.li_conv_mat(g, 0, Nx, Ny, *h, "y")
    # E_y is tangential to the walls: Laurent, i.e. the reference's ConvMat
    lau = O.conv_mat(g, 0, Nx, Ny, *h)
    assert np.abs(eyy - lau).max() < 1e-13
    # E_x crosses the walls: inverse of the Toeplitz matrix of 1/eps, no y coupling
    row = g.reshape(Ny, Nx)[0]
    inv = np.linalg.inv(_toeplitz_1d(1.0 / row, Nx, P))
    assert np.abs(exx - np.kron(inv, np.eye(Q))).max() < 1e-12
    # and the two rules genuinely differ here
    assert np.abs(exx - lau).max() > 1e-2


def test_y_grating_mirrors_x_grating():
    Nx, Ny, h = 8, 64, (2, 4)
    gx = C.lines_x(Ny, Nx, 500.0, 210.0, 9.0 - 0.4j, 1.5 + 0.0j)      # [Nx][Ny]: lines along x
    gy = np.ascontiguousarray(gx.T).ravel()                             # transpose: lines along y
    P, Q = 2 * h[0] + 1, 2 * h[1] + 1
    eyy = O.li_conv_mat(gy, 0, Nx, Ny, *h, "y")
    exx = O.li_conv_mat(gy, 0, Nx, Ny, *h, "x")
    col = gy.reshape(Ny, Nx)[:, 0]
    inv = np.linalg.inv(_toeplitz_1d(1.0 / col, Ny, Q))
    assert np.abs(eyy - np.kron(np.eye(P), inv)).max() < 1e-12
    assert np.abs(exx - O.conv_mat(gy, 0, Nx, Ny, *h)).max() < 1e-13


def test_uniform_and_crossed_grids():
    Nx, Ny, h = 48, 40, (3, 2)
    eps = 3.3 - 0.2j
    g = np.full(Nx * Ny, eps)
    N = (2 * h[0] + 1) * (2 * h[1] + 1)
    for ax in ("x", "y"):
        assert np.abs(O.li_conv_mat(g, 0, Nx, Ny, *h, ax) - eps * np.eye(N)).max() < 1e-14
    # a pillar: both components differ from Laurent, the matrices stay
    # finite, and x <-> y swap under a transposed grid
    gp = C.circle(Nx, Nx, 600.0, 600.0, 170.0, 11.0 + 0.0j, 1.0 + 0.0j)
    exx = O.li_conv_mat(gp.ravel(), 0, Nx, Nx, 3, 3, "x")
    eyy_t = O.li_conv_mat(np.ascontiguousarray(gp.T).ravel(), 0, Nx, Nx, 3, 3, "y")
    Pn = 7
    perm = (np.arange(Pn * Pn) % Pn) * Pn + np.arange(Pn * Pn) // Pn   # (p, q) -> (q, p)
    assert np.isfinite(exx).all()
    assert np.abs(exx - eyy_t[np.ix_(perm, perm)]).max() < 1e-12
    lau = O.conv_mat(gp.ravel(), 0, Nx, Nx, 3, 3)
    assert np.abs(exx - lau).max() > 1e-2


def _lamellar(rule, h, pol):
    Nx = 1200
    g = C.lines_x(Nx, 1, 1000.0, 500.0, -20.0 - 2.0j, 1.0 + 0.0j).ravel()   # lossy metal lines
    S = O.Stack(Nx, 1, 1, 1000.0, 1000.0, g, np.ones(Nx, complex), np.array([250.0]))
    par = O.Params(h, 0, 1.0, 1.0, 2.25, 1.0)
    pte, ptm = (1.0, 0.0) if pol == "TE" else (0.0, 1.0)
    src = O.Source(800.0, math.radians(10.0), 0.0, pte, ptm)
    return O.solve(S, src, par, rule=rule)


def test_lamellar_te_is_rule_independent():
    a, b = _lamellar("laurent", 12, "TE"), _lamellar("li", 12, "TE")
    assert abs(a.R_tot - b.R_tot) < 1e-12 and abs(a.T_tot - b.T_tot) < 1e-12


@pytest.mark.parametrize("h", [25, 35])
def test_lamellar_tm_converges_faster_with_li(h):
    ref = _lamellar("li", 60, "TM").R_tot
    e_li = abs(_lamellar("li", h, "TM").R_tot - ref)
    e_lau = abs(_lamellar("laurent", h, "TM").R_tot - ref)
    assert e_li < 0.3 * e_lau, (e_li, e_lau)
