"""Magnetic media and the empty stack through the C-ABI against the oracle
and the closed-form thin-film R/T: patterned permeability grids (the urc /
urc^-1 terms of rcwa.cpp:274-285, under both factorization rules),
permeability in the half-spaces (rcwa.cpp:361-372, 421-432, 579-582), and a
stack without layers (S_device = S_init, rcwa.cpp:237-250)."""
import math

import numpy as np
import pytest

from helpers import oracle_args
from oracle import rcwa_oracle as O
from rcwa_b200 import configs as C
from rcwa_b200 import lib as L
from thinfilm import thin_film_rt

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def ctx():
    c = L.Context(0)
    yield c
    c.close()


def _oracle_all(pb, rule="laurent"):
    S, _, par = oracle_args(pb, 0)
    convs = O.conv_mats(S, par, rule)
    return [O.solve(S, oracle_args(pb, i)[1], par, convs=convs) for i in range(len(pb.sources))]


@pytest.mark.parametrize("pol", ["TE", "TM"])
def test_magnetic_uniform_stack_thin_film(ctx, pol):
    eps = [4.0, 2.2 - 0.3j, 9.5 - 0.05j]
    mus = [1.7, 2.5 - 0.1j, 1.0]
    d = [120.0, 75.0, 33.0]
    st = C.make_stack(700.0, 650.0, [C.uniform(16, 16, e) for e in eps], d,
                      [C.uniform(16, 16, m) for m in mus])
    pte, ptm = (1.0, 0.0) if pol == "TE" else (0.0, 1.0)
    ths = (0.0, 20.0, 47.0)
    srcs = [C.SourceSpec(633.0, math.radians(th), 0.0, pte, ptm) for th in ths]
    pb = C.Problem("mu", st, srcs, C.ParamSpec(2, 2, 1.0, 1.3, 2.25, 1.6))
    R, T, Rt, Tt, stat = ctx.solve_sweep(pb)
    assert not stat.any()
    for i, th in enumerate(ths):
        Rf, Tf = thin_film_rt(eps, d, 1.0, 2.25, 633.0, math.radians(th), pol, mus, 1.3, 1.6)
        assert abs(Rt[i] - Rf) < 1e-11 and abs(Tt[i] - Tf) < 1e-11


@pytest.mark.parametrize("rule", ["laurent", "li"])
def test_patterned_permeability_matches_oracle(ctx, rule):
    nx, ny, Lx, Ly = 72, 60, 520.0, 470.0
    er = [C.circle(nx, ny, Lx, Ly, 140.0, 7.5 - 0.2j, 1.0 + 0.0j),
          C.lines_x(nx, ny, Lx, 200.0, 3.1 + 0.0j, 1.4 + 0.0j)]
    ur = [C.rect(nx, ny, Lx, Ly, 260.0, 150.0, 2.2 - 0.05j, 1.0 + 0.0j),
          C.circle(nx, ny, Lx, Ly, 90.0, 1.8 + 0.0j, 1.0 + 0.0j)]
    st = C.make_stack(Lx, Ly, er, [110.0, 70.0], ur)
    srcs = [C.SourceSpec(lam, th, ph, 0.6, 0.8)
            for lam, th, ph in ((690.0, 0.0, 0.0), (745.0, 0.35, 0.6))]
    pb = C.Problem("mu-pat", st, srcs, C.ParamSpec(3, 2, 1.0, 1.2, 2.25, 1.0))
    import torch
    g = ctx.geometry_create(pb.stack, pb.params, rule=rule)
    B, P, Q = len(srcs), 7, 5
    Rd = torch.empty(B * P * Q, dtype=torch.float64, device="cuda")
    Td = torch.empty_like(Rd)
    tot = torch.empty(2 * B, dtype=torch.float64, device="cuda")
    sd = torch.empty(B, dtype=torch.int32, device="cuda")
    try:
        ctx.solve_sweep_device(g, srcs, L.PREC_FP64, Rd.data_ptr(), Td.data_ptr(), tot.data_ptr(), sd.data_ptr())
        ctx.synchronize()
    finally:
        ctx.geometry_destroy(g)
    assert not sd.cpu().numpy().any()
    R = Rd.cpu().numpy().reshape(B, P, Q).transpose(0, 2, 1)
    T = Td.cpu().numpy().reshape(B, P, Q).transpose(0, 2, 1)
    for i, r in enumerate(_oracle_all(pb, rule)):
        assert np.abs(R[i] - r.R).max() <= TOL
        assert np.abs(T[i] - r.T).max() <= TOL


def test_empty_stack_is_a_bare_interface(ctx):
    st = C.StackSpec(16, 16, 400.0, 400.0, np.zeros(0, np.complex128), np.zeros(0, np.complex128),
                     np.zeros(0), np.zeros(0, bool))
    ths = (0.0, 30.0)
    srcs = [C.SourceSpec(633.0, math.radians(th), 0.0, 0.0, 1.0) for th in ths]
    pb = C.Problem("bare", st, srcs, C.ParamSpec(1, 1, 1.0, 1.0, 2.25, 1.0))
    R, T, Rt, Tt, stat = ctx.solve_sweep(pb)
    assert not stat.any()
    for i, th in enumerate(ths):
        ref = O.solve(*oracle_args(pb, i), rule="laurent")
        assert np.abs(R[i] - ref.R).max() <= TOL and np.abs(T[i] - ref.T).max() <= TOL
        Rf, Tf = thin_film_rt([], [], 1.0, 2.25, 633.0, math.radians(th), "TM")
        assert abs(Rt[i] - Rf) < 1e-11 and abs(Tt[i] - Tf) < 1e-11
