"""Li's factorization rule on the GPU (rcwa_geometry_create_ex with
RCWA_GEOM_LI_RULE) against the oracle's li_conv_mat path, through the C-ABI."""
import dataclasses
import math

import numpy as np
import pytest

from helpers import oracle_args
from oracle import rcwa_oracle as O
from rcwa_b200 import configs as C
from rcwa_b200 import lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-10   # |dR|, |dT| per order, as for the Laurent-rule parity


@pytest.fixture(scope="module")
def ctx():
    c = L.Context(0)
    yield c
    c.close()


def _device_sweep(ctx, pb, rule):
    import torch
    g = ctx.geometry_create(pb.stack, pb.params, rule=rule)
    B = len(pb.sources)
    N = (2 * pb.params.nx_harmonics + 1) * (2 * pb.params.ny_harmonics + 1)
    R = torch.empty(B * N, dtype=torch.float64, device="cuda")
    T = torch.empty_like(R)
    tot = torch.empty(2 * B, dtype=torch.float64, device="cuda")
    st = torch.empty(B, dtype=torch.int32, device="cuda")
    try:
        ctx.solve_sweep_device(g, pb.sources, L.PREC_FP64, R.data_ptr(), T.data_ptr(), tot.data_ptr(),
                               st.data_ptr())
        ctx.synchronize()
    finally:
        ctx.geometry_destroy(g)
    P, Q = 2 * pb.params.nx_harmonics + 1, 2 * pb.params.ny_harmonics + 1
    R = R.cpu().numpy().reshape(B, P, Q).transpose(0, 2, 1)
    T = T.cpu().numpy().reshape(B, P, Q).transpose(0, 2, 1)
    return R, T, st.cpu().numpy()


def _oracle(pb, rule):
    S, _, par = oracle_args(pb, 0)
    convs = O.conv_mats(S, par, rule)
    return [O.solve(S, oracle_args(pb, i)[1], par, convs=convs) for i in range(len(pb.sources))]


def _crossed():
    nx, ny, Lx, Ly = 64, 48, 620.0, 540.0
    grids = [C.circle(nx, ny, Lx, Ly, 160.0, 11.5 - 0.1j, 1.0 + 0.0j),
             C.uniform(nx, ny, 2.1 + 0.0j),
             C.rect(nx, ny, Lx, Ly, 300.0, 180.0, -9.0 - 1.5j, 2.25 + 0.0j)]
    st = C.make_stack(Lx, Ly, grids, [95.0, 40.0, 60.0])
    srcs = [C.SourceSpec(lam, th, ph, 0.6, 0.8)
            for lam, th, ph in ((710.0, 0.0, 0.0), (655.0, 0.31, 0.2), (820.0, 0.45, 1.1))]
    return C.Problem("crossed", st, srcs, C.ParamSpec(3, 2, 1.0, 1.0, 2.25, 1.0))


def test_crossed_grating_li_matches_oracle(ctx):
    pb = _crossed()
    R, T, st = _device_sweep(ctx, pb, "li")
    assert not st.any()
    ref = _oracle(pb, "li")
    for i, r in enumerate(ref):
        assert np.abs(R[i] - r.R).max() <= TOL
        assert np.abs(T[i] - r.T).max() <= TOL
    # and the rule is in effect: Laurent differs by more than the tolerance
    Rl, Tl, _ = _device_sweep(ctx, pb, "laurent")
    assert np.abs(Rl - R).max() > 1e-4


@pytest.mark.parametrize("axis", ["x", "y"])
def test_lamellar_tm_li_matches_oracle(ctx, axis):
    """Metal lines along one axis: exercises the row (x) and the strided
    column (y) line pass, with 1-point lines on the other axis."""
    n = 600
    line = C.lines_x(n, 1, 1000.0, 500.0, -20.0 - 2.0j, 1.0 + 0.0j)     # varies along x
    if axis == "x":
        nx, ny, grid, h, phi = n, 1, line, (18, 0), 0.0
    else:
        nx, ny, grid, h, phi = 1, n, np.ascontiguousarray(line.T), (0, 18), math.pi / 2
    st = C.make_stack(1000.0, 1000.0, [grid], [250.0])
    # TM in the plane of incidence that crosses the lines
    srcs = [C.SourceSpec(800.0, math.radians(10.0), phi, 0.0, 1.0),
            C.SourceSpec(930.0, math.radians(25.0), phi, 0.0, 1.0)]
    pb = C.Problem("lamellar", st, srcs, C.ParamSpec(*h, 1.0, 1.0, 2.25, 1.0))
    R, T, stat = _device_sweep(ctx, pb, "li")
    assert not stat.any()
    for i, r in enumerate(_oracle(pb, "li")):
        assert np.abs(R[i] - r.R).max() <= TOL
        assert np.abs(T[i] - r.T).max() <= TOL


def test_li_rule_errors(ctx):
    pb = _crossed()
    er = pb.stack.er.copy()
    er[5] = 0.0                      # a zero permittivity in a patterned layer
    bad = dataclasses.replace(pb.stack, er=er)
    with pytest.raises(L.RcwaError, match="Li rule"):
        ctx.geometry_create(bad, pb.params, rule="li")
    # the context stays usable, and the Laurent rule accepts the same grid
    g = ctx.geometry_create(bad, pb.params)
    ctx.geometry_destroy(g)
    import ctypes as Ct
    h = Ct.c_void_p()
    st = pb.stack
    keep = (L._c128(st.er), L._c128(st.ur), np.ascontiguousarray(st.t, dtype=np.float64))
    cst = L.CStack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, *(L._ptr(a) for a in keep))
    prm = L.c_params(pb.params)
    rc = ctx.lib.rcwa_geometry_create_ex(ctx.h, Ct.byref(cst), Ct.byref(prm), 0, 6, Ct.byref(h))
    assert rc == L.RCWA_ERR_INVALID
