"""Device-side rasterisers (rcwa_rasterize, rcwa_geometry_create_shapes)
through the C ABI: grids bit-identical to the host builders of
rcwa_b200.configs, and a geometry built from shapes alone solves to the same
R/T as the one built from host grids (the same device computation, so to
1e-13)."""
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


def _layers_and_grids(nx, ny, Lx, Ly):
    from rcwa_b200 import lib as L
    e1, e2, e3 = C.ref_eps(12.0 + 0.1j), C.ref_eps(6.5 + 0.3j), C.ref_eps(3.1)
    layers = [
        (1.0, 1.0, 110.0, [(L.SHAPE_CIRCLE, 0.0, 0.0, 0.3 * Lx, 0.0, e1, 1.0)]),      # pillar
        (e2, 1.0, 70.0, [(L.SHAPE_CIRCLE, 0.0, 0.0, 0.22 * Lx, 0.0, 1.0, 1.0)]),      # hole
        (1.0, 1.0, 90.0, [(L.SHAPE_LINES, 0.0, 0.0, 0.45 * Lx, 0.0, e3, 1.0)]),       # line-space
        (1.0, 1.0, 50.0, [(L.SHAPE_RECT, 0.0, 0.0, 0.5 * Lx, 0.3 * Ly, e1, 1.0)]),    # rectangle
        (6.0, 1.0, 30.0, [(L.SHAPE_TRIANGLE, 0.0, 0.0, 0.8 * Ly, 0.0, 2.0, 1.0)]),   # reference demo
    ]
    grids = [C.circle(nx, ny, Lx, Ly, 0.3 * Lx, e1, 1.0),
             C.circle(nx, ny, Lx, Ly, 0.22 * Lx, 1.0, e2),
             C.lines_x(nx, ny, Lx, 0.45 * Lx, e3, 1.0),
             C.rect(nx, ny, Lx, Ly, 0.5 * Lx, 0.3 * Ly, e1, 1.0),
             C.triangle_demo_grid(nx, ny, Lx, Ly)]
    return layers, grids


@pytest.mark.parametrize("nx,ny,Lx,Ly", [(128, 128, 500.0, 500.0), (97, 64, 430.0, 360.0), (256, 256, 1.75, 1.5)])
def test_rasterize_matches_host_builders(ctx, nx, ny, Lx, Ly):
    import torch
    layers, grids = _layers_and_grids(nx, ny, Lx, Ly)
    nl = len(layers)
    er = torch.empty(nl * ny * nx * 2, dtype=torch.float64, device="cuda")
    ur = torch.empty_like(er)
    t = torch.empty(nl, dtype=torch.float64, device="cuda")
    ctx.rasterize(nx, ny, Lx, Ly, layers, er.data_ptr(), ur.data_ptr(), t.data_ptr())
    ctx.synchronize()
    er_h = er.cpu().numpy().view(np.complex128).reshape(nl, ny, nx)
    ur_h = ur.cpu().numpy().view(np.complex128).reshape(nl, ny, nx)
    for l in range(nl):
        assert np.array_equal(er_h[l], grids[l]), l
        assert np.all(ur_h[l] == 1.0)
    assert np.array_equal(t.cpu().numpy(), [ly[2] for ly in layers])


def test_geometry_from_shapes_solves_like_host_grids(ctx):
    import torch
    nx = ny = 128
    Lx = Ly = 500.0
    layers, grids = _layers_and_grids(nx, ny, Lx, Ly)
    layers, grids = layers[:3], grids[:3]
    st = C.make_stack(Lx, Ly, grids, [ly[2] for ly in layers])
    par = C.ParamSpec(3, 3, 1.0, 1.0, 2.25, 1.0)
    srcs = [C.SourceSpec(lam, 0.2, 0.4, 0.6, 0.8) for lam in (520.0, 610.0, 700.0)]
    B, N = len(srcs), 49
    out = []
    for g in (ctx.geometry_create(st, par), ctx.geometry_create_shapes(nx, ny, Lx, Ly, layers, par)):
        R = torch.empty(B * N, dtype=torch.float64, device="cuda")
        T = torch.empty_like(R)
        tot = torch.empty(2 * B, dtype=torch.float64, device="cuda")
        s = torch.empty(B, dtype=torch.int32, device="cuda")
        from rcwa_b200 import lib as L
        ctx.solve_sweep_device(g, srcs, L.PREC_FP64, R.data_ptr(), T.data_ptr(), tot.data_ptr(), s.data_ptr())
        ctx.synchronize()
        ctx.geometry_destroy(g)
        out.append((R.cpu().numpy(), T.cpu().numpy(), s.cpu().numpy()))
    assert not out[0][2].any() and not out[1][2].any()
    assert np.abs(out[0][0] - out[1][0]).max() <= 1e-13
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-13
