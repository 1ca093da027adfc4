"""Generates the golden fixtures of this directory from the CPU oracle.

    python tests/golden/make_golden.py        (from the repository root)

The reference (rcwa.cpp / main.cpp) builds only against Eigen3, which this
environment lacks, and its repository holds no expected values; these
fixtures therefore record the oracle's own output on small seeded cases.
They pin later changes of the oracle (tests/test_oracle.py) and let the GPU
tests check the CUDA path against stored numbers without running the oracle
(tests/test_gpu_parity.py).  The oracle itself is pinned by the physics
known-answer tests in tests/test_oracle.py.

Cases:
  golden_small_c1     C1's geometry (circular pillars r=125 nm, eps 12, 500 nm
                      lattice, 200 nm) on a 128^2 grid, h = 2, lambda 600 nm,
                      TE and TM at normal incidence plus one oblique source.
  golden_small_mixed  two patterned layers (line grating along x, rectangular
                      hole) and one uniform film, lossy eps (Im < 0 in the
                      reference convention), rectangular period 420 x 380 nm,
                      h = (3, 2), a 96 x 80 grid, three oblique sources.
  golden_c4_m23       the C4 precision-stress stack (20-step staircased
                      trapezoidal posts on a film over a lossy substrate,
                      rcwa_b200.configs.c4_trapezoid) at M = 23 (n = 1058),
                      512 x 512 grids, one wavelength (600 nm), TM.
  golden_c4_m23_sweep the same stack at 250, 430 and 800 nm (the ends and the
                      middle of the C4 band).
  golden_c4_m31       the same stack at the largest C4 order, M = 31
                      (n = 1922), at 300 and 700 nm.
  golden_c3_full_<i>  requests i = 0, 1, 2 of the C3 distribution restricted
                      to its largest orders (odd M in 15..21, n = 450..882),
                      256 x 256 grids, drawn with numpy default_rng(2121).

    python tests/golden/make_golden.py golden_c4_m31   (one case)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "rcwa-cuda_b200"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

from rcwa_b200 import configs as C  # noqa: E402

CASES = ("golden_small_c1", "golden_small_mixed", "golden_c4_m23", "golden_c4_m23_sweep", "golden_c4_m31",
         "golden_c3_full_0", "golden_c3_full_1", "golden_c3_full_2")


def build_case(name: str) -> C.Problem:
    if name == "golden_small_c1":
        g = C.circle(128, 128, 500.0, 500.0, 125.0, 12.0, 1.0)
        st = C.make_stack(500.0, 500.0, [g], [200.0])
        srcs = [C.SourceSpec(600.0, 0.0, 0.0, 1.0, 0.0),
                C.SourceSpec(600.0, 0.0, 0.0, 0.0, 1.0),
                C.SourceSpec(640.0, np.radians(17.0), np.radians(30.0), 0.6, 0.8)]
        return C.Problem(name, st, srcs, C.ParamSpec(2, 2, 1.0, 1.0, 2.25, 1.0))
    if name == "golden_small_mixed":
        Nx, Ny, Lx, Ly = 96, 80, 420.0, 380.0
        e1, e2, e3 = (C.ref_eps(complex(11.7, 0.3)), C.ref_eps(complex(6.2, 0.8)),
                      C.ref_eps(complex(2.1, 0.02)))
        g1 = C.lines_x(Nx, Ny, Lx, 0.45 * Lx, e1, 1.0)
        g2 = C.rect(Nx, Ny, Lx, Ly, 0.5 * Lx, 0.35 * Ly, 1.0, e2)
        g3 = C.uniform(Nx, Ny, e3)
        st = C.make_stack(Lx, Ly, [g1, g2, g3], [95.0, 140.0, 60.0])
        srcs = [C.SourceSpec(530.0, np.radians(12.0), np.radians(25.0), 1.0, 0.0),
                C.SourceSpec(610.0, np.radians(33.0), np.radians(70.0), 0.0, 1.0),
                C.SourceSpec(745.0, np.radians(5.0), 0.0, 0.7071067811865476, 0.7071067811865476)]
        return C.Problem(name, st, srcs,
                         C.ParamSpec(3, 2, 1.0, 1.0, C.ref_eps(complex(2.25, 0.01)), 1.0))
    if name == "golden_c4_m23":
        return C.c4_trapezoid(M=23, lambdas=[600.0])
    if name == "golden_c4_m23_sweep":
        return C.c4_trapezoid(M=23, lambdas=[250.0, 430.0, 800.0])
    if name == "golden_c4_m31":
        return C.c4_trapezoid(M=31, lambdas=[300.0, 700.0])
    if name.startswith("golden_c3_full_"):
        i = int(name.rsplit("_", 1)[1])
        rng = np.random.default_rng(2121)
        pbs = [C.c3_request(rng, grid=256, m_max=21, m_min=15) for _ in range(i + 1)]
        return pbs[i]
    raise KeyError(name)


def main() -> None:
    from helpers import oracle_sweep
    for name in (sys.argv[1:] or CASES):
        pb = build_case(name)
        res = oracle_sweep(pb)
        np.savez_compressed(os.path.join(HERE, name + ".npz"),
                            R=np.array([r.R for r in res]), T=np.array([r.T for r in res]),
                            R_tot=np.array([r.R_tot for r in res]),
                            T_tot=np.array([r.T_tot for r in res]))
        print(name, [round(r.R_tot, 6) for r in res], [round(r.T_tot, 6) for r in res])


if __name__ == "__main__":
    main()
