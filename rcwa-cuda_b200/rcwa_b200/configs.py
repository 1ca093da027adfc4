"""Seeded synthetic layer stacks for the five workloads and the reference demo.

These are caller-side input builders: they rasterise permittivity grids in the
reference layout ``er[layer*Nx*Ny + iy*Nx + ix]`` (rcwa.hpp:56-60), sampled at
cell centres as in ``main.cpp:53-56``.

Loss convention: the reference uses ``e^{-jkz}`` so a lossy medium has
``Im(eps) < 0`` (rcwa.cpp:129-135; its lossy example at main.cpp:105 is
``6.0 - 0.13i``).  Workload descriptions quote loss as ``Im(eps) >= 0``
(e.g. ``15.1+0.2i``).  Every permittivity drawn or quoted here is conjugated
(:func:`ref_eps`) before it is written into a stack, so that lossy media decay.

Lengths are in nm; mu = 1 everywhere.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np


def ref_eps(eps) -> complex:
    """Quoted permittivity (loss as Im >= 0) -> reference convention (Im <= 0)."""
    return complex(np.conj(complex(eps)))


@dataclass
class StackSpec:
    """A layer stack in the reference's ``Device`` layout (rcwa.hpp:48-78)."""
    Nx: int
    Ny: int
    Lx: float
    Ly: float
    er: np.ndarray          # complex128, [num_layers*Ny*Nx]
    ur: np.ndarray          # complex128, [num_layers*Ny*Nx]
    t: np.ndarray           # float64, [num_layers]
    uniform: np.ndarray     # bool, [num_layers]: True when er and ur are constant

    @property
    def num_layers(self) -> int:
        return int(self.t.size)


@dataclass
class SourceSpec:
    """``Source`` (rcwa.hpp:81-95)."""
    lambda0: float
    theta: float
    phi: float
    pte: float
    ptm: float


@dataclass
class ParamSpec:
    """``RCWAParams`` (rcwa.hpp:98-112)."""
    nx_harmonics: int
    ny_harmonics: int
    er_ref: complex = 1.0 + 0.0j
    ur_ref: complex = 1.0 + 0.0j
    er_trn: complex = 2.25 + 0.0j
    ur_trn: complex = 1.0 + 0.0j


@dataclass
class Problem:
    """One or more solves that share a stack and harmonic orders (a sweep)."""
    name: str
    stack: StackSpec
    sources: List[SourceSpec]
    params: ParamSpec


# ----------------------------------------------------------------------------
# rasterisers (caller-side; sampled at cell centres)
# ----------------------------------------------------------------------------
def _centres(n: int, L: float) -> np.ndarray:
    return (np.arange(n) + 0.5) * (L / n)


def circle(Nx, Ny, Lx, Ly, r, eps_in, eps_out) -> np.ndarray:
    """Disc of radius ``r`` centred in the cell -> complex [Ny, Nx]."""
    x = _centres(Nx, Lx) - Lx / 2
    y = _centres(Ny, Ly) - Ly / 2
    inside = (x[None, :] ** 2 + y[:, None] ** 2) <= r * r
    return np.where(inside, complex(eps_in), complex(eps_out)).astype(np.complex128)


def lines_x(Nx, Ny, Lx, width, eps_line, eps_space) -> np.ndarray:
    """Lines running along y, ``width`` wide, centred in x -> [Ny, Nx]."""
    x = _centres(Nx, Lx) - Lx / 2
    inside = np.abs(x) <= width / 2
    g = np.where(inside, complex(eps_line), complex(eps_space))
    return np.broadcast_to(g[None, :], (Ny, Nx)).astype(np.complex128)


def rect(Nx, Ny, Lx, Ly, wx, wy, eps_in, eps_out) -> np.ndarray:
    """Centred wx x wy rectangle -> [Ny, Nx]."""
    x = _centres(Nx, Lx) - Lx / 2
    y = _centres(Ny, Ly) - Ly / 2
    inside = (np.abs(x[None, :]) <= wx / 2) & (np.abs(y[:, None]) <= wy / 2)
    return np.where(inside, complex(eps_in), complex(eps_out)).astype(np.complex128)


def uniform(Nx, Ny, eps) -> np.ndarray:
    return np.full((Ny, Nx), complex(eps), dtype=np.complex128)


def triangle_demo_grid(Nx, Ny, Lx, Ly) -> np.ndarray:
    """The reference demo's triangle of eps=2 in eps=6 (main.cpp:51-71)."""
    x = (np.arange(Nx) + 0.5) * Lx / Nx
    y = (np.arange(Ny) + 0.5) * Ly / Ny
    w = 0.8 * Ly
    xc, yc = Lx / 2.0, Ly / 2.0
    y_rel = y - (yc - w / 2.0)
    half_base = (w / 2.0) * (y_rel / w)
    inside = ((y_rel >= 0)[:, None] & (y_rel <= w)[:, None]
              & (np.abs(x[None, :] - xc) <= half_base[:, None]))
    return np.where(inside, 2.0 + 0j, 6.0 + 0j).astype(np.complex128)


def make_stack(Lx, Ly, grids: Sequence[np.ndarray], t: Sequence[float],
               ur_grids: Optional[Sequence[np.ndarray]] = None) -> StackSpec:
    Ny, Nx = grids[0].shape
    er = np.concatenate([np.asarray(g, np.complex128).reshape(-1) for g in grids])
    if ur_grids is None:
        ur = np.ones_like(er)
        ur_u = [True] * len(grids)
    else:
        ur = np.concatenate([np.asarray(g, np.complex128).reshape(-1) for g in ur_grids])
        ur_u = [bool(np.all(g == g.flat[0])) for g in ur_grids]
    uni = np.array([bool(np.all(g == g.flat[0])) and u for g, u in zip(grids, ur_u)])
    return StackSpec(Nx, Ny, float(Lx), float(Ly), er, ur, np.asarray(t, np.float64), uni)


# ----------------------------------------------------------------------------
# the workloads
# ----------------------------------------------------------------------------
def c1_pillars(grid: int = 512) -> Problem:
    """Single crossed grating: square lattice 500 nm, 200 nm layer of circular
    pillars r=125 nm, eps 12 in air, superstrate air, substrate 2.25, harmonics
    7x7 (N=49, n=98), lambda 600 nm, normal incidence, TE and TM."""
    g = circle(grid, grid, 500.0, 500.0, 125.0, 12.0, 1.0)
    st = make_stack(500.0, 500.0, [g], [200.0])
    srcs = [SourceSpec(600.0, 0.0, 0.0, 1.0, 0.0), SourceSpec(600.0, 0.0, 0.0, 0.0, 1.0)]
    return Problem("c1_pillars_h3", st, srcs, ParamSpec(3, 3, 1.0, 1.0, 2.25, 1.0))


def c2_eps(seed: int = 2) -> List[complex]:
    """Per-layer permittivities of the 3-layer stack: re U[2,16], im U[0,0.5]."""
    rng = np.random.default_rng(seed)
    re = rng.uniform(2.0, 16.0, size=3)
    im = rng.uniform(0.0, 0.5, size=3)
    return [ref_eps(complex(a, b)) for a, b in zip(re, im)]


def c2_sweep(n_lambda: int = 201, grid: int = 256, harmonics: int = 7,
             lambdas: Optional[Sequence[float]] = None) -> Problem:
    """3-layer stack, period 400x400: 1D line grating (50% duty, 120 nm), hole
    array r=100 nm (150 nm), uniform film (80 nm); eps per layer drawn with
    seed 2; harmonics 15x15 (N=225, n=450); grids 256^2; 201 wavelengths in
    [400, 800] nm; theta = 0; TM source (pte=0, ptm=1)."""
    L = 400.0
    e1, e2, e3 = c2_eps(2)
    g1 = lines_x(grid, grid, L, 0.5 * L, e1, 1.0)
    g2 = circle(grid, grid, L, L, 100.0, 1.0, e2)
    g3 = uniform(grid, grid, e3)
    st = make_stack(L, L, [g1, g2, g3], [120.0, 150.0, 80.0])
    lam = np.linspace(400.0, 800.0, n_lambda) if lambdas is None else np.asarray(lambdas, float)
    srcs = [SourceSpec(float(l), 0.0, 0.0, 0.0, 1.0) for l in lam]
    return Problem(f"c2_sweep_h{harmonics}", st, srcs, ParamSpec(harmonics, harmonics, 1.0, 1.0, 2.25, 1.0))


def c3_request(rng: np.random.Generator, grid: int = 256, m_max: int = 21, m_min: int = 5) -> Problem:
    """One solve of the uneven batch: odd M in m_min..m_max (h=(M-1)/2), 1-6 layers
    of pillar / hole / line-space, fill U[0.2,0.8], t U[20,300], square period
    U[300,800], lambda U[300,900], theta U[0,60 deg], phi U[0,90 deg],
    eps re U[1.5,16], im U[0,1]; superstrate air, substrate 2.25."""
    M = int(rng.choice(np.arange(m_min, m_max + 1, 2)))
    h = (M - 1) // 2
    L = int(rng.integers(1, 7))
    period = float(rng.uniform(300.0, 800.0))
    grids, ts = [], []
    for _ in range(L):
        kind = int(rng.integers(0, 3))
        fill = float(rng.uniform(0.2, 0.8))
        t = float(rng.uniform(20.0, 300.0))
        eps = ref_eps(complex(rng.uniform(1.5, 16.0), rng.uniform(0.0, 1.0)))
        if kind == 0:      # pillar of eps in air
            r = min(math.sqrt(fill * period * period / math.pi), period / 2)
            g = circle(grid, grid, period, period, r, eps, 1.0)
        elif kind == 1:    # air hole in an eps film
            r = min(math.sqrt(fill * period * period / math.pi), period / 2)
            g = circle(grid, grid, period, period, r, 1.0, eps)
        else:              # line-space along y
            g = lines_x(grid, grid, period, fill * period, eps, 1.0)
        grids.append(g)
        ts.append(t)
    lam = float(rng.uniform(300.0, 900.0))
    theta = math.radians(float(rng.uniform(0.0, 60.0)))
    phi = math.radians(float(rng.uniform(0.0, 90.0)))
    st = make_stack(period, period, grids, ts)
    src = SourceSpec(lam, theta, phi, 1.0 / math.sqrt(2.0), 1.0 / math.sqrt(2.0))
    return Problem(f"c3_M{M}_L{L}", st, [src], ParamSpec(h, h, 1.0, 1.0, 2.25, 1.0))


def c3_batch(count: int = 4096, seed: int = 3, grid: int = 256, m_max: int = 21) -> List[Problem]:
    rng = np.random.default_rng(seed)
    return [c3_request(rng, grid, m_max) for _ in range(count)]


C4_LINE_EPS = ref_eps(complex(12.0, 0.05))   # chosen line material (silicon-like)
C4_FILM_EPS = ref_eps(complex(2.1, 0.0))     # chosen film material (oxide-like)
C4_SUB_EPS = ref_eps(complex(15.1, 0.2))     # quoted substrate


def c4_trapezoid(M: int = 23, n_lambda: int = 64, grid: int = 512,
                 lambdas: Optional[Sequence[float]] = None) -> Problem:
    """Precision stress: crossed trapezoidal posts (pitch 90x90 nm, height 120
    nm, CD 45 nm at mid-height, sidewall 85 deg) staircased into 20 layers of
    6 nm, on a 10 nm film, over substrate 15.1+0.2i; harmonics M x M."""
    pitch, height, cd, swa = 90.0, 120.0, 45.0, math.radians(85.0)
    nsteps = 20
    dz = height / nsteps
    grids, ts = [], []
    for i in range(nsteps):              # layer 0 is the top of the post
        zc = height - (i + 0.5) * dz     # height of this slice above the film
        w = cd + 2.0 * (height / 2 - zc) / math.tan(swa)
        grids.append(rect(grid, grid, pitch, pitch, w, w, C4_LINE_EPS, 1.0))
        ts.append(dz)
    grids.append(uniform(grid, grid, C4_FILM_EPS))
    ts.append(10.0)
    st = make_stack(pitch, pitch, grids, ts)
    lam = np.linspace(250.0, 800.0, n_lambda) if lambdas is None else np.asarray(lambdas, float)
    srcs = [SourceSpec(float(l), 0.0, 0.0, 0.0, 1.0) for l in lam]
    h = (M - 1) // 2
    return Problem(f"c4_trap_M{M}", st, srcs, ParamSpec(h, h, 1.0, 1.0, C4_SUB_EPS, 1.0))


def demo_triangle(grid: int = 1024) -> Problem:
    """The reference's built-in case (main.cpp:37-109): triangle layer (t=0.5)
    plus a uniform eps=6 layer (t=0.3), Lx=1.75, Ly=1.5, h=3, eps_ref=2,
    eps_trn=9, lambda0=2, normal incidence, TM."""
    Lx, Ly = 1.75, 1.5
    g0 = triangle_demo_grid(grid, grid, Lx, Ly)
    g1 = uniform(grid, grid, 6.0)
    st = make_stack(Lx, Ly, [g0, g1], [0.5, 0.3])
    return Problem("reference_demo", st, [SourceSpec(2.0, 0.0, 0.0, 0.0, 1.0)],
                   ParamSpec(3, 3, 2.0, 1.0, 9.0, 1.0))


def poisson_arrivals(rate_hz: float, count: int, seed: int = 5) -> np.ndarray:
    """Arrival times (s) of a Poisson stream."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=count))
