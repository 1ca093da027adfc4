"""Closed-form zero-order R/T of a stack of homogeneous layers (characteristic
matrix method, Macleod's e^{i(wt-kz)} convention, which is the reference's
e^{-jkz} convention with loss as Im(eps) < 0).  Independent of the RCWA code:
used to pin the oracle and the GPU path on uniform stacks."""
from __future__ import annotations

import cmath
import math
from typing import Sequence

import numpy as np


def _kz(eps: complex, kx: float, mu: complex = 1.0) -> complex:
    """Normalised kz = sqrt(eps mu - kx^2) with Re >= 0 and Im <= 0 (forward,
    decaying for e^{-jkz})."""
    k = cmath.sqrt(complex(eps) * complex(mu) - kx * kx)
    if k.imag > 0 or (k.imag == 0 and k.real < 0):
        k = -k
    return k


def thin_film_rt(eps_layers: Sequence[complex], d: Sequence[float], eps_in: complex,
                 eps_out: complex, lambda0: float, theta: float, pol: str,
                 mu_layers: Sequence[complex] = None, mu_in: complex = 1.0, mu_out: complex = 1.0):
    """Return (R, T) for s ('TE') or p ('TM') polarisation; mu = 1 unless
    given (tangential admittances kz / mu for TE, eps / kz for TM)."""
    mu_layers = [1.0] * len(eps_layers) if mu_layers is None else mu_layers
    n_in = cmath.sqrt(complex(eps_in) * complex(mu_in))
    kx = (n_in * math.sin(theta)).real
    k0 = 2 * math.pi / lambda0

    def adm(eps, mu):
        kz = _kz(eps, kx, mu)
        return kz / complex(mu) if pol == "TE" else complex(eps) / kz

    M = np.eye(2, dtype=np.complex128)
    for eps, mu, dd in zip(eps_layers, mu_layers, d):
        kz = _kz(eps, kx, mu)
        eta = adm(eps, mu)
        delta = k0 * dd * kz
        Mj = np.array([[cmath.cos(delta), 1j * cmath.sin(delta) / eta],
                       [1j * eta * cmath.sin(delta), cmath.cos(delta)]])
        M = M @ Mj
    eta0, etam = adm(eps_in, mu_in), adm(eps_out, mu_out)
    B, C = M @ np.array([1.0, etam])
    r = (eta0 * B - C) / (eta0 * B + C)
    R = abs(r) ** 2
    T = 4 * eta0.real * etam.real / abs(eta0 * B + C) ** 2
    return float(R), float(T)
