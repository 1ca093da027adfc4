"""FP64 CPU oracle for the RCWA solve path -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product path (``rcwa_b200`` / ``librcwa_b200.so``) never calls into it.

It is a step-for-step NumPy/SciPy restatement of the reference solver
(``rcwa3d/src/rcwa.cpp`` driven by ``rcwa3d/src/main.cpp:111-191``), with the
reference's conventions kept exactly:

* complex128 everywhere (``rcwa3d/include/rcwa.hpp:11-17``);
* mode index ``m = ix*Q + iy`` (x slow, y fast), ``rcwa.cpp:63-64``;
* ``e^{-jkz}`` forward convention, loss means ``Im(eps) < 0``
  (``rcwa.cpp:129-135``);
* outputs ``R``/``T`` are Q x P arrays (``rcwa.cpp:576, 582``).

Parity status: the reference needs Eigen3 (``rcwa3d/CMakeLists.txt:7``), which
is not present on this machine, so the reference cannot be compiled and no
golden vectors exist in it.  Parity against the reference binary is therefore
UNPINNED.  The restatement is instead pinned to closed-form physics
(Fresnel/Airy thin-film formulas, energy conservation, symmetry and
eigen-basis invariance) in ``tests/test_oracle.py``.

Eigen call sites and their restatement here:

==========================  =====================================  ==========================
reference                   Eigen routine (version not pinned)     restatement
==========================  =====================================  ==========================
rcwa.cpp:24-41              Eigen::FFT fwd (kissfft), then /NxNy    numpy.fft.fft2 / (Nx*Ny)
rcwa.cpp:44-53              hand-written block swap                 numpy.fft.fftshift
``.lu().solve``             PartialPivLU                            scipy.linalg.lu_factor/solve
rcwa.cpp:298                ComplexEigenSolver (Schur + vectors)    scipy.linalg.eig (zgeev)
rcwa.cpp:339                Array exp                               numpy.exp
==========================  =====================================  ==========================

Eigenvalue order and eigenvector phases differ between Eigen and LAPACK; the
layer S-matrix is invariant under ``W -> W M`` for any permutation / (block-)
diagonal ``M`` because ``A``, ``B`` and ``A - X B A^-1 X B`` all left-multiply by
``M^-1`` which cancels in S11 and S12 (rcwa.cpp:335-348).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field as dc_field
from typing import List, Sequence

import numpy as np
import scipy.linalg as sla

__all__ = [
    "unsigned_sqrt", "conv_mat", "compute_wave_vectors", "gap_medium",
    "smatrix_init", "smatrix_layer", "smatrix_reflection",
    "smatrix_transmission", "redheffer_product", "source_mode_coeff",
    "reflected_field", "transmitted_field", "diffraction_efficiencies",
    "solve", "Stack", "Source", "Params", "Results", "SMatrix", "li_conv_mat",
]


# ----------------------------------------------------------------------------
# data model (rcwa.hpp:48-162)
# ----------------------------------------------------------------------------
@dataclass
class Stack:
    """``Device`` (rcwa.hpp:48-78): grids ``er``/``ur`` flat ``[layer][iy][ix]``."""
    Nx: int
    Ny: int
    num_layers: int
    Lx: float
    Ly: float
    er: np.ndarray
    ur: np.ndarray
    t: np.ndarray


@dataclass
class Source:
    """``Source`` (rcwa.hpp:81-95); k0 = 2*pi/lambda0 (rcwa.hpp:92)."""
    lambda0: float
    theta: float
    phi: float
    pte: float
    ptm: float

    @property
    def k0(self) -> float:
        return 2.0 * math.pi / self.lambda0


@dataclass
class Params:
    """``RCWAParams`` (rcwa.hpp:98-112)."""
    Nx_harmonics: int
    Ny_harmonics: int
    er_ref: complex
    ur_ref: complex
    er_trn: complex
    ur_trn: complex


@dataclass
class SMatrix:
    """``ScatteringMatrix`` (rcwa.hpp:132-162)."""
    S11: np.ndarray
    S12: np.ndarray
    S21: np.ndarray
    S22: np.ndarray


@dataclass
class Results:
    """``Results`` (rcwa.hpp:116-128): R, T are Q x P."""
    R: np.ndarray
    T: np.ndarray
    R_tot: float
    T_tot: float


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------
def unsigned_sqrt(z):
    """rcwa.hpp:24-28, 37-44: principal sqrt after turning an imaginary -0 into +0."""
    z = np.asarray(z, dtype=np.complex128)
    z = np.where(z.imag == 0.0, z.real + 0.0j, z)
    return np.sqrt(z)


def _lu_solve(A, B):
    """``A.lu().solve(B)`` -- Eigen PartialPivLU restated with LAPACK getrf/getrs."""
    return sla.lu_solve(sla.lu_factor(A, check_finite=False), B, check_finite=False)


# ----------------------------------------------------------------------------
# step functions (rcwa.cpp)
# ----------------------------------------------------------------------------
def conv_mat(field, layer, Nx, Ny, Nx_harmonics, Ny_harmonics):
    """rcwa.cpp:6-82 -- PQ x PQ Toeplitz convolution matrix of one layer's grid."""
    F = np.asarray(field, dtype=np.complex128)[layer * Nx * Ny:(layer + 1) * Nx * Ny]
    F = F.reshape(Ny, Nx)                              # row-major map, rcwa.cpp:16-21
    F = np.fft.fft2(F) / float(Nx * Ny)                # rcwa.cpp:24-41
    Fs = np.fft.fftshift(F)                            # rcwa.cpp:44-53
    P = 2 * Nx_harmonics + 1
    Q = 2 * Ny_harmonics + 1
    PQ = P * Q
    m = np.arange(PQ)
    px = m // Q - Nx_harmonics                         # x slow, rcwa.cpp:63
    py = m % Q - Ny_harmonics                          # y fast, rcwa.cpp:64
    kx = px[:, None] - px[None, :] + Nx // 2           # rcwa.cpp:71
    ky = py[:, None] - py[None, :] + Ny // 2           # rcwa.cpp:72
    ok = (kx >= 0) & (kx < Nx) & (ky >= 0) & (ky < Ny)  # rcwa.cpp:73
    C = np.zeros((PQ, PQ), dtype=np.complex128)
    C[ok] = Fs[ky[ok], kx[ok]]
    return C


def _dft_1d(lines, n, K):
    """Coefficients k = -K..K of the 1-D DFT of each row of ``lines`` (last axis,
    length n), divided by n; 0 where k + n//2 lies outside [0, n), the range
    rule of rcwa.cpp:71-73 applied to one axis."""
    F = np.fft.fft(lines, axis=-1) / float(n)
    k = np.arange(-K, K + 1)
    out = F[..., k % n]
    out[..., (k + n // 2 < 0) | (k + n // 2 >= n)] = 0.0
    return out


def li_conv_mat(field, layer, Nx, Ny, Nx_harmonics, Ny_harmonics, axis):
    """Li's factorization rule for crossed gratings (L. Li, J. Opt. Soc. Am. A
    14, 2758 (1997)) -- an option the reference does not have; its ConvMat
    (rcwa.cpp:6-82) is the Laurent rule everywhere.

    axis "x" gives eps_xx = [[ [[eps]]_x ]]_y: along each grid row (fixed y) the
    1-D Toeplitz matrix of 1/eps in the x harmonics is inverted (inverse rule,
    x being normal to the walls that the field component crosses), and the
    inverses are then convolved along y (Laurent rule).  axis "y" swaps the two
    axes.  The mode index is m = p*Q + q (x slow) as in conv_mat.
    """
    F = np.asarray(field, dtype=np.complex128)[layer * Nx * Ny:(layer + 1) * Nx * Ny].reshape(Ny, Nx)
    P = 2 * Nx_harmonics + 1
    Q = 2 * Ny_harmonics + 1
    if axis == "x":
        lines, na, nb, Pa, Pb = 1.0 / F, Nx, Ny, P, Q
    else:
        lines, na, nb, Pa, Pb = (1.0 / F).T, Ny, Nx, Q, P
    a = _dft_1d(lines, na, Pa - 1)                        # [nb][2Pa-1]
    d = np.arange(Pa)[:, None] - np.arange(Pa)[None, :] + Pa - 1
    eye = np.eye(Pa, dtype=np.complex128)
    M = np.stack([_lu_solve(a[i][d], eye) for i in range(nb)])   # [nb][Pa][Pa]
    c = _dft_1d(np.moveaxis(M, 0, -1), nb, Pb - 1)        # [Pa][Pa][2Pb-1]
    m = np.arange(P * Q)
    pa, pb = (m // Q, m % Q) if axis == "x" else (m % Q, m // Q)
    return c[pa[:, None], pa[None, :], pb[:, None] - pb[None, :] + Pb - 1]


def compute_wave_vectors(Lx, Ly, source: Source, params: Params):
    """rcwa.cpp:85-160 -> (k_inc[3], Kx, Ky, Kz_ref, Kz_trn), vectors of length PQ."""
    n_inc = np.sqrt(complex(params.er_ref) * complex(params.ur_ref))   # std::sqrt, :91
    st, ct = math.sin(source.theta), math.cos(source.theta)
    sp, cp = math.sin(source.phi), math.cos(source.phi)
    k_inc = [n_inc * st * cp, n_inc * st * sp, n_inc * ct]              # :99-103
    P = 2 * params.Nx_harmonics + 1
    Q = 2 * params.Ny_harmonics + 1
    kx_t = np.arange(-params.Nx_harmonics, params.Nx_harmonics + 1).astype(np.complex128)
    ky_t = np.arange(-params.Ny_harmonics, params.Ny_harmonics + 1).astype(np.complex128)
    kx_t = kx_t * (-(source.lambda0 / Lx)) + k_inc[0]                   # :110-112
    ky_t = ky_t * (-(source.lambda0 / Ly)) + k_inc[1]                   # :113-115
    # MeshGrid (rcwa.hpp:218-224): X[q,p] = kx[p], Y[q,p] = ky[q]; reshaped()
    # flattens column-major, so m = p*Q + q.
    Kx = np.repeat(kx_t, Q)
    Ky = np.tile(ky_t, P)
    a_ref = np.conj(params.ur_ref) * np.conj(params.er_ref)
    a_trn = np.conj(params.ur_trn) * np.conj(params.er_trn)
    Kz_ref = -np.conj(unsigned_sqrt(a_ref - Kx * Kx - Ky * Ky))        # :134
    Kz_trn = np.conj(unsigned_sqrt(a_trn - Kx * Kx - Ky * Ky))         # :135
    return k_inc, Kx, Ky, Kz_ref, Kz_trn


def _q_blocks(Kx, Ky, mu_eps):
    """The 2x2-block-of-diagonals Q used at rcwa.cpp:186-203, 361-372, 421-432."""
    N = Kx.size
    Q = np.zeros((2 * N, 2 * N), dtype=np.complex128)
    i = np.arange(N)
    KxKy = Kx * Ky
    Q[i, i] = KxKy
    Q[i, i + N] = mu_eps - Kx * Kx
    Q[i + N, i] = Ky * Ky - mu_eps
    Q[i + N, i + N] = -KxKy
    return Q


def gap_medium(Kx, Ky):
    """rcwa.cpp:163-234 -> (W0, V0): W0 = I, V0 = Q / (i Kz) column-wise."""
    Kz = np.conj(unsigned_sqrt(1.0 - Kx * Kx - Ky * Ky))                # :179
    N = Kx.size
    Q = _q_blocks(Kx, Ky, 1.0)                                          # :194-203
    W0 = np.eye(2 * N, dtype=np.complex128)                             # :209
    lam = np.concatenate([1j * Kz, 1j * Kz])                            # :214
    V0 = Q / lam[None, :]                                               # :223-226
    return W0, V0


def smatrix_init(Nx_harmonics, Ny_harmonics):
    """rcwa.cpp:237-250."""
    PQ = (2 * Nx_harmonics + 1) * (2 * Ny_harmonics + 1)
    Z = np.zeros((2 * PQ, 2 * PQ), dtype=np.complex128)
    I = np.eye(2 * PQ, dtype=np.complex128)
    return SMatrix(Z.copy(), I.copy(), I.copy(), Z.copy())


def layer_pq(erc, urc, Kx, Ky, li=None):
    """rcwa.cpp:262-286 -> (P_i, Q_i).

    ``li`` = (eps_xx, eps_yy, mu_xx, mu_yy) from li_conv_mat replaces erc / urc
    where they multiply the in-plane field components (Q: E_x, E_y; P: H_x,
    H_y); erc^-1 / urc^-1 (the z components) keep the Laurent rule.
    """
    exx, eyy, mxx, myy = (erc, erc, urc, urc) if li is None else li
    N = Kx.size
    DKx, DKy = np.diag(Kx), np.diag(Ky)
    erc_inv_Kx = _lu_solve(erc, DKx)                                    # :267
    erc_inv_Ky = _lu_solve(erc, DKy)                                    # :270
    P = np.zeros((2 * N, 2 * N), dtype=np.complex128)
    P[:N, :N] = Kx[:, None] * erc_inv_Ky                                # :273
    P[:N, N:] = myy - Kx[:, None] * erc_inv_Kx                          # :274
    P[N:, :N] = Ky[:, None] * erc_inv_Ky - mxx                          # :275
    P[N:, N:] = (-Ky)[:, None] * erc_inv_Kx                             # :276
    urc_inv_Kx = _lu_solve(urc, DKx)                                    # :280
    urc_inv_Ky = _lu_solve(urc, DKy)                                    # :281
    Qm = np.zeros((2 * N, 2 * N), dtype=np.complex128)
    Qm[:N, :N] = Kx[:, None] * urc_inv_Ky                               # :282
    Qm[:N, N:] = eyy - Kx[:, None] * urc_inv_Kx                         # :283
    Qm[N:, :N] = Ky[:, None] * urc_inv_Ky - exx                         # :284
    Qm[N:, N:] = (-Ky)[:, None] * urc_inv_Kx                            # :285
    return P, Qm


def layer_smatrix_from_modes(W, lam, Qm, W0, V0, k0, t):
    """rcwa.cpp:317-351 given eigenvectors ``W`` and ``lam = sqrt(lambda^2)``."""
    V = (Qm @ W) / lam[None, :]                                         # :326-330
    Wi_W0 = _lu_solve(W, W0)                                            # :335
    Vi_V0 = _lu_solve(V, V0)                                            # :336
    A = Wi_W0 + Vi_V0                                                   # :337
    B = Wi_W0 - Vi_V0                                                   # :338
    X = np.diag(np.exp(-k0 * t * lam))                                  # :339
    A_lu = sla.lu_factor(A, check_finite=False)                         # :345
    AiX = sla.lu_solve(A_lu, X, check_finite=False)
    D = A - X @ B @ AiX @ B                                             # :346
    D_lu = sla.lu_factor(D, check_finite=False)
    S11 = sla.lu_solve(D_lu, X @ B @ AiX @ A - B, check_finite=False)   # :347
    AiB = sla.lu_solve(A_lu, B, check_finite=False)
    S12 = sla.lu_solve(D_lu, X, check_finite=False) @ (A - B @ AiB)     # :348
    return SMatrix(S11, S12, S12.copy(), S11.copy())                    # :351


def smatrix_layer(erc, urc, Kx, Ky, W0, V0, k0, t, eig=None, li=None):
    """rcwa.cpp:254-352 -- one layer's (symmetric) S-matrix.

    ``eig`` may replace the eigensolver (rcwa.cpp:298) to test basis invariance;
    ``li`` selects Li's factorization rule (see layer_pq).
    """
    P, Qm = layer_pq(erc, urc, Kx, Ky, li)
    Omega2 = P @ Qm                                                     # :288
    if eig is None:
        lam2, W = sla.eig(Omega2, check_finite=False)                   # :298-306
    else:
        lam2, W = eig(Omega2)
    lam = unsigned_sqrt(lam2)                                           # :317
    return layer_smatrix_from_modes(W, lam, Qm, W0, V0, k0, t)


def _port_smatrix(Kx, Ky, Kz, er, ur, W0, V0, side):
    """Shared body of rcwa.cpp:354-411 (side='ref') and :414-466 (side='trn')."""
    N = Kx.size
    Qp = _q_blocks(Kx, Ky, ur * er) / ur                                # :361-372 / :421-432
    Wp = np.eye(2 * N, dtype=np.complex128)
    if side == "ref":
        lam = np.concatenate([-1j * Kz, -1j * Kz])                      # :377
    else:
        lam = np.concatenate([1j * Kz, 1j * Kz])                        # :437
    Vp = Qp / lam[None, :]
    W0i_Wp = _lu_solve(W0, Wp)                                          # :392 / :453
    V0i_Vp = _lu_solve(V0, Vp)                                          # :394 / :454
    A = W0i_Wp + V0i_Vp
    B = W0i_Wp - V0i_Vp
    AiB = _lu_solve(A, B)                                               # :400 / :458
    two_Ai = _lu_solve(A, 2.0 * np.eye(2 * N, dtype=np.complex128))     # :406 / :462
    half = 0.5 * (A - B @ AiB)                                          # :407 / :461
    BAi = _lu_solve(A.T, B.T).T                                         # :408 / :460
    if side == "ref":
        return SMatrix(-AiB, two_Ai, half, BAi), Wp                     # :405-410
    return SMatrix(BAi, half, two_Ai, -AiB), Wp                         # :460-465


def smatrix_reflection(params: Params, Kx, Ky, Kz_ref, W0, V0):
    """rcwa.cpp:354-411 -> (S_ref, W_ref)."""
    return _port_smatrix(Kx, Ky, Kz_ref, complex(params.er_ref), complex(params.ur_ref), W0, V0, "ref")


def smatrix_transmission(params: Params, Kx, Ky, Kz_trn, W0, V0):
    """rcwa.cpp:414-466 -> (S_trn, W_trn)."""
    return _port_smatrix(Kx, Ky, Kz_trn, complex(params.er_trn), complex(params.ur_trn), W0, V0, "trn")


def redheffer_product(A: SMatrix, B: SMatrix) -> SMatrix:
    """rcwa.cpp:588-615 -- star product A (x) B."""
    n = A.S22.shape[0]
    I = np.eye(n, dtype=np.complex128)
    F = sla.lu_factor(I - B.S11 @ A.S22, check_finite=False)           # :602, :605
    G = sla.lu_factor(I - A.S22 @ B.S11, check_finite=False)           # :603, :606
    S11 = A.S11 + A.S12 @ sla.lu_solve(F, B.S11, check_finite=False) @ A.S21   # :608
    S12 = A.S12 @ sla.lu_solve(F, B.S12, check_finite=False)                  # :609
    S21 = B.S21 @ sla.lu_solve(G, A.S21, check_finite=False)                  # :610
    S22 = B.S22 + B.S21 @ sla.lu_solve(G, A.S22, check_finite=False) @ B.S12  # :611
    return SMatrix(S11, S12, S21, S22)


def _normalize(v):
    """Eigen ``normalize()``: divide by the 2-norm, leave a zero vector unchanged."""
    nrm = math.sqrt(float(np.sum(np.abs(v) ** 2)))
    return v / nrm if nrm > 0.0 else v


def source_vectors(source: Source, k_inc):
    """rcwa.cpp:481-498 -> (a_TE, a_TM, Pol)."""
    k = [complex(c) for c in k_inc]
    if abs(source.theta) < 1e-6:                                        # :483
        a_te = np.array([0.0, 1.0, 0.0], dtype=np.complex128)
    else:
        a_te = np.array([-k[1], k[0], 0.0], dtype=np.complex128)        # :486
    a_te = _normalize(a_te)
    a_tm = np.array([k[1] * a_te[2] - k[2] * a_te[1],
                     k[2] * a_te[0] - k[0] * a_te[2],
                     k[0] * a_te[1] - k[1] * a_te[0]], dtype=np.complex128)  # :491
    a_tm = _normalize(a_tm)
    pol = _normalize(source.pte * a_te + source.ptm * a_tm)             # :495-498
    return a_te, a_tm, pol


def source_mode_coeff(source: Source, params: Params, k_inc, W_ref):
    """rcwa.cpp:469-523 -> csrc = W_ref^-1 esrc."""
    _, _, pol = source_vectors(source, k_inc)
    PQ = (2 * params.Nx_harmonics + 1) * (2 * params.Ny_harmonics + 1)
    esrc = np.zeros(2 * PQ, dtype=np.complex128)
    esrc[PQ // 2] = pol[0]                                              # :513
    esrc[PQ // 2 + PQ] = pol[1]                                         # :514
    return _lu_solve(W_ref, esrc)                                       # :520


def _field(S, csrc, Kx, Ky, Kz, Wp):
    PQ = Kx.size
    r = np.zeros(3 * PQ, dtype=np.complex128)
    r[:2 * PQ] = Wp @ (S @ csrc)
    r[2 * PQ:] = -(Kx * r[:PQ] + Ky * r[PQ:2 * PQ]) / Kz
    return r


def reflected_field(S_global: SMatrix, csrc, Kx, Ky, Kz_ref, W_ref):
    """rcwa.cpp:526-542."""
    return _field(S_global.S11, csrc, Kx, Ky, Kz_ref, W_ref)


def transmitted_field(S_global: SMatrix, csrc, Kx, Ky, Kz_trn, W_trn):
    """rcwa.cpp:544-561."""
    return _field(S_global.S21, csrc, Kx, Ky, Kz_trn, W_trn)


def diffraction_efficiencies(params: Params, r, t, k_inc, Kz_ref, Kz_trn) -> Results:
    """rcwa.cpp:564-585."""
    P = 2 * params.Nx_harmonics + 1
    Q = 2 * params.Ny_harmonics + 1
    PQ = P * Q
    rr = np.abs(r[:PQ]) ** 2 + np.abs(r[PQ:2 * PQ]) ** 2 + np.abs(r[2 * PQ:]) ** 2
    den = (complex(k_inc[2]) / params.ur_ref).real
    R = ((-Kz_ref / params.ur_ref).real / den) * rr
    tt = np.abs(t[:PQ]) ** 2 + np.abs(t[PQ:2 * PQ]) ** 2 + np.abs(t[2 * PQ:]) ** 2
    T = ((Kz_trn / params.ur_trn).real / den) * tt
    R = R.reshape(P, Q).T          # Eigen reshaped(Q, P) is column-major
    T = T.reshape(P, Q).T
    return Results(R, T, float(R.sum()), float(T.sum()))


# ----------------------------------------------------------------------------
# solve orchestration (main.cpp:111-191)
# ----------------------------------------------------------------------------
def conv_mats(stack: Stack, params: Params, rule: str = "laurent"):
    """main.cpp:125-138: erc/urc per layer.  rule "li" adds a third list of
    per-layer (eps_xx, eps_yy, mu_xx, mu_yy) (li_conv_mat)."""
    erc, urc = [], []
    h = (stack.Nx, stack.Ny, params.Nx_harmonics, params.Ny_harmonics)
    for l in range(stack.num_layers):
        erc.append(conv_mat(stack.er, l, *h))
        urc.append(conv_mat(stack.ur, l, *h))
    if rule == "laurent":
        return erc, urc
    if rule != "li":
        raise ValueError(f"unknown factorization rule {rule!r}")
    li = [(li_conv_mat(stack.er, l, *h, "x"), li_conv_mat(stack.er, l, *h, "y"),
           li_conv_mat(stack.ur, l, *h, "x"), li_conv_mat(stack.ur, l, *h, "y"))
          for l in range(stack.num_layers)]
    return erc, urc, li


def solve(stack: Stack, source: Source, params: Params, convs=None, return_smatrix=False,
          rule: str = "laurent"):
    """main.cpp:111-191: the reference's end-to-end solve for one source.

    ``convs`` optionally passes precomputed conv_mats output (it depends on the
    grid and harmonics only, not on the source); a 3-tuple carries Li's
    matrices and selects that rule, as does ``rule="li"``.
    """
    convs = convs if convs is not None else conv_mats(stack, params, rule)
    erc, urc = convs[0], convs[1]
    li = convs[2] if len(convs) > 2 else [None] * stack.num_layers
    k_inc, Kx, Ky, Kz_ref, Kz_trn = compute_wave_vectors(stack.Lx, stack.Ly, source, params)
    W0, V0 = gap_medium(Kx, Ky)
    S_dev = smatrix_init(params.Nx_harmonics, params.Ny_harmonics)
    for l in range(stack.num_layers):
        S_l = smatrix_layer(erc[l], urc[l], Kx, Ky, W0, V0, source.k0, float(stack.t[l]), li=li[l])
        S_dev = redheffer_product(S_dev, S_l)
    S_ref, W_ref = smatrix_reflection(params, Kx, Ky, Kz_ref, W0, V0)
    S_trn, W_trn = smatrix_transmission(params, Kx, Ky, Kz_trn, W0, V0)
    S_g = redheffer_product(redheffer_product(S_ref, S_dev), S_trn)
    csrc = source_mode_coeff(source, params, k_inc, W_ref)
    r = reflected_field(S_g, csrc, Kx, Ky, Kz_ref, W_ref)
    t = transmitted_field(S_g, csrc, Kx, Ky, Kz_trn, W_trn)
    res = diffraction_efficiencies(params, r, t, k_inc, Kz_ref, Kz_trn)
    if return_smatrix:
        return res, S_g
    return res
