"""ctypes binding of ``librcwa_b200.so`` (the C ABI of include/rcwa_b200.h).

This is the Python caller of the boundary -- the same calls a C/C++ caller
makes.  Loading fails loudly when the library has not been built; there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .configs import ParamSpec, Problem, SourceSpec, StackSpec

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "librcwa_b200.so")

RCWA_OK = 0
RCWA_ERR_INVALID = -1
RCWA_ERR_CUDA = -2
RCWA_ERR_NOMEM = -3
RCWA_ERR_NUMERIC = -4
RCWA_ERR_BUSY = -5
RCWA_ERR_NOTFOUND = -6

STATUS_SINGULAR = 1
STATUS_EIG_NOCONV = 2
STATUS_NONFINITE = 4
STATUS_WOOD_ANOMALY = 8
STATUS_REFINE_SLOW = 16

PREC_FP64 = 0
PREC_MIXED = 1
# stages that PREC_MIXED runs in reduced precision (Context.set_mixed)
MIXED_LAYER_GEMM = 1
MIXED_STAR_GEMM = 2
MIXED_LAYER_LU = 4
MIXED_STAR_LU = 8
MIXED_ALL = 15
MIXED_GEMM_TF32 = 16   # GEMM stages on split-TF32 instead of int8 slices
MIXED_REFINE_INT8 = 32  # LU refinement residuals on the int8-slice GEMM
GEOM_LI_RULE = 1   # rcwa_geometry_create_ex: Li's factorization rule


class RcwaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rcwa error {code}: {msg}")
        self.code = code


class CComplex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class CStack(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("num_layers", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double),
                ("er", C.c_void_p), ("ur", C.c_void_p), ("t", C.c_void_p)]


class CSource(C.Structure):
    _fields_ = [("lambda0", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
                ("pte", C.c_double), ("ptm", C.c_double)]


class CParams(C.Structure):
    _fields_ = [("nx_harmonics", C.c_int), ("ny_harmonics", C.c_int),
                ("er_ref", CComplex), ("ur_ref", CComplex),
                ("er_trn", CComplex), ("ur_trn", CComplex)]


class CShape(C.Structure):
    _fields_ = [("kind", C.c_int), ("cx", C.c_double), ("cy", C.c_double), ("a", C.c_double),
                ("b", C.c_double), ("eps", CComplex), ("mu", CComplex)]


class CLayerShapes(C.Structure):
    _fields_ = [("eps_bg", CComplex), ("mu_bg", CComplex), ("t", C.c_double), ("n_shapes", C.c_int),
                ("shapes", C.c_void_p)]


SHAPE_CIRCLE, SHAPE_RECT, SHAPE_LINES, SHAPE_TRIANGLE = 1, 2, 3, 4


class CServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_int), ("max_queue", C.c_int), ("precision", C.c_int), ("lanes", C.c_int),
                ("hbm_budget_bytes", C.c_uint64), ("mixed_stages", C.c_uint), ("refine_sweeps", C.c_int),
                ("gemm_digits", C.c_int)]


class CServerInfo(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("queued", C.c_uint64), ("in_flight", C.c_uint64),
                ("rejected", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("admitted_bytes", C.c_uint64), ("peak_admitted_bytes", C.c_uint64),
                ("budget_bytes", C.c_uint64), ("lanes", C.c_int)]


class CResult(C.Structure):
    _fields_ = [("R", C.c_void_p), ("T", C.c_void_p), ("R_tot", C.c_double),
                ("T_tot", C.c_double), ("status", C.c_uint32)]


_VP = C.c_void_p
_SIGS = {
    "rcwa_last_error": ([], C.c_char_p),
    "rcwa_version": ([], C.c_int),
    "rcwa_context_create": ([C.c_int, C.POINTER(_VP)], C.c_int),
    "rcwa_context_destroy": ([_VP], C.c_int),
    "rcwa_context_set_stream": ([_VP, _VP], C.c_int),
    "rcwa_context_synchronize": ([_VP], C.c_int),
    "rcwa_context_kernel_launches": ([_VP, C.POINTER(C.c_uint64)], C.c_int),
    "rcwa_context_set_mixed": ([_VP, C.c_uint, C.c_int, C.c_int], C.c_int),
    "rcwa_profile_enable": ([C.c_int], C.c_int),
    "rcwa_profile_reset": ([], C.c_int),
    "rcwa_profile_query": ([C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                            C.POINTER(C.c_double)], C.c_int),
    "rcwa_solve": ([_VP, C.POINTER(CStack), C.POINTER(CSource), C.POINTER(CParams), C.c_int,
                    C.POINTER(CResult)], C.c_int),
    "rcwa_solve_sweep": ([_VP, C.POINTER(CStack), C.POINTER(CSource), C.c_int, C.POINTER(CParams),
                          C.c_int, C.POINTER(CResult)], C.c_int),
    "rcwa_geometry_create": ([_VP, C.POINTER(CStack), C.POINTER(CParams), C.c_int, C.POINTER(_VP)], C.c_int),
    "rcwa_geometry_create_ex": ([_VP, C.POINTER(CStack), C.POINTER(CParams), C.c_int, C.c_uint,
                                 C.POINTER(_VP)], C.c_int),
    "rcwa_geometry_destroy": ([_VP], C.c_int),
    "rcwa_solve_sweep_device": ([_VP, _VP, C.POINTER(CSource), C.c_int, C.c_int, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_convmat": ([_VP, _VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _VP], C.c_int),
    "rcwa_wave_vectors": ([_VP, C.c_double, C.c_double, C.POINTER(CSource), C.POINTER(CParams),
                           _VP, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_gap_medium": ([_VP, C.c_int, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_smatrix_layer": ([_VP, C.c_int, _VP, _VP, _VP, _VP, _VP, C.c_double, C.c_double, _VP, _VP,
                            C.POINTER(C.c_uint32)], C.c_int),
    "rcwa_smatrix_reflection": ([_VP, C.POINTER(CParams), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_smatrix_transmission": ([_VP, C.POINTER(CParams), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_redheffer": ([_VP, C.c_int, C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                        C.POINTER(C.c_uint32)], C.c_int),
    "rcwa_efficiencies": ([_VP, C.POINTER(CSource), C.POINTER(CParams), _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                           C.POINTER(CResult)], C.c_int),
    "rcwa_eig": ([_VP, C.c_int, C.c_int, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_eig_noalloc": ([C.c_int, C.c_int, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_eig_set_sweep_cap": ([C.c_int], C.c_int),
    "rcwa_eig_set_cluster_size": ([C.c_int], C.c_int),
    "rcwa_debug_gemm_inject_timeout": ([C.c_int], C.c_int),
    "rcwa_lu_solve": ([_VP, C.c_int, C.c_int, C.c_int, _VP, _VP, _VP, _VP], C.c_int),
    "rcwa_lu_solve_ex": ([_VP, C.c_int, C.c_int, C.c_int, _VP, _VP, _VP, _VP, C.c_int, C.c_int], C.c_int),
    "rcwa_gemm_ex": ([_VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, CComplex, _VP, _VP,
                      CComplex, _VP], C.c_int),
    "rcwa_gemm": ([_VP, C.c_int, C.c_int, C.c_int, C.c_int, _VP, _VP, _VP, C.c_int], C.c_int),
    "rcwa_gemm_device": ([_VP, C.c_int, C.c_int, C.c_int, C.c_int, CComplex, _VP, _VP, CComplex, _VP, C.c_int],
                         C.c_int),
    "rcwa_set_gemm_table": ([_VP], C.c_int),
    "rcwa_rasterize": ([_VP, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.POINTER(CLayerShapes),
                        _VP, _VP, _VP], C.c_int),
    "rcwa_geometry_create_shapes": ([_VP, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                     C.POINTER(CLayerShapes), C.POINTER(CParams), C.POINTER(_VP)], C.c_int),
    "rcwa_solve_batch": ([_VP, C.c_int, C.POINTER(CStack), C.POINTER(CSource), C.POINTER(CParams),
                          C.c_int, C.POINTER(CResult)], C.c_int),
    "rcwa_server_create": ([C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_VP)], C.c_int),
    "rcwa_server_create_ex": ([C.c_int, C.POINTER(CServerConfig), C.POINTER(_VP)], C.c_int),
    "rcwa_server_info_get": ([_VP, C.POINTER(CServerInfo)], C.c_int),
    "rcwa_server_submit": ([_VP, C.POINTER(CStack), C.POINTER(CSource), C.POINTER(CParams),
                            C.POINTER(C.c_uint64)], C.c_int),
    "rcwa_server_poll": ([_VP, C.c_uint64, C.c_int, C.POINTER(CResult), C.POINTER(C.c_int)], C.c_int),
    "rcwa_server_stats": ([_VP, C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.POINTER(C.c_double)],
                          C.c_int),
    "rcwa_server_destroy": ([_VP], C.c_int),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library (no fallback: raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RcwaError(RCWA_ERR_INVALID, f"{path} is not built; run rcwa_b200.build.build()")
    lib = C.CDLL(path)
    for name, (args, res) in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def declared_symbols() -> List[str]:
    return list(_SIGS)


def profile_enable(on: bool = True):
    load().rcwa_profile_enable(1 if on else 0)


def profile_reset():
    load().rcwa_profile_reset()


def profile_query(name: str):
    """(total_ms, launches, flops) of one kernel family since the last reset."""
    ms, n, fl = C.c_double(), C.c_uint64(), C.c_double()
    _check(load().rcwa_profile_query(name.encode(), C.byref(ms), C.byref(n), C.byref(fl)))
    return float(ms.value), int(n.value), float(fl.value)


def _check(rc: int, allow_numeric: bool = False):
    if rc == RCWA_OK or (allow_numeric and rc == RCWA_ERR_NUMERIC):
        return rc
    raise RcwaError(rc, load().rcwa_last_error().decode())


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def _fortran(a) -> np.ndarray:
    """Column-major complex128 copy (the ABI's matrix layout)."""
    return np.asfortranarray(np.asarray(a, dtype=np.complex128))


def c_params(p: ParamSpec) -> CParams:
    cc = lambda z: CComplex(float(np.real(z)), float(np.imag(z)))
    return CParams(int(p.nx_harmonics), int(p.ny_harmonics), cc(p.er_ref), cc(p.ur_ref),
                   cc(p.er_trn), cc(p.ur_trn))


def c_source(s: SourceSpec) -> CSource:
    return CSource(float(s.lambda0), float(s.theta), float(s.phi), float(s.pte), float(s.ptm))


_tuning_applied = False


def apply_tuning(path: Optional[str] = None) -> bool:
    """Hands the tuner's GEMM kernel table (rcwa_b200/tune.py) to the
    library; False when no table has been written.  Done once by the first
    Context unless RCWA_NO_TUNING=1."""
    from . import tune
    ch = tune.load_table(path or tune.TABLE_PATH)
    if ch is None:
        return False
    arr = (C.c_int * 25)(*ch)
    _check(load().rcwa_set_gemm_table(arr))
    return True


class Context:
    """One CUDA stream + device workspace (``rcwa_context``)."""

    def __init__(self, device: int = 0):
        global _tuning_applied
        self.lib = load()
        h = C.c_void_p()
        _check(self.lib.rcwa_context_create(device, C.byref(h)))
        self.h = h
        if not _tuning_applied and os.environ.get("RCWA_NO_TUNING") != "1":
            _tuning_applied = True
            apply_tuning()

    def close(self):
        if self.h:
            self.lib.rcwa_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self):
        _check(self.lib.rcwa_context_synchronize(self.h))

    def set_stream(self, stream_ptr: int):
        _check(self.lib.rcwa_context_set_stream(self.h, C.c_void_p(stream_ptr)))

    def kernel_launches(self) -> int:
        v = C.c_uint64()
        _check(self.lib.rcwa_context_kernel_launches(self.h, C.byref(v)))
        return int(v.value)

    # ---- end to end -------------------------------------------------------
    def solve_sweep(self, pb: Problem, precision: int = PREC_FP64,
                    sources: Optional[Sequence[SourceSpec]] = None):
        """``rcwa_solve_sweep`` with host buffers.  Returns (R, T, R_tot, T_tot,
        status) with R/T shaped [n_sources, Q, P]."""
        st = pb.stack
        srcs = list(pb.sources if sources is None else sources)
        er, ur = _c128(st.er), _c128(st.ur)
        t = np.ascontiguousarray(st.t, dtype=np.float64)
        cst = CStack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, _ptr(er), _ptr(ur), _ptr(t))
        P = 2 * pb.params.nx_harmonics + 1
        Q = 2 * pb.params.ny_harmonics + 1
        ns = len(srcs)
        R = np.zeros((ns, P * Q))
        T = np.zeros((ns, P * Q))
        carr = (CSource * ns)(*[c_source(s) for s in srcs])
        res = (CResult * ns)()
        for i in range(ns):
            res[i].R = R[i].ctypes.data
            res[i].T = T[i].ctypes.data
        prm = c_params(pb.params)
        _check(self.lib.rcwa_solve_sweep(self.h, C.byref(cst), carr, ns, C.byref(prm), precision, res),
               allow_numeric=True)
        Rt = np.array([r.R_tot for r in res])
        Tt = np.array([r.T_tot for r in res])
        stat = np.array([r.status for r in res], dtype=np.uint32)
        # column-major Q x P -> [Q, P]
        R = R.reshape(ns, P, Q).transpose(0, 2, 1)
        T = T.reshape(ns, P, Q).transpose(0, 2, 1)
        return R, T, Rt, Tt, stat

    def geometry_create(self, st: StackSpec, p: ParamSpec, er_ptr=None, ur_ptr=None, t_ptr=None,
                        rule: str = "laurent"):
        """``rcwa_geometry_create_ex``.  With device pointers (e.g. torch tensors'
        data_ptr()) the grids are read in place on the GPU; otherwise the
        host arrays of ``st`` are used.  ``rule="li"`` selects Li's
        factorization rule (RCWA_GEOM_LI_RULE) instead of the reference's
        Laurent rule."""
        if rule not in ("laurent", "li"):
            raise ValueError(f"unknown factorization rule {rule!r}")
        flags = GEOM_LI_RULE if rule == "li" else 0
        on_dev = er_ptr is not None
        if on_dev:
            cst = CStack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, er_ptr, ur_ptr, t_ptr)
            keep = None
        else:
            er, ur = _c128(st.er), _c128(st.ur)
            t = np.ascontiguousarray(st.t, dtype=np.float64)
            keep = (er, ur, t)
            cst = CStack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, _ptr(er), _ptr(ur), _ptr(t))
        prm = c_params(p)
        h = C.c_void_p()
        _check(self.lib.rcwa_geometry_create_ex(self.h, C.byref(cst), C.byref(prm), 1 if on_dev else 0, flags,
                                                C.byref(h)))
        del keep
        return h

    def geometry_destroy(self, h):
        if h:
            self.lib.rcwa_geometry_destroy(h)

    def solve_sweep_device(self, geom, sources: Sequence[SourceSpec], precision: int,
                           R_ptr: int, T_ptr: int, tot_ptr: int, status_ptr: int):
        """``rcwa_solve_sweep_device``: asynchronous on the context stream."""
        ns = len(sources)
        carr = (CSource * ns)(*[c_source(s) for s in sources])
        _check(self.lib.rcwa_solve_sweep_device(self.h, geom, carr, ns, precision, R_ptr, T_ptr,
                                                tot_ptr, status_ptr))

    def solve_sweep_ptrs(self, st: StackSpec, p: ParamSpec, sources: Sequence[SourceSpec], precision: int,
                         er_ptr: int, ur_ptr: int, t_ptr: int, res_R: np.ndarray, res_T: np.ndarray):
        """``rcwa_solve_sweep`` on caller-owned host buffers (pinned or not):
        res_R/res_T are [n_sources, Q*P] float64 host arrays.  Returns
        (R_tot, T_tot, status)."""
        ns = len(sources)
        cst = CStack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, er_ptr, ur_ptr, t_ptr)
        carr = (CSource * ns)(*[c_source(s) for s in sources])
        res = (CResult * ns)()
        stride = res_R.strides[0]
        for i in range(ns):
            res[i].R = res_R.ctypes.data + i * stride
            res[i].T = res_T.ctypes.data + i * stride
        prm = c_params(p)
        _check(self.lib.rcwa_solve_sweep(self.h, C.byref(cst), carr, ns, C.byref(prm), precision, res),
               allow_numeric=True)
        return (np.array([r.R_tot for r in res]), np.array([r.T_tot for r in res]),
                np.array([r.status for r in res], dtype=np.uint32))

    # ---- step level -------------------------------------------------------
    def convmat(self, field, layer, Nx, Ny, nxh, nyh) -> np.ndarray:
        f = _c128(field)
        PQ = (2 * nxh + 1) * (2 * nyh + 1)
        out = np.zeros((PQ, PQ), dtype=np.complex128, order="F")
        _check(self.lib.rcwa_convmat(self.h, _ptr(f), layer, Nx, Ny, nxh, nyh, _ptr(out)))
        return out

    def wave_vectors(self, Lx, Ly, src: SourceSpec, p: ParamSpec):
        PQ = (2 * p.nx_harmonics + 1) * (2 * p.ny_harmonics + 1)
        kinc = np.zeros(3, np.complex128)
        arrs = [np.zeros(PQ, np.complex128) for _ in range(4)]
        cs, cp = c_source(src), c_params(p)
        _check(self.lib.rcwa_wave_vectors(self.h, Lx, Ly, C.byref(cs), C.byref(cp), _ptr(kinc),
                                          *[_ptr(a) for a in arrs]))
        return (kinc, *arrs)

    def gap_medium(self, Kx, Ky):
        Kx, Ky = _c128(Kx), _c128(Ky)
        n = 2 * Kx.size
        W0 = np.zeros((n, n), np.complex128, order="F")
        V0 = np.zeros((n, n), np.complex128, order="F")
        _check(self.lib.rcwa_gap_medium(self.h, Kx.size, _ptr(Kx), _ptr(Ky), _ptr(W0), _ptr(V0)))
        return W0, V0

    def smatrix_layer(self, erc, urc, Kx, Ky, V0, k0, t):
        erc, urc, V0 = _fortran(erc), _fortran(urc), _fortran(V0)
        Kx, Ky = _c128(Kx), _c128(Ky)
        n = 2 * Kx.size
        S11 = np.zeros((n, n), np.complex128, order="F")
        S12 = np.zeros((n, n), np.complex128, order="F")
        st = C.c_uint32()
        _check(self.lib.rcwa_smatrix_layer(self.h, Kx.size, _ptr(erc), _ptr(urc), _ptr(Kx), _ptr(Ky),
                                           _ptr(V0), k0, t, _ptr(S11), _ptr(S12), C.byref(st)))
        return S11, S12, int(st.value)

    def smatrix_port(self, side: str, p: ParamSpec, Kx, Ky, Kz, V0):
        Kx, Ky, Kz, V0 = _c128(Kx), _c128(Ky), _c128(Kz), _fortran(V0)
        n = 2 * Kx.size
        S = [np.zeros((n, n), np.complex128, order="F") for _ in range(4)]
        cp = c_params(p)
        f = self.lib.rcwa_smatrix_reflection if side == "ref" else self.lib.rcwa_smatrix_transmission
        _check(f(self.h, C.byref(cp), _ptr(Kx), _ptr(Ky), _ptr(Kz), _ptr(V0), *[_ptr(s) for s in S]))
        return S

    def redheffer(self, A, B):
        A = [_fortran(a) for a in A]
        B = [_fortran(b) for b in B]
        n = A[0].shape[0]
        S = [np.zeros((n, n), np.complex128, order="F") for _ in range(4)]
        pa = (C.c_void_p * 4)(*[_ptr(a) for a in A])
        pb = (C.c_void_p * 4)(*[_ptr(b) for b in B])
        ps = (C.c_void_p * 4)(*[_ptr(s) for s in S])
        st = C.c_uint32()
        _check(self.lib.rcwa_redheffer(self.h, n, pa, pb, ps, C.byref(st)))
        return S, int(st.value)

    def efficiencies(self, src: SourceSpec, p: ParamSpec, k_inc, Kx, Ky, Kzr, Kzt, S11, S21):
        k_inc, Kx, Ky, Kzr, Kzt = (_c128(a) for a in (k_inc, Kx, Ky, Kzr, Kzt))
        S11, S21 = _fortran(S11), _fortran(S21)
        PQ = Kx.size
        R, T = np.zeros(PQ), np.zeros(PQ)
        res = CResult(R.ctypes.data, T.ctypes.data, 0.0, 0.0, 0)
        cs, cp = c_source(src), c_params(p)
        _check(self.lib.rcwa_efficiencies(self.h, C.byref(cs), C.byref(cp), _ptr(k_inc), _ptr(Kx), _ptr(Ky),
                                          _ptr(Kzr), _ptr(Kzt), _ptr(S11), _ptr(S21), C.byref(res)))
        P = 2 * p.nx_harmonics + 1
        Q = 2 * p.ny_harmonics + 1
        return R.reshape(P, Q).T, T.reshape(P, Q).T, res.R_tot, res.T_tot, int(res.status)

    def eig(self, A):
        """Batched eigen-decomposition: A is [batch, n, n] or [n, n]."""
        A = np.asarray(A, dtype=np.complex128)
        single = A.ndim == 2
        if single:
            A = A[None]
        b, n, _ = A.shape
        Af = np.ascontiguousarray(A.transpose(0, 2, 1))   # column-major per matrix
        lam = np.zeros((b, n), np.complex128)
        W = np.zeros((b, n, n), np.complex128)
        st = np.zeros(b, np.uint32)
        _check(self.lib.rcwa_eig(self.h, n, b, _ptr(Af), _ptr(lam), _ptr(W), _ptr(st)), allow_numeric=True)
        W = W.transpose(0, 2, 1)
        if single:
            return lam[0], W[0], int(st[0])
        return lam, W, st

    def set_mixed(self, stages: int = MIXED_ALL, refine_sweeps: int = 1, gemm_digits: int = 5):
        """Stages run in reduced precision by PREC_MIXED solves on this context,
        the FP64 refinement sweeps of their LU solves and the digits per
        operand of the int8-slice GEMM."""
        _check(self.lib.rcwa_context_set_mixed(self.h, stages, refine_sweeps, gemm_digits))

    def lu_solve(self, A, B, precision: int = PREC_FP64, refine_sweeps: int = 1):
        A = np.asarray(A, dtype=np.complex128)
        B = np.asarray(B, dtype=np.complex128)
        single = A.ndim == 2
        if single:
            A, B = A[None], B[None]
        if B.ndim == 2:
            B = B[..., None]
        b, n, _ = A.shape
        m = B.shape[2]
        Af = np.ascontiguousarray(A.transpose(0, 2, 1))
        Bf = np.ascontiguousarray(B.transpose(0, 2, 1))
        X = np.zeros((b, m, n), np.complex128)
        st = np.zeros(b, np.uint32)
        _check(self.lib.rcwa_lu_solve_ex(self.h, n, m, b, _ptr(Af), _ptr(Bf), _ptr(X), _ptr(st),
                                         precision, refine_sweeps), allow_numeric=True)
        X = X.transpose(0, 2, 1)
        return (X[0], int(st[0])) if single else (X, st)

    def gemm(self, A, B, precision: int = PREC_FP64):
        A = np.asarray(A, dtype=np.complex128)
        B = np.asarray(B, dtype=np.complex128)
        single = A.ndim == 2
        if single:
            A, B = A[None], B[None]
        b, m, k = A.shape
        n = B.shape[2]
        Af = np.ascontiguousarray(A.transpose(0, 2, 1))
        Bf = np.ascontiguousarray(B.transpose(0, 2, 1))
        Cf = np.zeros((b, n, m), np.complex128)
        _check(self.lib.rcwa_gemm(self.h, m, n, k, b, _ptr(Af), _ptr(Bf), _ptr(Cf), precision))
        Cm = Cf.transpose(0, 2, 1)
        return Cm[0] if single else Cm

    def gemm_device(self, A_ptr, B_ptr, C_ptr, m, n, k, batch, precision: int = PREC_FP64, alpha=1.0, beta=0.0):
        """``rcwa_gemm_device``: C = alpha A B + beta C on batch-packed
        column-major device arrays, asynchronous on the context's stream."""
        a, b = complex(alpha), complex(beta)
        _check(self.lib.rcwa_gemm_device(self.h, m, n, k, batch, CComplex(a.real, a.imag), A_ptr, B_ptr,
                                         CComplex(b.real, b.imag), C_ptr, precision))

    def gemm_ex(self, A, B, C=None, opa=0, opb=0, alpha=1.0, beta=0.0):
        """``rcwa_gemm_ex``: alpha op(A) op(B) + beta C on [b, rows, cols]
        arrays; op = 1 uses the conjugate transpose of the stored matrix."""
        A = np.asarray(A, dtype=np.complex128)
        B = np.asarray(B, dtype=np.complex128)
        b = A.shape[0]
        m = A.shape[2] if opa else A.shape[1]
        k = A.shape[1] if opa else A.shape[2]
        n = B.shape[1] if opb else B.shape[2]
        Af = np.ascontiguousarray(A.transpose(0, 2, 1))
        Bf = np.ascontiguousarray(B.transpose(0, 2, 1))
        Cf = (np.zeros((b, n, m), np.complex128) if C is None
              else np.ascontiguousarray(np.asarray(C, dtype=np.complex128).transpose(0, 2, 1)))
        al, be = complex(alpha), complex(beta)
        _check(self.lib.rcwa_gemm_ex(self.h, opa, opb, m, n, k, b, CComplex(al.real, al.imag), _ptr(Af),
                                     _ptr(Bf), CComplex(be.real, be.imag), _ptr(Cf)))
        return Cf.transpose(0, 2, 1)

    # ---- device-side rasterisers --------------------------------------------
    @staticmethod
    def _layers(layers):
        """layers: [(eps_bg, mu_bg, t, [(kind, cx, cy, a, b, eps, mu), ...]), ...]"""
        cc = lambda z: CComplex(float(np.real(z)), float(np.imag(z)))
        keep = []
        arr = (CLayerShapes * max(1, len(layers)))()
        for i, (eb, mb, t, shapes) in enumerate(layers):
            sa = (CShape * max(1, len(shapes)))()
            for j, (k, cx, cy, a, b, e, m) in enumerate(shapes):
                sa[j] = CShape(int(k), float(cx), float(cy), float(a), float(b), cc(e), cc(m))
            keep.append(sa)
            arr[i] = CLayerShapes(cc(eb), cc(mb), float(t), len(shapes), C.cast(sa, C.c_void_p).value)
        return arr, keep

    def rasterize(self, nx, ny, lx, ly, layers, er_ptr, ur_ptr, t_ptr=None):
        """``rcwa_rasterize`` into device buffers (e.g. torch tensors' data_ptr())."""
        arr, keep = self._layers(layers)
        _check(self.lib.rcwa_rasterize(self.h, nx, ny, lx, ly, len(layers), arr, er_ptr, ur_ptr, t_ptr))
        del keep

    def geometry_create_shapes(self, nx, ny, lx, ly, layers, p: ParamSpec):
        arr, keep = self._layers(layers)
        h = C.c_void_p()
        _check(self.lib.rcwa_geometry_create_shapes(self.h, nx, ny, lx, ly, len(layers), arr,
                                                    C.byref(c_params(p)), C.byref(h)))
        del keep
        return h

    # ---- batches of unrelated problems --------------------------------------
    def solve_batch(self, problems: Sequence[Problem], precision: int = PREC_FP64,
                    source_index: Optional[Sequence[int]] = None):
        """``rcwa_solve_batch``: problem i is (problems[i].stack,
        problems[i].sources[source_index[i] or 0], problems[i].params).
        Returns (R, T, R_tot, T_tot, status) as lists ([Q, P] arrays)."""
        n = len(problems)
        if n == 0:
            return [], [], np.zeros(0), np.zeros(0), np.zeros(0, np.uint32)
        keep = []
        stacks = (CStack * n)()
        srcs = (CSource * n)()
        prms = (CParams * n)()
        res = (CResult * n)()
        outR, outT = [], []
        for i, pb in enumerate(problems):
            st = pb.stack
            er, ur = _c128(st.er), _c128(st.ur)
            t = np.ascontiguousarray(st.t, dtype=np.float64)
            keep += [er, ur, t]
            stacks[i] = CStack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, _ptr(er), _ptr(ur), _ptr(t))
            k = 0 if source_index is None else int(source_index[i])
            srcs[i] = c_source(pb.sources[k])
            prms[i] = c_params(pb.params)
            P = 2 * pb.params.nx_harmonics + 1
            Q = 2 * pb.params.ny_harmonics + 1
            R = np.zeros(P * Q)
            T = np.zeros(P * Q)
            outR.append(R)
            outT.append(T)
            res[i].R = R.ctypes.data
            res[i].T = T.ctypes.data
        _check(self.lib.rcwa_solve_batch(self.h, n, stacks, srcs, prms, precision, res),
               allow_numeric=True)
        del keep
        Rs, Ts = [], []
        for pb, R, T in zip(problems, outR, outT):
            P = 2 * pb.params.nx_harmonics + 1
            Q = 2 * pb.params.ny_harmonics + 1
            Rs.append(R.reshape(P, Q).T)
            Ts.append(T.reshape(P, Q).T)
        return (Rs, Ts, np.array([r.R_tot for r in res]), np.array([r.T_tot for r in res]),
                np.array([r.status for r in res], dtype=np.uint32))


class Server:
    """``rcwa_server_*``: a serving loop with continuous batching on one GPU."""

    def __init__(self, device: int = 0, max_batch: int = 256, max_queue: int = 100000,
                 precision: int = PREC_FP64, lanes: int = 0, hbm_budget_bytes: int = 0,
                 mixed_stages: int = 0, refine_sweeps: int = 0, gemm_digits: int = 0):
        self.lib = load()
        self.h = C.c_void_p()
        cfg = CServerConfig(max_batch, max_queue, precision, lanes, int(hbm_budget_bytes), mixed_stages,
                            refine_sweeps, gemm_digits)
        _check(self.lib.rcwa_server_create_ex(device, C.byref(cfg), C.byref(self.h)))

    def info(self) -> dict:
        """Counters of the server: completed / queued / in-flight / rejected
        requests, latency p50 / p99 (ms), admitted and peak admitted device
        bytes against the budget, lanes."""
        i = CServerInfo()
        _check(self.lib.rcwa_server_info_get(self.h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in CServerInfo._fields_}

    def submit(self, pb: Problem, source_index: int = 0) -> int:
        st = pb.stack
        er, ur = _c128(st.er), _c128(st.ur)
        t = np.ascontiguousarray(st.t, dtype=np.float64)
        cst = CStack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, _ptr(er), _ptr(ur), _ptr(t))
        tk = C.c_uint64()
        _check(self.lib.rcwa_server_submit(self.h, C.byref(cst), C.byref(c_source(pb.sources[source_index])),
                                           C.byref(c_params(pb.params)), C.byref(tk)))
        return int(tk.value)

    def poll(self, ticket: int, pb: Problem, wait: bool = True):
        """(done, R [Q, P], T [Q, P], R_tot, T_tot, status) of one request."""
        P = 2 * pb.params.nx_harmonics + 1
        Q = 2 * pb.params.ny_harmonics + 1
        R = np.zeros(P * Q)
        T = np.zeros(P * Q)
        res = CResult(R.ctypes.data, T.ctypes.data, 0.0, 0.0, 0)
        done = C.c_int(0)
        _check(self.lib.rcwa_server_poll(self.h, ticket, 1 if wait else 0, C.byref(res), C.byref(done)),
               allow_numeric=True)
        return (bool(done.value), R.reshape(P, Q).T, T.reshape(P, Q).T, res.R_tot, res.T_tot,
                int(res.status))

    def stats(self):
        n, p50, p99 = C.c_uint64(), C.c_double(), C.c_double()
        _check(self.lib.rcwa_server_stats(self.h, C.byref(n), C.byref(p50), C.byref(p99)))
        return int(n.value), float(p50.value), float(p99.value)

    def close(self):
        if self.h:
            self.lib.rcwa_server_destroy(self.h)
            self.h = C.c_void_p()
