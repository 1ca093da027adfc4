"""Oracle timing helpers for the CPU-baseline leg and the reference arm of
bench.py (test infrastructure: the oracle is the checker and the timed CPU
port, never the product).

The CPU port is timed as one solve per process with single-threaded BLAS,
one process per host core, all cores busy.  Worker processes are started with the "spawn" method (the parent has
a CUDA context) and build the wavelength-independent convolution matrices
once."""
from __future__ import annotations

import multiprocessing as mp
import os
import time

from oracle import rcwa_oracle as O
from helpers import oracle_args


def oracle_one_solve_result(pb, i, convs=None):
    S, src, par = oracle_args(pb, i)
    if convs is None:
        convs = O.conv_mats(S, par)
    return O.solve(S, src, par, convs=convs), convs


def oracle_one_solve(pb, i, convs=None):
    return oracle_one_solve_result(pb, i, convs)[1]


_W = {}


def _init(pb):
    S, _, par = oracle_args(pb, 0)
    _W["pb"] = pb
    _W["convs"] = O.conv_mats(S, par)


def _solve(i):
    pb = _W["pb"]
    S, src, par = oracle_args(pb, i)
    t0 = time.perf_counter()
    r = O.solve(S, src, par, convs=_W["convs"])
    return i, r.R, r.T, r.R_tot, r.T_tot, time.perf_counter() - t0


class OraclePool:
    """`procs` single-threaded oracle processes for the sources of `pb`."""

    def __init__(self, pb, procs=None):
        self.procs = procs or os.cpu_count() or 1
        saved = {k: os.environ.get(k) for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")}
        for k in saved:
            os.environ[k] = "1"
        try:
            self.pool = mp.get_context("spawn").Pool(self.procs, initializer=_init, initargs=(pb,))
        finally:
            for k, v in saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v

    def run(self, indices):
        """Solves the given source indices in parallel; (results by index, wall seconds)."""
        t0 = time.perf_counter()
        out = self.pool.map(_solve, list(indices), chunksize=1)
        return {o[0]: o for o in out}, time.perf_counter() - t0

    def close(self):
        self.pool.terminate()
        self.pool.join()
