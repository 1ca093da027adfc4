"""Oracle timing helpers for the CPU-baseline leg of bench.py (test
infrastructure: the oracle is the checker and the timed CPU port, never the
product)."""
from __future__ import annotations

from oracle import rcwa_oracle as O
from helpers import oracle_args


def oracle_one_solve_result(pb, i, convs=None):
    S, src, par = oracle_args(pb, i)
    if convs is None:
        convs = O.conv_mats(S, par)
    return O.solve(S, src, par, convs=convs), convs


def oracle_one_solve(pb, i, convs=None):
    return oracle_one_solve_result(pb, i, convs)[1]
