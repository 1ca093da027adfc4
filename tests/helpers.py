"""Shared test helpers: run the oracle on a configs.Problem."""
from __future__ import annotations

import numpy as np

from oracle import rcwa_oracle as O


def oracle_args(pb, i=0):
    st, s, p = pb.stack, pb.sources[i], pb.params
    S = O.Stack(st.Nx, st.Ny, st.num_layers, st.Lx, st.Ly, st.er, st.ur, st.t)
    src = O.Source(s.lambda0, s.theta, s.phi, s.pte, s.ptm)
    par = O.Params(p.nx_harmonics, p.ny_harmonics, p.er_ref, p.ur_ref, p.er_trn, p.ur_trn)
    return S, src, par


def oracle_solve(pb, i=0, convs=None):
    S, src, par = oracle_args(pb, i)
    return O.solve(S, src, par, convs=convs)


def oracle_sweep(pb, idx=None):
    S, _, par = oracle_args(pb, 0)
    convs = O.conv_mats(S, par)
    idx = range(len(pb.sources)) if idx is None else idx
    return [O.solve(S, oracle_args(pb, i)[1], par, convs=convs) for i in idx]
