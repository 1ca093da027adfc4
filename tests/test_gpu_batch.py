"""Batches of unrelated problems (rcwa_solve_batch) and the serving loop
(rcwa_server_*), through the C ABI, against the FP64 oracle and against the
single-problem entry point.  Tolerance: |dR|, |dT| <= 1e-10 per order, as
for every FP64 end-to-end test."""
import numpy as np
import pytest

from rcwa_b200 import configs as C
from helpers import oracle_solve

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def ctx():
    from rcwa_b200 import lib as L
    c = L.Context(0)
    yield c
    c.close()


def _mixed_list(seed=11, count=14):
    """C3-distributed requests at small sizes (M in {5, 7}, 64^2 grids) plus a
    stack with a uniform layer and a rectangular-period stack, so that the
    batch holds several groups of different shape and repeated shapes."""
    rng = np.random.default_rng(seed)
    pbs = [C.c3_request(rng, grid=64, m_max=7) for _ in range(count)]
    g1 = C.circle(64, 64, 500.0, 500.0, 140.0, C.ref_eps(9.0 + 0.2j), 1.0)
    g2 = C.uniform(64, 64, C.ref_eps(2.3 + 0.01j))
    st = C.make_stack(500.0, 500.0, [g1, g2], [110.0, 40.0])
    pbs.append(C.Problem("uniform_mix", st, [C.SourceSpec(610.0, 0.3, 0.2, 0.6, 0.8)],
                         C.ParamSpec(2, 2, 1.0, 1.0, 2.25, 1.0)))
    g3 = C.rect(48, 40, 430.0, 360.0, 200.0, 150.0, C.ref_eps(7.0 + 0.4j), 1.0)
    st3 = C.make_stack(430.0, 360.0, [g3], [95.0])
    pbs.append(C.Problem("rect_period", st3, [C.SourceSpec(560.0, 0.4, 1.1, 1.0, 0.0)],
                         C.ParamSpec(3, 2, 1.0, 1.0, 2.25, 1.0)))
    return pbs


def test_batch_matches_oracle(ctx):
    pbs = _mixed_list()
    R, T, Rt, Tt, st = ctx.solve_batch(pbs)
    assert len({(p.params.nx_harmonics, p.stack.num_layers) for p in pbs}) > 3   # several groups
    for i, pb in enumerate(pbs):
        ref = oracle_solve(pb)
        assert st[i] == 0, (i, st[i])
        assert np.abs(R[i] - ref.R).max() <= TOL, (i, np.abs(R[i] - ref.R).max())
        assert np.abs(T[i] - ref.T).max() <= TOL, (i, np.abs(T[i] - ref.T).max())
        assert abs(Rt[i] - ref.R_tot) <= TOL and abs(Tt[i] - ref.T_tot) <= TOL


def test_batch_matches_single_solves(ctx):
    """Each problem of a C3 list solved alone gives the batch's answer."""
    rng = np.random.default_rng(3)
    pbs = [C.c3_request(rng, grid=64, m_max=9) for _ in range(24)]
    R, T, Rt, Tt, st = ctx.solve_batch(pbs)
    for i in (0, 5, 11, 17, 23):
        R1, T1, Rt1, Tt1, st1 = ctx.solve_sweep(pbs[i])
        assert np.abs(R1[0] - R[i]).max() <= 1e-12
        assert np.abs(T1[0] - T[i]).max() <= 1e-12
        assert st1[0] == st[i]


def test_batch_empty_and_invalid(ctx):
    from rcwa_b200 import lib as L
    R, T, Rt, Tt, st = ctx.solve_batch([])
    assert len(R) == 0
    pb = _mixed_list(count=1)[0]
    import dataclasses
    bad = C.Problem("bad", dataclasses.replace(pb.stack, Lx=-1.0), pb.sources, pb.params)
    with pytest.raises(L.RcwaError) as e:
        ctx.solve_batch([pb, bad])
    assert e.value.code == L.RCWA_ERR_INVALID


def test_server_roundtrip(ctx):
    """Requests submitted to the server (continuous batching, max_batch 5)
    come back equal to one rcwa_solve_batch call over the same list."""
    from rcwa_b200 import lib as L
    pbs = _mixed_list(seed=21, count=12)
    R, T, Rt, Tt, st = ctx.solve_batch(pbs)
    srv = L.Server(0, max_batch=5, max_queue=1000)
    try:
        tickets = [srv.submit(pb) for pb in pbs]
        for i, (tk, pb) in enumerate(zip(tickets, pbs)):
            done, Ri, Ti, Rti, Tti, sti = srv.poll(tk, pb, wait=True)
            assert done
            assert np.abs(Ri - R[i]).max() <= 1e-12 and np.abs(Ti - T[i]).max() <= 1e-12
            assert sti == st[i]
        n, p50, p99 = srv.stats()
        assert n == len(pbs) and 0.0 < p50 <= p99
        with pytest.raises(L.RcwaError) as e:
            srv.poll(tickets[0], pbs[0])       # already collected
        assert e.value.code == L.RCWA_ERR_NOTFOUND
    finally:
        srv.close()


def _long_request():
    """One slow request: harmonics 23 x 23 (n = 1058), six patterned layers."""
    g = [C.circle(128, 128, 520.0, 520.0, 150.0 + 10 * i, C.ref_eps(6.0 + i + 0.1j), 1.0) for i in range(6)]
    st = C.make_stack(520.0, 520.0, g, [60.0 + 10 * i for i in range(6)])
    return C.Problem("long", st, [C.SourceSpec(700.0, 0.2, 0.3, 0.6, 0.8)], C.ParamSpec(11, 11, 1.0, 1.0, 2.25, 1.0))


def test_server_short_requests_overtake_a_long_one(ctx):
    """Continuous batching across lanes: short requests submitted right after
    a long one finish while the long one is still running, and every result
    equals the same problem solved alone (FP64, 1e-10)."""
    from rcwa_b200 import lib as L
    long_pb = _long_request()
    shorts = _mixed_list(seed=31, count=4)
    srv = L.Server(0, max_batch=8, max_queue=100, lanes=2)
    try:
        t_long = srv.submit(long_pb)
        import time
        time.sleep(0.05)    # the long request is admitted first, on its own lane
        tks = [srv.submit(pb) for pb in shorts]
        res = [srv.poll(tk, pb, wait=True) for tk, pb in zip(tks, shorts)]
        done_long = srv.poll(t_long, long_pb, wait=False)[0]
        assert not done_long, "the short requests waited for the long one"
        rl = srv.poll(t_long, long_pb, wait=True)
        for pb, r in list(zip(shorts, res)) + [(long_pb, rl)]:
            R1, T1, Rt1, Tt1, st1 = ctx.solve_sweep(pb)
            assert r[5] == st1[0]
            assert np.abs(r[1] - R1[0]).max() <= TOL and np.abs(r[2] - T1[0]).max() <= TOL
        info = srv.info()
        assert info["completed"] == len(shorts) + 1 and info["in_flight"] == 0 and info["lanes"] == 2
    finally:
        srv.close()


def test_server_admission_by_device_footprint(ctx):
    """With a budget that holds about one request, submissions are queued (not
    refused), admitted as memory frees, and the admitted footprint never
    exceeds the budget; results match one batched solve of the list."""
    from rcwa_b200 import lib as L
    pbs = _mixed_list(seed=41, count=6)
    R, T, Rt, Tt, st = ctx.solve_batch(pbs)
    probe = L.Server(0, max_batch=8, max_queue=100, lanes=1)
    try:
        probe.poll(probe.submit(pbs[0]), pbs[0], wait=True)
        one = probe.info()["peak_admitted_bytes"]
    finally:
        probe.close()
    assert one > 0
    budget = int(1.5 * one)
    srv = L.Server(0, max_batch=8, max_queue=100, lanes=2, hbm_budget_bytes=budget)
    try:
        tks = [srv.submit(pb) for pb in pbs]
        for i, (tk, pb) in enumerate(zip(tks, pbs)):
            done, Ri, Ti, Rti, Tti, sti = srv.poll(tk, pb, wait=True)
            assert done and sti == st[i]
            assert np.abs(Ri - R[i]).max() <= 1e-12 and np.abs(Ti - T[i]).max() <= 1e-12
        info = srv.info()
        assert info["completed"] == len(pbs) and info["rejected"] == 0
        assert info["budget_bytes"] == budget
        # a single request above the budget would run alone; these all fit, so
        # the footprint in flight stayed within it
        assert 0 < info["peak_admitted_bytes"] <= budget
    finally:
        srv.close()


def test_server_backpressure(ctx):
    """A full queue refuses with RCWA_ERR_BUSY and counts the refusal."""
    from rcwa_b200 import lib as L
    long_pb = _long_request()
    srv = L.Server(0, max_batch=1, max_queue=1, lanes=1)
    try:
        t0 = srv.submit(long_pb)        # admitted at once
        import time
        time.sleep(0.05)
        t1 = srv.submit(long_pb)        # waits in the queue
        with pytest.raises(L.RcwaError) as e:
            srv.submit(long_pb)
        assert e.value.code == L.RCWA_ERR_BUSY
        srv.poll(t0, long_pb, wait=True)
        srv.poll(t1, long_pb, wait=True)
        assert srv.info()["rejected"] == 1
    finally:
        srv.close()


def test_server_mixed_precision(ctx):
    """A mixed-precision server: every result within 1e-6 of the FP64 batch."""
    from rcwa_b200 import lib as L
    pbs = _mixed_list(seed=51, count=8)
    R, T, Rt, Tt, st = ctx.solve_batch(pbs)
    srv = L.Server(0, max_batch=4, max_queue=100, precision=L.PREC_MIXED, lanes=2)
    try:
        tks = [srv.submit(pb) for pb in pbs]
        for i, (tk, pb) in enumerate(zip(tks, pbs)):
            done, Ri, Ti, Rti, Tti, sti = srv.poll(tk, pb, wait=True)
            assert done and sti == st[i]
            assert np.abs(Ri - R[i]).max() <= 1e-6 and np.abs(Ti - T[i]).max() <= 1e-6
    finally:
        srv.close()
