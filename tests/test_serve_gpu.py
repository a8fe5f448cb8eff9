"""Served form (ts_server_*): every result equals the same solve run alone.

Requests of different problems, sizes and structures are submitted while
others run; some run packed (one cluster each of a shared persistent launch),
the large ones plain (their own stream).  Each result -- objective
bookkeeping, recomputed best objective, iteration and evaluation counts, best
solution -- must equal the plain solver's on the same graph and parameters.
"""
import time

import numpy as np
import pytest

import ts_b200 as T
from test_parity_gpu import node_weight_graph, rand_graph

pytestmark = pytest.mark.gpu


def alone(n, u, v, w, problem, kind, **kw):
    g = T.Graph(n, u, v, w, kind, drop_self_loops=problem == T.PROBLEM_MDP)
    s = T.Solver(g, problem, m=kw.get("m", 0), max_iter=kw["max_iter"], tenure_policy=kw["tenure_policy"],
                 tenure=kw["tenure"], piter=kw.get("piter", 500), gamma=kw.get("gamma", 150),
                 maxt=kw.get("maxt", 200), seed=kw["seed"])
    try:
        s.init(kw.get("initial"))
        s.step(kw["max_iter"])
        return s.result()
    finally:
        s.close()
        g.close()


def requests():
    rng = np.random.default_rng(11)
    out = []
    for q in range(14):
        problem = T.PROBLEM_MDP if q % 3 else T.PROBLEM_MAXBS
        n = int(rng.integers(60, 900))
        u, v, w = node_weight_graph(n, float(rng.uniform(4, 14)), 300 + q)
        kind = T.STRUCT_NAMES[q % 6]
        kw = dict(max_iter=int(rng.integers(50, 400)), tenure_policy=T.TENURE_FIXED,
                  tenure=int(rng.integers(3, 25)), seed=int(rng.integers(1, 1 << 30)),
                  piter=int(rng.integers(10, 80)), gamma=int(rng.integers(4, 40)))
        if problem == T.PROBLEM_MDP:
            kw["m"] = max(2, n // 10)
        out.append((n, u, v, w, problem, kind, kw))
    # two large ones that run plain (pairs per iteration >= 2^20)
    u, v, w = node_weight_graph(2400, 10.0, 77)
    out.append((2400, u, v, w, T.PROBLEM_MAXBS, "csr",
                dict(max_iter=300, tenure_policy=T.TENURE_FIXED, tenure=40, seed=5, piter=60, gamma=40)))
    u, v, w = node_weight_graph(6000, 8.0, 78)
    out.append((6000, u, v, w, T.PROBLEM_MDP, "csr-bb",
                dict(m=600, max_iter=200, tenure_policy=T.TENURE_REF, tenure=15, seed=6)))
    # weights of both signs on the masked CSR path (packed)
    u, v, w = rand_graph(400, 0.03, 91, wlo=-1000, whi=1000)
    out.append((400, u, v, w, T.PROBLEM_MAXBS, "csr",
                dict(max_iter=250, tenure_policy=T.TENURE_FIXED, tenure=12, seed=9, piter=50, gamma=16)))
    # explicit starts
    n = 300
    u, v, w = rand_graph(n, 0.05, 90)
    part = np.ones(n, np.int32)
    part[np.arange(1, n, 2)] = 0
    out.append((n, u, v, w, T.PROBLEM_MAXBS, "hash",
                dict(max_iter=200, tenure_policy=T.TENURE_FIXED, tenure=9, seed=7, piter=30, gamma=12,
                     initial=part)))
    out.append((n, u, v, w, T.PROBLEM_MDP, "wswap",
                dict(m=30, max_iter=150, tenure_policy=T.TENURE_REF, tenure=15, seed=8,
                     initial=np.arange(0, 60, 2, dtype=np.int32))))
    return out


def test_served_results_equal_alone_results(gpu):
    reqs = requests()
    srv = T.Server(round_ms=2.0)
    tickets = {}
    try:
        # staggered arrivals: later requests join while earlier ones run
        for k, (n, u, v, w, problem, kind, kw) in enumerate(reqs):
            t = srv.submit(n, u, v, w, problem, kind=kind, **kw)
            tickets[t] = k
            if k % 4 == 3:
                time.sleep(0.01)
        got = {}
        deadline = time.time() + 300
        while len(got) < len(reqs) and time.time() < deadline:
            for d in srv.poll(wait_ms=50):
                got[d.ticket] = d
        st = srv.stats()
    finally:
        srv.close()
    assert len(got) == len(reqs)
    assert st.completed == len(reqs) and st.queued == 0 and st.active == 0
    execs = {d.executor for d in got.values()}
    assert execs == {"packed", "plain"}
    for t, d in got.items():
        n, u, v, w, problem, kind, kw = reqs[tickets[t]]
        assert d.status == 0, (t, d.status)
        a = alone(n, u, v, w, problem, kind, **kw)
        r = d.result
        assert (r.iterations, r.evaluations, r.cur, r.best, r.best_true, r.perturbations, r.stopped) == \
               (a.iterations, a.evaluations, a.cur, a.best, a.best_true, a.perturbations, a.stopped), (t, kind)
        np.testing.assert_array_equal(r.best_sol, a.best_sol)
        assert d.submit_s <= d.admit_s <= d.done_s
    # the work overlapped: some request was admitted before another one completed
    ds = list(got.values())
    assert any(a.admit_s < b.done_s and b.admit_s < a.done_s for i, a in enumerate(ds) for b in ds[i + 1:])


def test_server_budget_admits_fifo_and_reports_errors(gpu):
    u, v, w = node_weight_graph(400, 6.0, 3)
    srv = T.Server(max_bytes=1 << 20, round_ms=1.0)  # small budget: one request at a time
    try:
        t1 = srv.submit(400, u, v, w, T.PROBLEM_MDP, kind="csr", m=40, max_iter=100, seed=1)
        t2 = srv.submit(400, u, v, w, T.PROBLEM_MDP, kind="csr", m=40, max_iter=100, seed=2)
        bad = srv.submit(400, u, v, w, T.PROBLEM_MDP, kind="csr", m=4, max_iter=10,
                         initial=np.array([1, 1, 2, 3], np.int32))
        got = {}
        deadline = time.time() + 120
        while len(got) < 3 and time.time() < deadline:
            for d in srv.poll(wait_ms=50):
                got[d.ticket] = d
    finally:
        srv.close()
    assert got[t1].status == 0 and got[t2].status == 0
    assert got[t1].done_s <= got[t2].admit_s + 1e-6  # admitted only after the first one left
    assert got[bad].status == 1
    with pytest.raises(T.TsError):
        T.Server().submit(10, [0], [1], [1], T.PROBLEM_MDP, m=10)
