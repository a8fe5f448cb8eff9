"""The CPU oracle against known answers and an independent restatement."""
import numpy as np
import pytest

import naive
from oracle import oracle as O


def _rand_graph(n, p, seed, wlo=1, whi=50, dup=False, selfloops=False):
    rng = np.random.default_rng(seed)
    a, b = np.triu_indices(n, 1)
    keep = rng.random(len(a)) < p
    u, v = a[keep], b[keep]
    if dup and len(u):
        k = rng.integers(0, len(u), size=max(1, len(u) // 5))
        u = np.concatenate([u, v[k]])  # reversed duplicates
        v = np.concatenate([v, a[keep][k]])
    if selfloops:
        s = rng.integers(0, n, size=3)
        u = np.concatenate([u, s])
        v = np.concatenate([v, s])
    w = rng.integers(wlo, whi + 1, size=len(u))
    return u.astype(np.int32), v.astype(np.int32), w.astype(np.int32)


def test_tenure_tables_known_answers():
    # determine_tabu_tenure (GPU-MDP-CSR.cu:461-476)
    exp = {0: 15, 100: 15, 101: 30, 200: 30, 201: 15, 301: 60, 400: 60, 701: 120, 800: 120,
           801: 15, 901: 30, 1101: 60, 1301: 30, 1400: 30, 1401: 15, 1500: 15, 1601: 30}
    for it, t in exp.items():
        assert O.mdp_tenure(it) == t == naive.mdp_tenure(it)
    # round(0.7 * C1), half away from zero; 0.7*15 rounds to the double 10.5
    assert [O.mdp_c2(c) for c in (15, 30, 60, 120, 20, 100)] == [11, 21, 42, 84, 14, 70]
    # tabuTenure (GPU-MAXBS-CSR.cu:248-263), maxt=200: 25,50,25,100,... blocks of 4*tenure
    assert O.maxbs_tenure(0, 200) == 25
    assert O.maxbs_tenure(100, 200) == 25 and O.maxbs_tenure(101, 200) == 50
    assert O.maxbs_tenure(300, 200) == 50 and O.maxbs_tenure(301, 200) == 25
    assert O.maxbs_tenure(401, 200) == 100
    for it in range(0, 7000, 37):
        assert O.maxbs_tenure(it, 200) == naive.maxbs_tenure(it, 200)
        assert O.maxbs_tenure(it, 8) == naive.maxbs_tenure(it, 8)


def test_penalty_key_matches_float32():
    rng = np.random.default_rng(0)
    gs = np.concatenate([rng.integers(-2**30, 2**30, 5000), np.arange(-3000, 3000)])
    for g in gs:
        g = int(g)
        assert O.maxbs_penalty(g) == naive.penalty(g)
    # quantised to 1024 around -1e10; recovery leaves the 1023 residue
    assert O.maxbs_penalty(0) == -10000000000
    assert (O.maxbs_penalty(1234) + 9999999999) % 1024 == 1023


def test_round_f32_against_numpy():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.integers(-2**62, 2**62, 3000), rng.integers(-2**26, 2**26, 3000),
                         np.array([0, 1, -1, 2**24, 2**24 + 1, 2**24 + 3, 2**25 + 2])])
    for x in xs:
        assert O.round_f32(int(x)) == int(np.float32(np.float64(int(x)))) or abs(int(x)) >= 2**53


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
@pytest.mark.parametrize("tenure", [None, 3])
def test_mdp_oracle_equals_naive(seed, tenure):
    n, m = 14, 5
    u, v, w = _rand_graph(n, 0.45, seed, dup=(seed == 3), selfloops=(seed == 4))
    g = O.Graph(n, u, v, w, drop_self_loops=True)
    init = O.mdp_random_initial(n, m, seed)
    iters = 60
    r = O.run(g, O.MDP, m=m, max_iter=iters, initial=init,
              tenure_policy=O.TENURE_REF if tenure is None else O.TENURE_FIXED,
              tenure=tenure or 0)
    tr, cur, best = naive.run_mdp(n, list(zip(u.tolist(), v.tolist(), w.tolist())), m, init.tolist(),
                                  iters, tenure_fixed=tenure)
    assert len(r.trace) == len(tr)
    for rec, t in zip(r.trace, tr):
        assert rec["iter"] == t[0] and rec["idx"] == t[1] and rec["key"] == t[2]
        if t[3] != "break":
            assert rec["cur"] == t[3] and rec["best"] == t[4]
    assert r.cur == cur and r.best == best


@pytest.mark.parametrize("seed", [5, 6, 7])
@pytest.mark.parametrize("tenure", [None, 4])
def test_maxbs_oracle_equals_naive(seed, tenure):
    n = 13
    u, v, w = _rand_graph(n, 0.4, seed, selfloops=(seed == 7))
    g = O.Graph(n, u, v, w, drop_self_loops=False)
    part = O.maxbs_random_partition(n, seed)
    iters, piter, gamma = 70, 6, 6
    k = max(1, min(gamma, n) // 2)
    draws = O.maxbs_perturb_draws(n, seed, False, iters // piter + 2, k)
    r = O.run(g, O.MAXBS, max_iter=iters, initial=part, piter=piter, gamma=gamma, seed=seed,
              maxt=16, tenure_policy=O.TENURE_REF if tenure is None else O.TENURE_FIXED,
              tenure=tenure or 0)
    tr, cur, best = naive.run_maxbs(n, list(zip(u.tolist(), v.tolist(), w.tolist())), part.tolist(),
                                    iters, draws.tolist(), piter, tenure_fixed=tenure, maxt=16)
    assert len(r.trace) == len(tr)
    for rec, t in zip(r.trace, tr):
        assert (rec["iter"], rec["idx"], rec["key"], rec["cur"], rec["best"]) == t
    assert r.cur == cur and r.best == best


def test_mdp_break_on_all_tabu():
    # Complete graph with equal weights: after a few moves every pair is tabu and
    # nothing is aspirated -> the reference's value == -INF break.
    n, m = 6, 3
    a, b = np.triu_indices(n, 1)
    w = np.full(len(a), 7, np.int32)
    g = O.Graph(n, a, b, w, drop_self_loops=True)
    r = O.run(g, O.MDP, m=m, max_iter=100, initial=np.array([0, 1, 2], np.int32),
              tenure_policy=O.TENURE_FIXED, tenure=50)
    assert r.stopped
    assert r.trace[-1]["kind"] == O.REC_BREAK and r.trace[-1]["key"] == -99999
    assert r.iterations < 100


def test_maxbs_penalised_choice_when_all_tabu():
    n = 6
    a, b = np.triu_indices(n, 1)
    w = (np.arange(len(a)) % 5 + 1).astype(np.int32)
    g = O.Graph(n, a, b, w, drop_self_loops=False)
    part = np.array([0, 0, 0, 1, 1, 1], np.int32)
    r = O.run(g, O.MAXBS, max_iter=40, initial=part, tenure_policy=O.TENURE_FIXED, tenure=30,
              piter=1000, gamma=4)
    pen = r.trace["key"] < -2_500_000_000
    assert pen.any(), "expected penalised picks once everything is tabu"
    # recovered gains keep the 1023 residue of the 1024 quantisation
    for rec in r.trace[pen]:
        assert (rec["key"] + 9999999999) % 1024 == 1023


def test_objective_bookkeeping_matches_recompute():
    n, m = 40, 8
    u, v, w = _rand_graph(n, 0.2, 11)
    g = O.Graph(n, u, v, w, drop_self_loops=True)
    r = O.run(g, O.MDP, m=m, max_iter=200, seed=11, tenure_policy=O.TENURE_FIXED, tenure=5)
    assert r.best == r.best_true
    rows = naive.csr(n, list(zip(u.tolist(), v.tolist(), w.tolist())), True)
    inside = set(r.sol[:m].tolist())
    cur = sum(w for a in inside for (z, w) in rows[a] if z in inside) // 2
    assert cur == r.cur


def test_threads_do_not_change_result():
    n, m = 300, 40
    u, v, w = _rand_graph(n, 0.05, 12)
    g = O.Graph(n, u, v, w, drop_self_loops=True)
    r1 = O.run(g, O.MDP, m=m, max_iter=80, seed=3, threads=1, tenure_policy=O.TENURE_FIXED, tenure=10)
    r4 = O.run(g, O.MDP, m=m, max_iter=80, seed=3, threads=4, tenure_policy=O.TENURE_FIXED, tenure=10)
    assert np.array_equal(r1.trace, r4.trace)
