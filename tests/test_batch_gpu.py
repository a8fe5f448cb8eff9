"""Batched form (ts_batch_*) against the plain solver and the oracle.

Every solve of a batch must give, bit for bit, what the plain one-instance path
gives for the same graph, parameters and start: iterations, evaluation count,
objective bookkeeping, best objective recomputed from the graph and the best
solution itself -- whatever group, cluster size, slot or replay it ran in.
"""
import numpy as np
import pytest

import ts_b200 as T
from oracle import oracle as O
from test_parity_gpu import node_weight_graph, rand_graph

pytestmark = pytest.mark.gpu


def plain(spec):
    s = T.Solver(spec.graph, spec.problem, m=spec.m, max_iter=spec.max_iter,
                 tenure_policy=spec.tenure_policy, tenure=spec.tenure, maxt=spec.maxt,
                 piter=spec.piter, gamma=spec.gamma, seed=spec.seed, sweep=spec.sweep)
    try:
        s.init(spec.initial)
        s.step(spec.max_iter)
        return s.result()
    finally:
        s.close()


def assert_same(a, b, what=""):
    fa = (a.iterations, a.evaluations, a.cur, a.best, a.best_true, a.perturbations, a.stopped,
          a.device_error)
    fb = (b.iterations, b.evaluations, b.cur, b.best, b.best_true, b.perturbations, b.stopped,
          b.device_error)
    assert fa == fb, f"{what}: batch {fa} != plain {fb}"
    np.testing.assert_array_equal(a.best_sol, b.best_sol, err_msg=what)


def graph(n, u, v, w, kind, problem):
    return T.Graph(n, u, v, w, kind, drop_self_loops=problem == T.PROBLEM_MDP)


def mixed_specs(kind, sweep=T.PASS_AUTO):
    """MDP and MaxBS solves on small graphs, seeded and explicit starts."""
    specs, graphs = [], []
    for seed in (1, 2):
        u, v, w = rand_graph(60, 0.3, seed, whi=50)
        g = graph(60, u, v, w, kind, T.PROBLEM_MDP)
        graphs.append(g)
        specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=10, max_iter=400, seed=seed))
        specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=17, max_iter=150,
                                    tenure_policy=T.TENURE_FIXED, tenure=5, seed=seed + 10,
                                    initial=np.arange(3, 20, dtype=np.int32)))
    u, v, w = node_weight_graph(300, 9.0, 4)
    g = graph(300, u, v, w, kind, T.PROBLEM_MDP)
    graphs.append(g)
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=30, max_iter=300, tenure_policy=T.TENURE_FIXED,
                                tenure=20, seed=3))
    for seed in (1, 2):
        u, v, w = rand_graph(41, 0.25, 20 + seed, whi=60)
        g = graph(41, u, v, w, kind, T.PROBLEM_MAXBS)
        graphs.append(g)
        specs.append(T.BatchJobSpec(g, T.PROBLEM_MAXBS, max_iter=300, tenure_policy=T.TENURE_FIXED,
                                    tenure=30, piter=25, gamma=12, seed=seed))
    u, v, w = rand_graph(201, 0.05, 31, selfloops=True)
    g = graph(201, u, v, w, kind, T.PROBLEM_MAXBS)
    graphs.append(g)
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MAXBS, max_iter=250, tenure_policy=T.TENURE_FIXED,
                                tenure=7, piter=30, gamma=20, seed=9))
    u, v, w = node_weight_graph(500, 12.0, 3)
    g = graph(500, u, v, w, kind, T.PROBLEM_MAXBS)
    graphs.append(g)
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MAXBS, max_iter=600, tenure_policy=T.TENURE_REF,
                                maxt=40, piter=40, gamma=30, seed=3))
    part = np.ones(500, np.int32)
    part[np.arange(0, 500, 2)] = 0
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MAXBS, max_iter=200, tenure_policy=T.TENURE_FIXED,
                                tenure=10, piter=50, gamma=40, seed=12, initial=part))
    for sp in specs:
        sp.sweep = sweep
    return specs, graphs


@pytest.mark.parametrize("sweep", [T.PASS_TILE, T.PASS_ROWS], ids=["tile", "rows"])
@pytest.mark.parametrize("kind", T.STRUCT_NAMES)
def test_batch_matches_plain(gpu, kind, sweep):
    specs, graphs = mixed_specs(kind, sweep)
    got = T.batch_solve(specs)
    for q, s in enumerate(specs):
        assert_same(got[q], plain(s), f"{kind} job {q}")
    for g in graphs:
        g.close()


def test_batch_all_structures_in_one_launch_and_replay(gpu):
    specs, graphs = [], []
    for kind in T.STRUCT_NAMES:
        sp, gr = mixed_specs(kind)
        specs += sp
        graphs += gr
    b = T.Batch(specs)
    info = b.info()
    assert info.jobs == len(specs) and info.groups >= len(T.STRUCT_NAMES) * 2
    first = b.run()
    again = b.run()  # a replay recomputes every solve from its start
    for q in range(len(specs)):
        assert_same(again[q], first[q], f"replay job {q}")
        assert_same(first[q], plain(specs[q]), f"job {q}")
    b.close()
    for g in graphs:
        g.close()


@pytest.mark.parametrize("sweep", [T.PASS_TILE, T.PASS_ROWS], ids=["tile", "rows"])
@pytest.mark.parametrize("kind", ["csr", "wswap", "csr-bitset-bb", "hash", "csr-bb", "csr-bitset"])
def test_cluster_sizes_agree_with_oracle(gpu, kind, sweep):
    c = T.gen.config1()
    n, m = c["n"], c["m"]
    g = graph(n, c["u"], c["v"], c["w"], kind, T.PROBLEM_MDP)
    specs = [T.BatchJobSpec(g, T.PROBLEM_MDP, m=m, max_iter=200, tenure_policy=T.TENURE_FIXED,
                            tenure=20, seed=1, cluster=cs, sweep=sweep) for cs in (1, 2, 4, 8)]
    u, v, w = node_weight_graph(1500, 10.0, 7)
    gb = graph(1500, u, v, w, kind, T.PROBLEM_MAXBS)
    specs += [T.BatchJobSpec(gb, T.PROBLEM_MAXBS, max_iter=300, tenure_policy=T.TENURE_FIXED,
                             tenure=25, piter=60, gamma=50, seed=5, cluster=cs, sweep=sweep)
              for cs in (1, 2, 4, 8)]
    got = T.batch_solve(specs)
    og = O.Graph(n, c["u"], c["v"], c["w"], drop_self_loops=True)
    om = O.run(og, O.MDP, m=m, max_iter=200, tenure_policy=T.TENURE_FIXED, tenure=20, seed=1, threads=0)
    ogb = O.Graph(1500, u, v, w, drop_self_loops=False)
    ob = O.run(ogb, O.MAXBS, max_iter=300, tenure_policy=T.TENURE_FIXED, tenure=25, piter=60, gamma=50,
               seed=5, threads=0)
    for q, r in enumerate(got):
        o = om if q < 4 else ob
        assert (r.iterations, r.evaluations, r.cur, r.best, r.best_true, r.stopped) == \
               (o.iterations, o.evaluations, o.cur, o.best, o.best_true, o.stopped), f"{kind} job {q}"
        assert r.device_error == 0
    for q in (1, 2, 3):
        np.testing.assert_array_equal(got[q].best_sol, got[0].best_sol)
        np.testing.assert_array_equal(got[4 + q].best_sol, got[4].best_sol)
    g.close()
    gb.close()


def test_slot_reuse_many_uneven_solves(gpu):
    # 3 slots per group, ~30 solves each: every slot runs many solves in turn
    rng = np.random.default_rng(5)
    specs, graphs = [], []
    for q in range(120):
        n = int(rng.integers(20, 400))
        u, v, w = node_weight_graph(n, float(rng.uniform(3, 12)), 100 + q)
        problem = T.PROBLEM_MDP if q % 2 == 0 else T.PROBLEM_MAXBS
        g = graph(n, u, v, w, "csr" if q % 4 < 2 else "csr-bb", problem)
        graphs.append(g)
        m = max(1, int(n * rng.uniform(0.05, 0.2)))
        specs.append(T.BatchJobSpec(g, problem, m=m, max_iter=int(rng.integers(0, 300)),
                                    tenure_policy=T.TENURE_FIXED, tenure=int(rng.integers(1, 15)),
                                    piter=int(rng.integers(5, 60)), gamma=int(rng.integers(2, 40)),
                                    seed=int(rng.integers(1, 1 << 31)), cluster=1))
    got = T.batch_solve(specs, max_slots=3)
    for q, s in enumerate(specs):
        assert_same(got[q], plain(s), f"job {q}")
    for g in graphs:
        g.close()


@pytest.mark.parametrize("kind", T.STRUCT_NAMES)
def test_batch_edge_cases(gpu, kind):
    graphs, specs = [], []
    n = 8
    a, b = np.triu_indices(n, 1)
    g = graph(n, a.astype(np.int32), b.astype(np.int32), np.full(len(a), 7, np.int32), kind, T.PROBLEM_MDP)
    graphs.append(g)
    # all-tabu break (the reference's value == -INF exit)
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=4, max_iter=100, tenure_policy=T.TENURE_FIXED,
                                tenure=50, initial=np.array([0, 1, 2, 3], np.int32)))
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=4, max_iter=0))
    n = 50
    u, v, _ = rand_graph(n, 0.3, 10)
    g = graph(n, u, v, np.full(len(u), 3, np.int32), kind, T.PROBLEM_MDP)
    graphs.append(g)
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=1, max_iter=50, tenure_policy=T.TENURE_FIXED, tenure=2))
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=n - 1, max_iter=50, tenure_policy=T.TENURE_FIXED,
                                tenure=2, seed=7))
    e = np.zeros(0, np.int32)
    g = graph(n, e, e, e, kind, T.PROBLEM_MDP)
    graphs.append(g)
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MDP, m=5, max_iter=30, tenure_policy=T.TENURE_FIXED, tenure=3))
    g = graph(3, np.array([0], np.int32), np.array([2], np.int32), np.array([5], np.int32), kind,
              T.PROBLEM_MAXBS)
    graphs.append(g)
    specs.append(T.BatchJobSpec(g, T.PROBLEM_MAXBS, max_iter=20, tenure_policy=T.TENURE_FIXED, tenure=1,
                                piter=3, gamma=2))
    got = T.batch_solve(specs)
    assert got[0].stopped
    assert got[1].iterations == 0
    for q, s in enumerate(specs):
        assert_same(got[q], plain(s), f"{kind} job {q}")
    for g in graphs:
        g.close()


@pytest.mark.parametrize("kind", ["csr", "wswap", "csr-bb"])
def test_batch_int64_keys(gpu, kind):
    # 4 * max weighted degree >= 2^30: the 64-bit key path
    n = 120
    u, v, _ = rand_graph(n, 0.1, 44)
    w = np.random.default_rng(3).integers(1 << 26, 1 << 27, size=len(u)).astype(np.int32)
    specs, graphs = [], []
    for problem in (T.PROBLEM_MDP, T.PROBLEM_MAXBS):
        g = graph(n, u, v, w, kind, problem)
        graphs.append(g)
        assert 4 * g.info().max_weighted_degree >= 1 << 30
        specs.append(T.BatchJobSpec(g, problem, m=20, max_iter=150, tenure_policy=T.TENURE_FIXED,
                                    tenure=9, piter=20, gamma=10, seed=2))
    got = T.batch_solve(specs)
    for q, s in enumerate(specs):
        assert_same(got[q], plain(s), f"{kind} job {q}")
    for g in graphs:
        g.close()


def test_batch_rejects_bad_jobs(gpu):
    u, v, w = rand_graph(30, 0.3, 1)
    g = graph(30, u, v, w, "csr", T.PROBLEM_MDP)
    bad = [
        T.BatchJobSpec(g, T.PROBLEM_MDP, m=0),
        T.BatchJobSpec(g, T.PROBLEM_MDP, m=30),
        T.BatchJobSpec(g, T.PROBLEM_MDP, m=5, cluster=3),
        T.BatchJobSpec(g, T.PROBLEM_MDP, m=3, initial=np.array([1, 1, 2], np.int32)),
        T.BatchJobSpec(g, T.PROBLEM_MAXBS, initial=np.zeros(30, np.int32)),
    ]
    for spec in bad:
        with pytest.raises(T.TsError) as ei:
            T.batch_solve([spec])
        assert ei.value.status == 1
    g.close()


@pytest.mark.parametrize("kind", ["csr", "csr-bb", "wswap"])
def test_batch_negative_weights(gpu, kind):
    """Weights of both signs: the CSR sweep masks adjacent pairs (no w >= 0
    assumption) in every cluster size."""
    u, v, w = rand_graph(700, 0.02, 93, wlo=-1000, whi=1000)
    g = graph(700, u, v, w, kind, T.PROBLEM_MAXBS)
    gm = graph(700, u, v, w, kind, T.PROBLEM_MDP)
    specs = []
    for cl in (1, 2, 4):
        specs.append(T.BatchJobSpec(g, T.PROBLEM_MAXBS, max_iter=300, tenure_policy=T.TENURE_FIXED,
                                    tenure=20, piter=60, gamma=24, seed=cl, cluster=cl))
        specs.append(T.BatchJobSpec(gm, T.PROBLEM_MDP, m=70, max_iter=300, tenure_policy=T.TENURE_FIXED,
                                    tenure=10, seed=10 + cl, cluster=cl))
    res = T.batch_solve(specs)
    for q, (r, sp) in enumerate(zip(res, specs)):
        assert_same(r, plain(sp), f"job {q}")


_SHARED_KERNEL_CHILD = r"""
import sys
import numpy as np
sys.path[:0] = sys.argv[1:]
import ts_b200 as T
from test_batch_gpu import assert_same, plain

def sparse(n, seed):
    rng = np.random.default_rng(seed)
    u = rng.integers(0, n, size=3 * n).astype(np.int32)
    v = rng.integers(0, n, size=3 * n).astype(np.int32)
    w = rng.integers(1, 1000, size=3 * n).astype(np.int32)
    return u, v, w

# MDP over CSR stages 4 bytes per column of a tile: n - m = 15000 and 13000
# columns need 61440 and 53248 bytes of shared memory, both above the default
# 48 KB, in the same kernel instantiation but in two groups (cluster 2 and 1).
ga = T.Graph(16000, *sparse(16000, 1), "csr", drop_self_loops=True)
gb = T.Graph(14000, *sparse(14000, 2), "csr", drop_self_loops=True)
specs = [T.BatchJobSpec(ga, T.PROBLEM_MDP, m=1000, max_iter=60, seed=5, cluster=2),
         T.BatchJobSpec(gb, T.PROBLEM_MDP, m=1000, max_iter=20, seed=6, cluster=1)]
b = T.Batch(specs)
assert b.info().groups == 2
b.launch()
b.sync()
for q, (r, sp) in enumerate(zip(b.results(), specs)):
    assert_same(r, plain(sp), f"job {q}")
b.close()
print("ok")
"""


def test_groups_sharing_a_kernel_with_different_shared_memory(gpu):
    """Two groups of one kernel instantiation, the larger-staging one planned
    first: planning the second must not lower the kernel's shared-memory
    opt-in below what the first one's launch needs.  Runs in a fresh process
    so no earlier test has raised the opt-in already."""
    import os
    import subprocess
    import sys
    from conftest import PKG, ROOT
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run([sys.executable, "-c", _SHARED_KERNEL_CHILD, here, PKG, ROOT],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-3000:]
