"""GPU path against the CPU oracle at the benchmark configurations' full sizes.

The small-instance parity tests (test_parity_gpu.py) cannot reach the code
paths that only large instances take: rows above the staging budget left in
global memory, bitmap rows too large to stage, many column chunks per row,
multi-gigabyte WSwap matrices, 64-bit perturbation draws (more than 2^31 swap
pairs), hub rows of thousands of entries.  These tests run the configurations
the benchmark measures, each structure through the C-ABI, and compare with the
oracle (one oracle run per configuration: the trajectory does not depend on
the structure):

* config 1 -- MDP, Erdos-Renyi n = 2,000, mean degree 20, m = 200, tenure 20,
  all 10,000 iterations, with each of the two pair sweeps;
* config 3 -- MDP, Chung-Lu n = 200,000 (exponent 2.3, mean degree 50, max
  5,000), m = 2,000, tenure 100, all 500 iterations;
* config 2 -- Max Bisection, conflict graph n = 100,000 (2.5e9 pairs per
  iteration), tenure 50, 100 iterations from the seeded random partition;
* config 2 past perturbation events -- the same graph from a partition near a
  local optimum (the best one of a 40,000-iteration CSR run), Piter 50, so
  several perturbation events (75 random moves each, drawn over 2.5e9 pairs)
  fall inside 150 iterations.

Per iteration: flat move index, key, current and best objective, record kind
and tenures; at the end: positions, tabu list, contributions and the best
solution -- all bit-exact.
"""
import numpy as np
import pytest

import ts_b200 as T
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STRUCTS = T.STRUCT_NAMES


def gpu_run(problem, kind, wl, *, m, iters, tenure, piter=500, gamma=150, seed=1, initial=None,
            sweep=T.PASS_AUTO):
    drop = problem == T.PROBLEM_MDP
    g = T.Graph(wl["n"], wl["u"], wl["v"], wl["w"], kind, drop_self_loops=drop)
    s = T.Solver(g, problem, m=m, max_iter=iters, tenure_policy=T.TENURE_FIXED, tenure=tenure,
                 piter=piter, gamma=gamma, seed=seed, trace=True, sweep=sweep)
    try:
        s.init(initial)
        done = s.step(iters)
        return dict(done=done, trace=s.trace(), res=s.result(), state=s.state())
    finally:
        s.close()
        g.close()


def assert_same(kind, problem, n, got, ores):
    tr, res = got["trace"], got["res"]
    sol, pos, tab, vg = got["state"]
    assert len(tr) == len(ores.trace), (kind, len(tr), len(ores.trace))
    for f in ("iter", "idx", "key", "cur", "best", "kind", "tenure", "tenure2"):
        if not np.array_equal(tr[f], ores.trace[f]):
            bad = np.nonzero(tr[f] != ores.trace[f])[0][0]
            raise AssertionError(f"{kind}: trace field {f} differs first at record {bad}: "
                                 f"gpu={tr[bad]} oracle={ores.trace[bad]}")
    assert res.iterations == ores.iterations == got["done"]
    assert (res.evaluations, res.cur, res.best, res.best_true, res.stopped) == \
        (ores.evaluations, ores.cur, ores.best, ores.best_true, ores.stopped)
    assert res.device_error == 0
    np.testing.assert_array_equal(sol, ores.sol)
    np.testing.assert_array_equal(pos, ores.pos)
    np.testing.assert_array_equal(tab, ores.tab)
    np.testing.assert_array_equal(vg, ores.vg)
    if problem == T.PROBLEM_MDP:
        np.testing.assert_array_equal(res.best_sol, ores.best_sol)
    else:
        part = np.ones(n, np.int32)
        part[ores.best_sol[: n // 2]] = 0
        np.testing.assert_array_equal(res.best_sol, part)


# ---------------------------------------------------------------- config 1
@pytest.fixture(scope="module")
def c1():
    wl = T.gen.config1()
    og = O.Graph(wl["n"], wl["u"], wl["v"], wl["w"], drop_self_loops=True)
    ores = O.run(og, O.MDP, m=wl["m"], max_iter=10_000, tenure_policy=O.TENURE_FIXED, tenure=20,
                 seed=1, threads=0)
    return wl, ores


@pytest.mark.parametrize("sweep", [T.PASS_TILE, T.PASS_ROWS], ids=["tile", "rows"])
@pytest.mark.parametrize("kind", STRUCTS)
def test_config1_full_10000_iterations(gpu, c1, kind, sweep):
    wl, ores = c1
    got = gpu_run(T.PROBLEM_MDP, kind, wl, m=wl["m"], iters=10_000, tenure=20, sweep=sweep)
    assert_same(kind, T.PROBLEM_MDP, wl["n"], got, ores)


# ---------------------------------------------------------------- config 3
@pytest.fixture(scope="module")
def c3():
    wl = T.gen.config3()
    og = O.Graph(wl["n"], wl["u"], wl["v"], wl["w"], drop_self_loops=True)
    ores = O.run(og, O.MDP, m=wl["m"], max_iter=500, tenure_policy=O.TENURE_FIXED, tenure=100,
                 seed=1, threads=0)
    return wl, ores


@pytest.mark.parametrize("kind", STRUCTS)
def test_config3_full_500_iterations(gpu, c3, kind):
    wl, ores = c3
    deg = np.bincount(np.concatenate([wl["u"], wl["v"]]), minlength=wl["n"])
    assert deg.max() > 1000  # hub rows, far above any staging budget, are part of the case
    got = gpu_run(T.PROBLEM_MDP, kind, wl, m=wl["m"], iters=500, tenure=100)
    assert_same(kind, T.PROBLEM_MDP, wl["n"], got, ores)


# ---------------------------------------------------------------- config 2
@pytest.fixture(scope="module")
def c2_graph():
    return T.gen.config2()


@pytest.fixture(scope="module")
def c2(c2_graph):
    wl = c2_graph
    og = O.Graph(wl["n"], wl["u"], wl["v"], wl["w"], drop_self_loops=False)
    ores = O.run(og, O.MAXBS, max_iter=100, tenure_policy=O.TENURE_FIXED, tenure=50, piter=500,
                 gamma=150, seed=1, threads=0)
    return wl, ores


@pytest.mark.parametrize("kind", STRUCTS)
def test_config2_100_iterations(gpu, c2, kind):
    wl, ores = c2
    got = gpu_run(T.PROBLEM_MAXBS, kind, wl, m=0, iters=100, tenure=50)
    assert_same(kind, T.PROBLEM_MAXBS, wl["n"], got, ores)


@pytest.fixture(scope="module")
def c2_perturbed(gpu, c2_graph):
    wl = c2_graph
    n = wl["n"]
    # start near a local optimum: the best bisection of a long CSR run
    g = T.Graph(n, wl["u"], wl["v"], wl["w"], "csr", drop_self_loops=False)
    s = T.Solver(g, T.PROBLEM_MAXBS, max_iter=40_000, tenure_policy=T.TENURE_FIXED, tenure=50,
                 piter=10**9, gamma=150, seed=3)
    try:
        s.init(None)
        s.step(40_000)
        start = s.result().best_sol.astype(np.int32)
    finally:
        s.close()
        g.close()
    assert int((start == 0).sum()) == n // 2
    og = O.Graph(n, wl["u"], wl["v"], wl["w"], drop_self_loops=False)
    ores = O.run(og, O.MAXBS, max_iter=150, tenure_policy=O.TENURE_FIXED, tenure=50, piter=50,
                 gamma=150, seed=7, initial=start, threads=0)
    return wl, start, ores


@pytest.mark.parametrize("kind", STRUCTS)
def test_config2_past_perturbation_events(gpu, c2_perturbed, kind):
    wl, start, ores = c2_perturbed
    pert = ores.trace["kind"] == O.REC_PERTURB
    assert pert.sum() >= 75  # at least one whole event of 75 moves
    # draws over 2.5e9 pairs reach past the int32 range of the reference's index type
    assert ores.trace["idx"][pert].max() > 2**31 - 1
    got = gpu_run(T.PROBLEM_MAXBS, kind, wl, m=0, iters=150, tenure=50, piter=50, seed=7,
                  initial=start)
    assert_same(kind, T.PROBLEM_MAXBS, wl["n"], got, ores)
