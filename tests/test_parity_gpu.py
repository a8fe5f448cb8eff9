"""GPU path (through the C-ABI) against the CPU oracle: bit-exact trajectories.

Every case compares, per iteration, the chosen flat move index, its key, the
objective bookkeeping (cur/best) and the tenures; then the final positions,
tabu list and contributions, and the best solution.  The cases run both pair
sweeps (``sweep``): the tile pass (one structure query per column for a tile
of 32 rows) and the per-row pass, which the library picks by instance size.
"""
import numpy as np
import pytest

import ts_b200 as T
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STRUCTS = T.STRUCT_NAMES
SWEEPS = pytest.mark.parametrize("sweep", [T.PASS_TILE, T.PASS_ROWS], ids=["tile", "rows"])


def rand_graph(n, p, seed, wlo=1, whi=1000, dup=False, selfloops=False):
    rng = np.random.default_rng(seed)
    a, b = np.triu_indices(n, 1)
    keep = rng.random(len(a)) < p
    u, v = a[keep], b[keep]
    if dup and len(u):
        k = rng.integers(0, len(u), size=max(1, len(u) // 5))
        u2, v2 = v[k], u[k]
        u = np.concatenate([u, u2])
        v = np.concatenate([v, v2])
    if selfloops:
        s = rng.integers(0, n, size=4)
        u = np.concatenate([u, s])
        v = np.concatenate([v, s])
    w = rng.integers(wlo, whi + 1, size=len(u))
    return u.astype(np.int32), v.astype(np.int32), w.astype(np.int32)


def node_weight_graph(n, avg_deg, seed):
    u, v, w, _ = T.gen.erdos_renyi(n, avg_deg, seed)
    return u, v, w


def compare_run(problem, kind, n, u, v, w, *, m=0, iters, tenure_policy, tenure=0, maxt=200,
                piter=500, gamma=150, seed=1, initial=None, step_chunks=(None,), sweep=T.PASS_AUTO):
    drop = problem == T.PROBLEM_MDP
    og = O.Graph(n, u, v, w, drop_self_loops=drop)
    ores = O.run(og, O.MDP if problem == T.PROBLEM_MDP else O.MAXBS, m=m, max_iter=iters,
                 tenure_policy=tenure_policy, tenure=tenure, maxt=maxt, piter=piter, gamma=gamma,
                 seed=seed, initial=initial, threads=0)
    g = T.Graph(n, u, v, w, kind, drop_self_loops=drop)
    s = T.Solver(g, problem, m=m, max_iter=iters, tenure_policy=tenure_policy, tenure=tenure,
                 maxt=maxt, piter=piter, gamma=gamma, seed=seed, trace=True, sweep=sweep)
    try:
        s.init(initial)
        done = 0
        for c in step_chunks:
            done += s.step(iters if c is None else c)
        if step_chunks[-1] is not None:
            done += s.step(iters)
        tr = s.trace()
        res = s.result()
        sol, pos, tab, vg = s.state()
    finally:
        s.close()
        g.close()
    assert len(tr) == len(ores.trace), (len(tr), len(ores.trace))
    for f in ("iter", "idx", "key", "cur", "best", "kind", "tenure", "tenure2"):
        if not np.array_equal(tr[f], ores.trace[f]):
            bad = np.nonzero(tr[f] != ores.trace[f])[0][0]
            raise AssertionError(f"{kind}: trace field {f} differs first at record {bad}: "
                                 f"gpu={tr[bad]} oracle={ores.trace[bad]}")
    assert res.iterations == ores.iterations == done
    assert res.evaluations == ores.evaluations
    assert res.cur == ores.cur and res.best == ores.best
    assert res.best_true == ores.best_true
    assert res.stopped == ores.stopped
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
    return ores


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_mdp_small_ref_tenure(gpu, kind, seed, sweep):
    n, m = 60, 10
    u, v, w = rand_graph(n, 0.3, seed, whi=50)
    compare_run(T.PROBLEM_MDP, kind, n, u, v, w, m=m, iters=400, tenure_policy=T.TENURE_REF,
                seed=seed, sweep=sweep)


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
def test_mdp_config1_shape(gpu, kind, sweep):
    # ER n=2000, mean degree 20, m=200, fixed tenure 20 (C2=14), reference random start.
    c = T.gen.config1()
    compare_run(T.PROBLEM_MDP, kind, c["n"], c["u"], c["v"], c["w"], m=c["m"], iters=300,
                tenure_policy=T.TENURE_FIXED, tenure=20, seed=1, sweep=sweep)


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
def test_mdp_all_tabu_break(gpu, kind, sweep):
    n, m = 8, 4
    a, b = np.triu_indices(n, 1)
    w = np.full(len(a), 7, np.int32)
    o = compare_run(T.PROBLEM_MDP, kind, n, a.astype(np.int32), b.astype(np.int32), w, m=m,
                    iters=100, tenure_policy=T.TENURE_FIXED, tenure=50,
                    initial=np.array([0, 1, 2, 3], np.int32), sweep=sweep)
    assert o.stopped


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
def test_mdp_duplicates_ties_and_extremes(gpu, kind, sweep):
    # duplicated edges (contributions sum, lookup = first entry), uniform weights (ties)
    n = 50
    u, v, w = rand_graph(n, 0.25, 9, dup=True)
    compare_run(T.PROBLEM_MDP, kind, n, u, v, w, m=7, iters=200, tenure_policy=T.TENURE_FIXED,
                tenure=6, seed=4, sweep=sweep)
    u, v, _ = rand_graph(n, 0.3, 10)
    compare_run(T.PROBLEM_MDP, kind, n, u, v, np.full(len(u), 3, np.int32), m=9, iters=200,
                tenure_policy=T.TENURE_REF, seed=5, sweep=sweep)
    # m = 1 and m = n-1
    compare_run(T.PROBLEM_MDP, kind, n, u, v, np.full(len(u), 3, np.int32), m=1, iters=50,
                tenure_policy=T.TENURE_FIXED, tenure=2, seed=6, sweep=sweep)
    compare_run(T.PROBLEM_MDP, kind, n, u, v, np.full(len(u), 3, np.int32), m=n - 1, iters=50,
                tenure_policy=T.TENURE_FIXED, tenure=2, seed=7, sweep=sweep)
    # no edges at all
    e = np.zeros(0, np.int32)
    compare_run(T.PROBLEM_MDP, kind, n, e, e, e, m=5, iters=30, tenure_policy=T.TENURE_FIXED,
                tenure=3, seed=8, sweep=sweep)


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
@pytest.mark.parametrize("seed", [1, 2])
def test_maxbs_small_penalised_and_perturbed(gpu, kind, seed, sweep):
    n = 41
    u, v, w = rand_graph(n, 0.25, 20 + seed, whi=60)
    compare_run(T.PROBLEM_MAXBS, kind, n, u, v, w, iters=300, tenure_policy=T.TENURE_FIXED,
                tenure=30, piter=25, gamma=12, seed=seed, sweep=sweep)


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
def test_maxbs_ref_tenure_perturbation(gpu, kind, sweep):
    n = 500
    u, v, w = node_weight_graph(n, 12.0, 3)
    o = compare_run(T.PROBLEM_MAXBS, kind, n, u, v, w, iters=600, tenure_policy=T.TENURE_REF,
                    maxt=40, piter=40, gamma=30, seed=3, sweep=sweep)
    assert (o.trace["kind"] == O.REC_PERTURB).any()


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
def test_maxbs_odd_n_selfloops_and_steps(gpu, kind, sweep):
    n = 201
    u, v, w = rand_graph(n, 0.05, 31, selfloops=True)
    compare_run(T.PROBLEM_MAXBS, kind, n, u, v, w, iters=250, tenure_policy=T.TENURE_FIXED,
                tenure=7, piter=30, gamma=20, seed=9, step_chunks=(1, 17, 100), sweep=sweep)


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
def test_maxbs_explicit_partition(gpu, kind, sweep):
    n = 300
    u, v, w = node_weight_graph(n, 9.0, 4)
    part = np.ones(n, np.int32)
    part[np.arange(0, n, 2)[: n // 2]] = 0
    compare_run(T.PROBLEM_MAXBS, kind, n, u, v, w, iters=200, tenure_policy=T.TENURE_FIXED,
                tenure=10, piter=50, gamma=40, seed=12, initial=part, sweep=sweep)


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
@pytest.mark.parametrize("n,p", [(120, 0.2), (2600, 0.01)])
def test_maxbs_negative_weights(gpu, kind, n, p, sweep):
    # Weights of both signs (the instance readers accept negative fixed-point
    # weights): no sweep may assume w >= 0 for adjacent pairs.  n = 2600 puts
    # several 1024-column passes in a row.
    u, v, w = rand_graph(n, p, 41 + n, wlo=-1000, whi=1000)
    compare_run(T.PROBLEM_MAXBS, kind, n, u, v, w, iters=200, tenure_policy=T.TENURE_FIXED,
                tenure=15, piter=40, gamma=20, seed=5, sweep=sweep)


@SWEEPS
@pytest.mark.parametrize("kind", STRUCTS)
def test_mdp_negative_weights(gpu, kind, sweep):
    n, m = 300, 40
    u, v, w = rand_graph(n, 0.1, 77, wlo=-500, whi=500)
    compare_run(T.PROBLEM_MDP, kind, n, u, v, w, m=m, iters=300, tenure_policy=T.TENURE_FIXED,
                tenure=10, seed=4, sweep=sweep)


def test_lookup_interface_all_structures(gpu):
    n = 3000
    u, v, w = rand_graph(n, 0.002, 41, dup=True)
    og = O.Graph(n, u, v, w, drop_self_loops=True)
    rng = np.random.default_rng(0)
    qa = np.concatenate([u, rng.integers(0, n, 5000).astype(np.int32)])
    qb = np.concatenate([v, rng.integers(0, n, 5000).astype(np.int32)])
    expect = np.array([og.lookup(int(a), int(b)) for a, b in zip(qa, qb)], np.int32)
    for kind in STRUCTS:
        g = T.Graph(n, u, v, w, kind)
        got = g.lookup(qa, qb)
        g.close()
        np.testing.assert_array_equal(got, expect, err_msg=kind)


def test_hash_no_aliasing_beyond_16_bits(gpu):
    # (u<<16)|v in uint32 aliases once ids exceed 65,535 (GPU-MDP-Hash.cu:175,421):
    # (1, 70000) and (2, 70000 - 65536) share a key there; here they must not.
    n = 70_001
    u = np.array([1, 2, 5, 65_535], np.int32)
    v = np.array([70_000, 70_000 - 65_536, 69_999, 70_000], np.int32)
    w = np.array([11, 22, 33, 44], np.int32)
    for kind in STRUCTS:
        g = T.Graph(n, u, v, w, kind)
        got = g.lookup(np.concatenate([u, v, [3]]), np.concatenate([v, u, [7]]))
        g.close()
        np.testing.assert_array_equal(got, [11, 22, 33, 44, 11, 22, 33, 44, 0], err_msg=kind)


def test_graph_info_and_errors(gpu):
    u, v, w = rand_graph(100, 0.1, 2)
    g = T.Graph(100, u, v, w, "hash")
    gi = g.info()
    assert gi.n == 100 and gi.num_edges == len(u) and gi.num_entries == 2 * len(u)
    assert gi.hash_slots >= gi.num_entries
    g.close()
    with pytest.raises(T.TsError) as e:
        T.Graph(10, np.array([0], np.int32), np.array([10], np.int32), np.array([1], np.int32))
    assert e.value.status == 1
    g = T.Graph(10, np.array([0], np.int32), np.array([1], np.int32), np.array([1], np.int32))
    with pytest.raises(T.TsError):
        T.Solver(g, T.PROBLEM_MDP, m=10)
    s = T.Solver(g, T.PROBLEM_MDP, m=3)
    with pytest.raises(T.TsError) as e:
        s.step(1)
    assert e.value.status == 6
    with pytest.raises(T.TsError):
        s.init(np.array([1, 1, 2], np.int32))
    s.close()
    s = T.Solver(g, T.PROBLEM_MAXBS)
    with pytest.raises(T.TsError):
        s.init(np.zeros(10, np.int32))
    s.close()
    g.close()


@pytest.mark.parametrize("kind", ["csr", "wswap", "csr-bb", "hash"])
def test_int64_keys(gpu, kind):
    # 4 * max weighted degree >= 2^30 selects 64-bit pair keys
    n = 120
    u, v, _ = rand_graph(n, 0.1, 44)
    w = np.random.default_rng(3).integers(1 << 26, 1 << 27, size=len(u)).astype(np.int32)
    compare_run(T.PROBLEM_MDP, kind, n, u, v, w, m=20, iters=150, tenure_policy=T.TENURE_FIXED,
                tenure=9, seed=2)
    compare_run(T.PROBLEM_MAXBS, kind, n, u, v, w, iters=150, tenure_policy=T.TENURE_FIXED,
                tenure=9, piter=20, gamma=10, seed=2)


@pytest.mark.parametrize("kind", ["csr", "hash", "csr-bitset-bb"])
def test_caller_supplied_perturbation_stream(gpu, kind):
    # ts_solver_set_perturbations: the search uses the caller's events, here the
    # stream of another seed; the oracle with that seed must agree move for move
    n = 160
    u, v, w = node_weight_graph(n, 7.0, 21)
    part = np.ones(n, np.int32)
    part[np.arange(0, n, 2)] = 0
    iters, piter, gamma = 400, 15, 16
    events = iters // piter + 1
    draws = T.perturb_draws(n, 99, gamma, False, events)
    og = O.Graph(n, u, v, w, drop_self_loops=False)
    o = O.run(og, O.MAXBS, max_iter=iters, tenure_policy=T.TENURE_FIXED, tenure=12, piter=piter, gamma=gamma,
              seed=99, initial=part, threads=0)
    g = T.Graph(n, u, v, w, kind, drop_self_loops=False)
    s = T.Solver(g, T.PROBLEM_MAXBS, max_iter=iters, tenure_policy=T.TENURE_FIXED, tenure=12, piter=piter,
                 gamma=gamma, seed=5, trace=True)
    try:
        s.init(part)
        s.set_perturbations(draws)
        s.step(iters)
        tr = s.trace()
        r = s.result()
        assert (o.trace["kind"] == O.REC_PERTURB).any()
        for f in ("iter", "idx", "key", "cur", "best", "kind"):
            np.testing.assert_array_equal(tr[f], o.trace[f])
        assert (r.best, r.best_true, r.cur) == (o.best, o.best_true, o.cur)
        # too few events: the search stops with a device error instead of inventing moves
        s.init(part)
        s.set_perturbations(draws[:1])
        with pytest.raises(T.TsError) as ei:
            s.step(iters)
        assert ei.value.status == 5
        s.init(part)
        s.step(1)
        with pytest.raises(T.TsError):
            s.set_perturbations(draws)  # only before the first step
    finally:
        s.close()
        g.close()


def hub_graph(n, seed, hubs=((24, 5000), (24, 1500)), base_deg=10):
    """Erdos-Renyi background plus groups of hub vertices joined to random
    vertices: (count, degree) per group.  The 32 largest degrees exceed one
    tile index many times over, so the tile pass splits tiles over CTAs."""
    rng = np.random.default_rng(seed)
    u, v, w, _ = T.gen.erdos_renyi(n, base_deg, seed)
    us, vs = [u], [v]
    ids = rng.permutation(n)
    k = 0
    for count, deg in hubs:
        for h in ids[k:k + count]:
            nb = rng.choice(n, size=deg, replace=False)
            nb = nb[nb != h]
            us.append(np.full(len(nb), h, np.int32))
            vs.append(nb.astype(np.int32))
        k += count
    u = np.concatenate(us).astype(np.int32)
    v = np.concatenate(vs).astype(np.int32)
    w = rng.integers(1, 1000, size=len(u)).astype(np.int32)
    return u, v, w


@pytest.mark.parametrize("kind", ["hash", "csr-bitset", "csr-bb", "csr-bitset-bb"])
@pytest.mark.parametrize("problem", [T.PROBLEM_MDP, T.PROBLEM_MAXBS], ids=["mdp", "maxbs"])
def test_tile_slices_with_hub_rows(gpu, kind, problem):
    # hubs of degree 5,000 (more entries than a tile index holds: heavy rows)
    # and 1,500; MDP pulls them into the solution within a few iterations
    n = 6000
    u, v, w = hub_graph(n, 17)
    mdp = problem == T.PROBLEM_MDP
    m = 600 if mdp else 0
    g = T.Graph(n, u, v, w, kind, drop_self_loops=mdp)
    s = T.Solver(g, problem, m=m, max_iter=10, tenure_policy=T.TENURE_FIXED, tenure=20, seed=1,
                 sweep=T.PASS_TILE)
    try:
        info = s.info()
        assert info.slices > 1 and info.grid % info.slices == 0
    finally:
        s.close()
        g.close()
    compare_run(problem, kind, n, u, v, w, m=m, iters=200 if mdp else 100, tenure_policy=T.TENURE_FIXED,
                tenure=20, sweep=T.PASS_TILE, step_chunks=(37, None))
