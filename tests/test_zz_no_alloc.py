"""ts_best_swap_noalloc: one iteration's decision without any device allocation.

Some callers cannot allocate device memory: plugins whose host application
owns all of the GPU's memory through its own pool, and services held to a
fixed device-memory budget.  They keep the graph and the tabu state in their own
buffers and ask the library which swap the next iteration makes; the library
then works in a fixed scratch array compiled into it.

This file checks, on two calls in a row (so the second call starts from the
scratch contents the first one left), that the decision equals the move the
regular solver entry point makes from the same state.  It is collected last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import ts_b200 as T
from ts_b200 import _capi as C

pytestmark = pytest.mark.gpu


def _entry():
    f = C.lib().ts_best_swap_noalloc
    f.restype = ctypes.c_int
    f.argtypes = ([ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                   ctypes.c_int64] + [ctypes.c_void_p] * 8)
    return f


def _csr(n, u, v, w, drop_self):
    """Rows sorted by neighbour id, stable in input order (the library's layout)."""
    a = np.concatenate([u, v]).astype(np.int64)
    b = np.concatenate([v, u]).astype(np.int64)
    ww = np.concatenate([w, w]).astype(np.int32)
    order = np.arange(len(u))
    seq = np.concatenate([order, order])  # both entries of edge e carry e
    if drop_self:
        keep = a != b
        a, b, ww, seq = a[keep], b[keep], ww[keep], seq[keep]
    idx = np.lexsort((seq, b, a))
    a, b, ww = a[idx], b[idx], ww[idx]
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, a + 1, 1)
    rowptr = np.cumsum(rowptr)
    return rowptr, b.astype(np.int32), ww


@pytest.mark.parametrize("problem", [T.PROBLEM_MDP, T.PROBLEM_MAXBS])
def test_noalloc_decision_matches_solver_twice(gpu, problem):
    import torch

    n = 3000
    u, v, w, _ = T.gen.erdos_renyi(n, 10.0, seed=17)
    m = 300 if problem == T.PROBLEM_MDP else n // 2
    g = T.Graph(n, u, v, w, "csr", drop_self_loops=problem == T.PROBLEM_MDP)
    s = T.Solver(g, problem, m=m, max_iter=1000, tenure_policy=T.TENURE_FIXED, tenure=9,
                 piter=10**6, gamma=150, seed=5, trace=True)
    try:
        s.init(None)
        s.step(40)
        rowptr, col, wt = _csr(n, u, v, w, problem == T.PROBLEM_MDP)
        dev = torch.device("cuda", torch.cuda.current_device())
        d_rowptr = torch.from_numpy(rowptr).to(dev)
        d_col = torch.from_numpy(col).to(dev)
        d_w = torch.from_numpy(wt).to(dev)
        out = torch.full((2,), -7, dtype=torch.int64, device=dev)
        f = _entry()
        stream = torch.cuda.current_stream(dev).cuda_stream
        for _ in range(2):
            sol, _pos, tab, vg = s.state()
            r = s.result()
            d_sol = torch.from_numpy(sol).to(dev)
            d_vg = torch.from_numpy(vg).to(dev)
            d_tab = torch.from_numpy(tab).to(dev)
            st = f(problem, n, m, r.iterations, r.cur, r.best, d_rowptr.data_ptr(), d_col.data_ptr(),
                   d_w.data_ptr(), d_sol.data_ptr(), d_vg.data_ptr(), d_tab.data_ptr(), out.data_ptr(),
                   stream)
            assert st == 0, C.lib().ts_last_error()
            torch.cuda.synchronize(dev)
            key, idx = (int(x) for x in out.tolist())
            assert s.step(1) == 1
            tr = s.trace()
            rec = tr[(tr["iter"] == r.iterations) & (tr["kind"] == 0)]
            assert len(rec) == 1
            assert (idx, key) == (int(rec[0]["idx"]), int(rec[0]["key"]))
    finally:
        s.close()
        g.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    f = _entry()
    too_big = 262144 + 1  # TS_NOALLOC_MAX_N + 1
    st = f(T.PROBLEM_MDP, too_big, 10, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, None)
    assert st == C.ERR_INVALID_ARG
    assert b"scratch" in C.lib().ts_last_error()
