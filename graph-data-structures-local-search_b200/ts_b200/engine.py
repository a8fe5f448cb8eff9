"""Host-side mirror of the reference's tabu-search operators over the C-ABI.

``Graph`` replaces the loaders/structure builders (read_instance/createCSR,
src/mdp/GPU-MDP-CSR.cu:210-367; load, src/maxbisection/GPU-MAXBS-CSR.cu:137-173;
the Hash/Bitset/WSwap builders of the variant files).  ``Solver`` replaces
``tabu_search(int *sol)`` (GPU-MDP-CSR.cu:611-693) and
``perturbationBasedTabuSearch`` (GPU-MAXBS-CSR.cu:401-512); the free functions
``tabu_search`` and ``perturbation_based_tabu_search`` keep those names and
argument meanings.  All compute runs in libts_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _capi as C


def struct_id(kind) -> int:
    if isinstance(kind, str):
        if kind not in C.STRUCT_NAMES:
            raise ValueError(f"unknown structure {kind!r}; one of {C.STRUCT_NAMES}")
        return C.STRUCT_NAMES.index(kind)
    k = int(kind)
    if not 0 <= k < len(C.STRUCT_NAMES):
        raise ValueError(f"unknown structure id {k}")
    return k


class Graph:
    """Undirected weighted graph + one lookup structure, resident on the GPU."""

    def __init__(self, n: int, u, v, w, kind="csr", *, drop_self_loops: bool = True,
                 stream: int | None = None, device_arrays: bool = False):
        C.lib()
        self.n = int(n)
        self.kind = struct_id(kind)
        h = ctypes.c_void_p()
        if device_arrays:
            # u, v, w expose __cuda_array_interface__ / data_ptr() (e.g. torch tensors).
            pu, pv, pw = (_dev_ptr(x) for x in (u, v, w))
            ne = int(_numel(u))
            C.check(C.lib().ts_graph_create_device(self.n, ne, pu, pv, pw, self.kind,
                                                   int(drop_self_loops), stream, ctypes.byref(h)),
                    "ts_graph_create_device")
        else:
            uu = np.ascontiguousarray(u, dtype=np.int32)
            vv = np.ascontiguousarray(v, dtype=np.int32)
            ww = np.ascontiguousarray(w, dtype=np.int32)
            if not (len(uu) == len(vv) == len(ww)):
                raise ValueError("u, v, w must have the same length")
            C.check(C.lib().ts_graph_create(self.n, len(uu), C.ptr(uu), C.ptr(vv), C.ptr(ww),
                                            self.kind, int(drop_self_loops), stream,
                                            ctypes.byref(h)), "ts_graph_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def info(self) -> C.GraphInfo:
        gi = C.GraphInfo()
        C.check(C.lib().ts_graph_info_get(self._h, ctypes.byref(gi)), "ts_graph_info_get")
        return gi

    def lookup(self, u, v) -> np.ndarray:
        uu = np.ascontiguousarray(u, dtype=np.int32)
        vv = np.ascontiguousarray(v, dtype=np.int32)
        out = np.zeros(len(uu), np.int32)
        C.check(C.lib().ts_lookup_host(self._h, len(uu), C.ptr(uu), C.ptr(vv), C.ptr(out)),
                "ts_lookup_host")
        return out

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            C.lib().ts_graph_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _numel(x) -> int:
    if hasattr(x, "numel"):
        return int(x.numel())
    return int(len(x))


def _dev_ptr(x):
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.__cuda_array_interface__["data"][0])


def default_params(problem: int) -> C.Params:
    p = C.Params()
    C.check(C.lib().ts_params_default(problem, ctypes.byref(p)), "ts_params_default")
    return p


@dataclass
class SolveResult:
    iterations: int
    evaluations: int
    cur: int
    best: int
    best_true: int
    perturbations: int
    stopped: bool
    best_sol: np.ndarray
    device_error: int


class Solver:
    """One tabu-search state on the device (positions, contributions, tabu list)."""

    def __init__(self, graph: Graph, problem: int, *, m: int = 0, max_iter: int = 50000,
                 tenure_policy: int = C.TENURE_REF, tenure: int = 15, maxt: int = 200,
                 piter: int = 500, gamma: int = 150, seed: int = 1, trace: bool = False,
                 sweep: int = C.PASS_AUTO):
        self.graph = graph
        p = default_params(problem)
        p.m = m
        p.max_iter = max_iter
        p.tenure_policy = tenure_policy
        p.tenure = tenure
        p.maxt = maxt
        p.piter = piter
        p.gamma = gamma
        p.seed = seed & 0xFFFFFFFF
        p.trace = int(trace)
        p.pass_ = int(sweep)
        self.params = p
        self.problem = problem
        h = ctypes.c_void_p()
        C.check(C.lib().ts_solver_create(graph.handle, ctypes.byref(p), ctypes.byref(h)),
                "ts_solver_create")
        self._h = h
        self.n = graph.n
        self.m = m if problem == C.PROBLEM_MDP else graph.n // 2

    def init(self, initial=None) -> None:
        arr = None if initial is None else np.ascontiguousarray(initial, dtype=np.int32)
        C.check(C.lib().ts_solver_init(self._h, C.ptr(arr)), "ts_solver_init")

    def set_perturbations(self, draws) -> None:
        """MaxBS: use the caller's perturbation events (rows of k move indices)."""
        d = np.ascontiguousarray(draws, dtype=np.int64)
        n_events = d.shape[0] if d.ndim == 2 else (len(d) // max(1, self._k()))
        C.check(C.lib().ts_solver_set_perturbations(self._h, C.ptr(d.reshape(-1)), n_events),
                "ts_solver_set_perturbations")

    def _k(self) -> int:
        return max(1, min(self.params.gamma, self.n) // 2)

    def step(self, k: int) -> int:
        done = ctypes.c_int64(0)
        C.check(C.lib().ts_solver_step(self._h, int(k), ctypes.byref(done)), "ts_solver_step")
        return int(done.value)

    def prepare(self, k: int) -> int:
        adm = ctypes.c_int64(0)
        C.check(C.lib().ts_solver_prepare(self._h, int(k), ctypes.byref(adm)), "ts_solver_prepare")
        return int(adm.value)

    def enqueue(self, k: int) -> None:
        C.check(C.lib().ts_solver_enqueue(self._h, int(k)), "ts_solver_enqueue")

    def sync(self) -> int:
        it = ctypes.c_int64(0)
        C.check(C.lib().ts_solver_sync(self._h, ctypes.byref(it)), "ts_solver_sync")
        return int(it.value)

    def result(self) -> SolveResult:
        r = C.Result()
        best = np.zeros(self.m if self.problem == C.PROBLEM_MDP else self.n, np.int32)
        C.check(C.lib().ts_solver_result(self._h, ctypes.byref(r), C.ptr(best)), "ts_solver_result")
        return SolveResult(r.iterations, r.evaluations, r.cur, r.best, r.best_true,
                           r.perturbations, bool(r.stopped), best, r.device_error)

    def state(self):
        n = self.n
        sol, pos, tab = (np.zeros(n, np.int32) for _ in range(3))
        vg = np.zeros(n, np.int64)
        C.check(C.lib().ts_solver_state(self._h, C.ptr(sol), C.ptr(pos), C.ptr(tab), C.ptr(vg)),
                "ts_solver_state")
        return sol, pos, tab, vg

    def info(self) -> C.SolverInfo:
        """Launch geometry and element widths of the iteration kernel."""
        out = C.SolverInfo()
        C.check(C.lib().ts_solver_info_get(self._h, ctypes.byref(out)), "ts_solver_info_get")
        return out

    def trace(self) -> np.ndarray:
        cnt = ctypes.c_int64(0)
        C.check(C.lib().ts_solver_trace(self._h, None, 0, ctypes.byref(cnt)), "ts_solver_trace")
        out = np.zeros(cnt.value, dtype=C.TRACE_DTYPE)
        got = ctypes.c_int64(0)
        C.check(C.lib().ts_solver_trace(self._h, C.ptr(out), len(out), ctypes.byref(got)),
                "ts_solver_trace")
        return out

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            C.lib().ts_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def random_start(problem: int, n: int, m: int, seed: int) -> np.ndarray:
    """The reference's seeded random start (host only, no GPU)."""
    out = np.zeros(m if problem == C.PROBLEM_MDP else n, np.int32)
    C.check(C.lib().ts_random_start(problem, n, m, seed & 0xFFFFFFFF, C.ptr(out)), "ts_random_start")
    return out


def perturb_draws(n: int, seed: int, gamma: int, init_random: bool, n_events: int) -> np.ndarray:
    """MaxBS perturbation move indices, one row per event (host only)."""
    k = max(1, min(gamma, n) // 2)
    out = np.zeros(n_events * k, np.int64)
    C.check(C.lib().ts_perturb_draws(n, seed & 0xFFFFFFFF, gamma, int(init_random), n_events,
                                     C.ptr(out)), "ts_perturb_draws")
    return out.reshape(n_events, k)


def tabu_search(graph: Graph, sol, *, m: int | None = None, max_iter: int = 50000,
                tenure_policy: int = C.TENURE_REF, tenure: int = 15) -> SolveResult:
    """MDP tabu search from the selected set ``sol`` (GPU-MDP-CSR.cu:611-693)."""
    sol = np.asarray(sol, dtype=np.int32)
    s = Solver(graph, C.PROBLEM_MDP, m=len(sol) if m is None else m, max_iter=max_iter,
               tenure_policy=tenure_policy, tenure=tenure)
    try:
        s.init(sol)
        s.step(max_iter)
        return s.result()
    finally:
        s.close()


def perturbation_based_tabu_search(graph: Graph, part, piter: int, max_iter: int, gamma: int,
                                   maxt: int, *, seed: int = 1, tenure_policy: int = C.TENURE_REF,
                                   tenure: int = 25) -> SolveResult:
    """Max Bisection tabu search with perturbation (GPU-MAXBS-CSR.cu:401-512).

    ``part`` is the 0/1 side of every vertex (part 0 holds floor(n/2)); the
    perturbation stream is mt19937(seed)."""
    s = Solver(graph, C.PROBLEM_MAXBS, max_iter=max_iter, piter=piter, gamma=gamma, maxt=maxt,
               seed=seed, tenure_policy=tenure_policy, tenure=tenure)
    try:
        s.init(np.asarray(part, dtype=np.int32))
        s.step(max_iter)
        return s.result()
    finally:
        s.close()


@dataclass
class BatchJobSpec:
    """One solve of a batch: graph, problem parameters and start (None: seeded random)."""
    graph: Graph
    problem: int
    m: int = 0
    max_iter: int = 50000
    tenure_policy: int = C.TENURE_REF
    tenure: int = 15
    maxt: int = 200
    piter: int = 500
    gamma: int = 150
    seed: int = 1
    initial: np.ndarray | None = None
    cluster: int = 0  # CTAs per solve: 0 auto, 1, 2, 4 or 8
    sweep: int = C.PASS_AUTO  # ts_pass


class Batch:
    """Many independent solves in one persistent launch, captured as a CUDA graph.

    Each solve gives the result ``Solver(...).init(initial); step(max_iter)``
    gives for the same graph and parameters (ts_batch_create)."""

    def __init__(self, jobs, *, max_bytes: int = 0, max_slots: int = 0, stream=None):
        jobs = list(jobs)
        if not jobs:
            raise ValueError("a batch needs at least one job")
        arr = (C.BatchJob * len(jobs))()
        keep = []  # start arrays must live until create returns
        self.sizes = []
        for q, j in enumerate(jobs):
            p = default_params(j.problem)
            p.m = j.m
            p.max_iter = j.max_iter
            p.tenure_policy = j.tenure_policy
            p.tenure = j.tenure
            p.maxt = j.maxt
            p.piter = j.piter
            p.gamma = j.gamma
            p.seed = j.seed & 0xFFFFFFFF
            p.pass_ = int(j.sweep)
            arr[q].graph = j.graph.handle.value
            arr[q].params = p
            init = None if j.initial is None else np.ascontiguousarray(j.initial, dtype=np.int32)
            keep.append(init)
            arr[q].initial = None if init is None else init.ctypes.data
            arr[q].cluster = j.cluster
            self.sizes.append(j.m if j.problem == C.PROBLEM_MDP else j.graph.n)
        self.jobs = jobs
        opts = C.BatchOpts()
        opts.max_bytes = max_bytes
        opts.max_slots = max_slots
        h = ctypes.c_void_p()
        st = None if stream is None else ctypes.c_void_p(int(stream))
        C.check(C.lib().ts_batch_create(arr, len(jobs), ctypes.byref(opts), st, ctypes.byref(h)),
                "ts_batch_create")
        self._h = h
        del keep

    def info(self) -> C.BatchInfo:
        out = C.BatchInfo()
        C.check(C.lib().ts_batch_info_get(self._h, ctypes.byref(out)), "ts_batch_info_get")
        return out

    def launch(self) -> None:
        C.check(C.lib().ts_batch_launch(self._h), "ts_batch_launch")

    def sync(self) -> None:
        C.check(C.lib().ts_batch_sync(self._h), "ts_batch_sync")

    def results(self, best_solutions: bool = True) -> list[SolveResult]:
        n = len(self.jobs)
        res = (C.Result * n)()
        words = int(sum(self.sizes))
        best = np.zeros(max(1, words), np.int32) if best_solutions else None
        C.check(C.lib().ts_batch_results(self._h, res, C.ptr(best)), "ts_batch_results")
        out, off = [], 0
        for q in range(n):
            r = res[q]
            sol = best[off:off + self.sizes[q]].copy() if best_solutions else None
            off += self.sizes[q]
            out.append(SolveResult(r.iterations, r.evaluations, r.cur, r.best, r.best_true,
                                   r.perturbations, bool(r.stopped), sol, r.device_error))
        return out

    def run(self) -> list[SolveResult]:
        self.launch()
        self.sync()
        return self.results()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            C.lib().ts_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_solve(jobs, **kw) -> list[SolveResult]:
    """Runs every job once in one batch and returns their results in job order."""
    b = Batch(jobs, **kw)
    try:
        return b.run()
    finally:
        b.close()


@dataclass
class Served:
    """A completed request: its result, best solution and server-clock times (s)."""
    ticket: int
    status: int
    executor: str
    kind: int
    result: SolveResult | None
    submit_s: float
    admit_s: float
    done_s: float
    footprint_bytes: int

    @property
    def latency_s(self) -> float:
        return self.done_s - self.submit_s


class Server:
    """Request loop with continuous batching (ts_server_*).

    ``submit`` copies the request's edge list and returns a ticket; ``poll``
    returns completed requests.  Each result equals the plain solver's on the
    same graph and parameters."""

    def __init__(self, *, max_bytes: int = 0, round_ms: float = 0.0, plain_min_pairs: int = 0):
        o = C.ServerOpts()
        o.max_bytes = max_bytes
        o.round_ms = round_ms
        o.plain_min_pairs = plain_min_pairs
        h = ctypes.c_void_p()
        C.check(C.lib().ts_server_create(ctypes.byref(o), ctypes.byref(h)), "ts_server_create")
        self._h = h
        self._pending = {}  # ticket -> (best array, problem)

    def submit(self, n: int, u, v, w, problem: int, *, kind=-1, drop_self_loops=None, m: int = 0,
               max_iter: int = 1000, tenure_policy: int = C.TENURE_FIXED, tenure: int = 20,
               maxt: int = 200, piter: int = 500, gamma: int = 150, seed: int = 1, initial=None) -> int:
        u = np.ascontiguousarray(u, dtype=np.int32)
        v = np.ascontiguousarray(v, dtype=np.int32)
        w = np.ascontiguousarray(w, dtype=np.int32)
        p = default_params(problem)
        p.m = m
        p.max_iter = max_iter
        p.tenure_policy = tenure_policy
        p.tenure = tenure
        p.maxt = maxt
        p.piter = piter
        p.gamma = gamma
        p.seed = seed & 0xFFFFFFFF
        q = C.Request()
        q.n = n
        q.num_edges = len(u)
        q.u, q.v, q.w = u.ctypes.data, v.ctypes.data, w.ctypes.data
        q.kind = -1 if kind is None or kind == -1 else struct_id(kind)
        q.drop_self_loops = int(problem == C.PROBLEM_MDP) if drop_self_loops is None else int(drop_self_loops)
        q.params = p
        init = None if initial is None else np.ascontiguousarray(initial, dtype=np.int32)
        q.initial = None if init is None else init.ctypes.data
        best = np.zeros(m if problem == C.PROBLEM_MDP else n, np.int32)
        q.best_sol = best.ctypes.data
        t = ctypes.c_int64(0)
        C.check(C.lib().ts_server_submit(self._h, ctypes.byref(q), ctypes.byref(t)), "ts_server_submit")
        self._pending[t.value] = best
        return t.value

    def poll(self, wait_ms: int = 0, cap: int = 256) -> list[Served]:
        buf = (C.Served * cap)()
        got = ctypes.c_int32(0)
        C.check(C.lib().ts_server_poll(self._h, buf, cap, ctypes.byref(got), int(wait_ms)), "ts_server_poll")
        out = []
        for k in range(got.value):
            d = buf[k]
            best = self._pending.pop(d.ticket, None)
            r = d.result
            res = None
            if d.status == C.OK:
                res = SolveResult(r.iterations, r.evaluations, r.cur, r.best, r.best_true, r.perturbations,
                                  bool(r.stopped), best, r.device_error)
            out.append(Served(d.ticket, d.status, "plain" if d.executor else "packed", d.kind, res,
                              d.submit_s, d.admit_s, d.done_s, d.footprint_bytes))
        return out

    def now(self) -> float:
        return C.lib().ts_server_now(self._h)

    def stats(self) -> C.ServerStats:
        s = C.ServerStats()
        C.check(C.lib().ts_server_stats_get(self._h, ctypes.byref(s)), "ts_server_stats_get")
        return s

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            C.lib().ts_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
