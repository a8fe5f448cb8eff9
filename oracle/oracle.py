"""ctypes view of the CPU oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker and the timed CPU baseline.  The C++ it loads
restates the reference loops (src/mdp/GPU-MDP-CSR.cu:611-693,
src/maxbisection/GPU-MAXBS-CSR.cu:401-512) in exact int64 arithmetic.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libts_oracle.so")
_lib = None

MDP, MAXBS = 0, 1
TENURE_REF, TENURE_FIXED = 0, 1
INIT_EXPLICIT, INIT_RANDOM = 0, 1
REC_MOVE, REC_BREAK, REC_PERTURB = 0, 1, 2

TRACE_DTYPE = np.dtype([
    ("iter", "<i8"), ("idx", "<i8"), ("key", "<i8"), ("cur", "<i8"), ("best", "<i8"),
    ("kind", "<i4"), ("tenure", "<i4"), ("tenure2", "<i4"), ("pad", "<i4"),
])


class _Params(ctypes.Structure):
    _fields_ = [
        ("problem", ctypes.c_int32), ("m", ctypes.c_int32), ("max_iter", ctypes.c_int64),
        ("tenure_policy", ctypes.c_int32), ("tenure_fixed", ctypes.c_int32),
        ("maxt", ctypes.c_int32), ("piter", ctypes.c_int32), ("gamma", ctypes.c_int32),
        ("seed", ctypes.c_uint32), ("init_mode", ctypes.c_int32), ("threads", ctypes.c_int32),
    ]


class _Result(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int64), ("evaluations", ctypes.c_int64),
        ("cur", ctypes.c_int64), ("best", ctypes.c_int64), ("best_true", ctypes.c_int64),
        ("n_trace", ctypes.c_int64), ("stopped", ctypes.c_int32), ("pad", ctypes.c_int32),
    ]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        L.or_graph_create.restype = P
        L.or_graph_create.argtypes = [ctypes.c_int32, ctypes.c_int64, P, P, P, ctypes.c_int]
        L.or_graph_destroy.argtypes = [P]
        L.or_graph_num_entries.restype = ctypes.c_int64
        L.or_graph_num_entries.argtypes = [P]
        L.or_lookup.restype = ctypes.c_int32
        L.or_lookup.argtypes = [P, ctypes.c_int32, ctypes.c_int32]
        L.or_mdp_random_initial.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32, P]
        L.or_maxbs_random_partition.argtypes = [ctypes.c_int32, ctypes.c_uint32, P]
        L.or_run.restype = ctypes.c_int
        L.or_run.argtypes = [P, ctypes.POINTER(_Params), P, ctypes.POINTER(_Result), P,
                             ctypes.c_int64, P, P, P, P, P]
        L.or_mdp_tenure.restype = ctypes.c_int32
        L.or_mdp_tenure.argtypes = [ctypes.c_int64]
        L.or_mdp_c2.restype = ctypes.c_int32
        L.or_mdp_c2.argtypes = [ctypes.c_int32]
        L.or_maxbs_tenure.restype = ctypes.c_int32
        L.or_maxbs_tenure.argtypes = [ctypes.c_int64, ctypes.c_int32]
        L.or_round_f32.restype = ctypes.c_int64
        L.or_round_f32.argtypes = [ctypes.c_int64]
        L.or_maxbs_penalty.restype = ctypes.c_int64
        L.or_maxbs_penalty.argtypes = [ctypes.c_int64]
        L.or_maxbs_perturb_draws.argtypes = [ctypes.c_int32, ctypes.c_uint32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, P]
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Graph:
    """CSR of an undirected edge list, with the reference loaders' rules."""

    def __init__(self, n: int, u, v, w, drop_self_loops: bool):
        self.n = int(n)
        self._u = np.ascontiguousarray(u, dtype=np.int32)
        self._v = np.ascontiguousarray(v, dtype=np.int32)
        self._w = np.ascontiguousarray(w, dtype=np.int32)
        h = lib().or_graph_create(self.n, len(self._u), _ptr(self._u), _ptr(self._v),
                                  _ptr(self._w), int(drop_self_loops))
        if not h:
            raise ValueError("oracle: invalid edge list")
        self._h = ctypes.c_void_p(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.or_graph_destroy(h)
            self._h = None

    def lookup(self, a: int, b: int) -> int:
        return int(lib().or_lookup(self._h, a, b))


@dataclass
class RunResult:
    iterations: int
    evaluations: int
    cur: int
    best: int
    best_true: int
    stopped: bool
    trace: np.ndarray
    sol: np.ndarray
    pos: np.ndarray
    tab: np.ndarray
    vg: np.ndarray
    best_sol: np.ndarray


def run(graph: Graph, problem: int, *, m: int = 0, max_iter: int, tenure_policy=TENURE_FIXED,
        tenure: int = 20, maxt: int = 200, piter: int = 500, gamma: int = 150, seed: int = 1,
        initial=None, threads: int = 1, trace_cap: int | None = None) -> RunResult:
    n = graph.n
    p = _Params()
    p.problem = problem
    p.m = m if problem == MDP else n // 2
    p.max_iter = max_iter
    p.tenure_policy = tenure_policy
    p.tenure_fixed = tenure
    p.maxt = maxt
    p.piter = piter
    p.gamma = gamma
    p.seed = seed & 0xFFFFFFFF
    p.init_mode = INIT_RANDOM if initial is None else INIT_EXPLICIT
    p.threads = threads
    init = None if initial is None else np.ascontiguousarray(initial, dtype=np.int32)
    if trace_cap is None:
        npert = max(1, min(gamma, n) // 2)
        trace_cap = max_iter + 1 + (0 if problem == MDP else (max_iter // max(piter, 1) + 1) * npert)
    trace = np.zeros(trace_cap, dtype=TRACE_DTYPE)
    mm = p.m
    sol = np.zeros(n, np.int32)
    pos = np.zeros(n, np.int32)
    tab = np.zeros(n, np.int32)
    vg = np.zeros(n, np.int64)
    best_sol = np.zeros(mm if problem == MDP else n, np.int32)
    r = _Result()
    rc = lib().or_run(graph._h, ctypes.byref(p), _ptr(init), ctypes.byref(r), _ptr(trace),
                      trace_cap, _ptr(sol), _ptr(pos), _ptr(tab), _ptr(vg), _ptr(best_sol))
    if rc != 0:
        raise ValueError(f"oracle: or_run failed ({rc})")
    return RunResult(r.iterations, r.evaluations, r.cur, r.best, r.best_true, bool(r.stopped),
                     trace[:min(r.n_trace, trace_cap)].copy(), sol, pos, tab, vg, best_sol)


def sweep_sample(graph: Graph, problem: int, *, m: int = 0, rows: int, sweeps: int = 1,
                 seed: int = 1, threads: int = 0, initial=None):
    """Times `sweeps` argmax sweeps over the first `rows` inside positions of the
    start state (a bounded sample of one iteration's pair evaluation).
    Returns (seconds, pairs, key, idx)."""
    L = lib()
    if not hasattr(L, "_sample_bound"):
        L.or_sweep_sample.restype = ctypes.c_double
        L.or_sweep_sample.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Params), ctypes.c_void_p,
                                      ctypes.c_int32, ctypes.c_int32,
                                      ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int64)]
        L._sample_bound = True
    p = _Params()
    p.problem = problem
    p.m = m if problem == MDP else graph.n // 2
    p.max_iter = 1
    p.tenure_policy = TENURE_FIXED
    p.tenure_fixed = 1
    p.maxt = 200
    p.piter = 500
    p.gamma = 150
    p.seed = seed & 0xFFFFFFFF
    p.init_mode = INIT_RANDOM if initial is None else INIT_EXPLICIT
    p.threads = threads
    init = None if initial is None else np.ascontiguousarray(initial, dtype=np.int32)
    pairs, key, idx = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
    t = L.or_sweep_sample(graph._h, ctypes.byref(p), _ptr(init), rows, sweeps, ctypes.byref(pairs),
                          ctypes.byref(key), ctypes.byref(idx))
    if t < 0:
        raise ValueError("oracle: sweep_sample failed")
    return float(t), int(pairs.value), int(key.value), int(idx.value)


def max_threads() -> int:
    return os.cpu_count() or 1


def mdp_random_initial(n: int, m: int, seed: int) -> np.ndarray:
    out = np.zeros(m, np.int32)
    lib().or_mdp_random_initial(n, m, seed & 0xFFFFFFFF, _ptr(out))
    return out


def maxbs_random_partition(n: int, seed: int) -> np.ndarray:
    out = np.zeros(n, np.int32)
    lib().or_maxbs_random_partition(n, seed & 0xFFFFFFFF, _ptr(out))
    return out


def maxbs_perturb_draws(n: int, seed: int, init_random: bool, n_events: int, k: int) -> np.ndarray:
    out = np.zeros(n_events * k, np.int64)
    lib().or_maxbs_perturb_draws(n, seed & 0xFFFFFFFF, int(init_random), n_events, k, _ptr(out))
    return out.reshape(n_events, k)


def mdp_tenure(it: int) -> int:
    return int(lib().or_mdp_tenure(it))


def mdp_c2(c1: int) -> int:
    return int(lib().or_mdp_c2(c1))


def maxbs_tenure(it: int, maxt: int) -> int:
    return int(lib().or_maxbs_tenure(it, maxt))


def round_f32(x: int) -> int:
    return int(lib().or_round_f32(x))


def maxbs_penalty(g: int) -> int:
    return int(lib().or_maxbs_penalty(g))
