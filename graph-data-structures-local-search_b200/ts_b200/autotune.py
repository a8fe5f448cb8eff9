"""Size-bucket autotuner for the batched form.

For every (problem, size bucket) it times short batches of a representative
instance on each candidate lookup structure and cluster size (CTAs per solve)
and keeps the fastest, measured as swap pairs evaluated per second of device
time.  Results do not depend on the choice -- every structure and cluster size
gives the same trajectory -- so the table only decides speed.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import _capi as C
from . import gen
from .engine import Batch, BatchJobSpec, Graph

DEFAULT_BUCKETS = ((200, 600), (600, 2000), (2000, 6000), (6000, 20001))


@dataclass
class Choice:
    kind: str
    cluster: int
    pairs_per_s: float


class Table:
    """(problem, n) -> (structure, cluster size)."""

    def __init__(self, buckets=DEFAULT_BUCKETS):
        self.buckets = tuple(buckets)
        self.choice: dict[tuple[int, int], Choice] = {}
        self.trials: list[dict] = []

    def bucket_of(self, n: int) -> int:
        for b, (lo, hi) in enumerate(self.buckets):
            if lo <= n < hi:
                return b
        return len(self.buckets) - 1 if n >= self.buckets[-1][0] else 0

    def pick(self, problem: int, n: int) -> tuple[str, int]:
        c = self.choice.get((problem, self.bucket_of(n)))
        return ("csr", 0) if c is None else (c.kind, c.cluster)

    def as_dict(self) -> dict:
        out = {}
        for (p, b), c in sorted(self.choice.items()):
            lo, hi = self.buckets[b]
            out[f"{'mdp' if p == C.PROBLEM_MDP else 'maxbs'} n in [{lo},{hi})"] = {
                "structure": c.kind, "cluster": c.cluster, "pairs_per_s": c.pairs_per_s}
        return out


def _trial(problem: int, n: int, kind: str, cluster: int, jobs: int, iters: int, seed: int) -> float:
    u, v, w, _ = gen.erdos_renyi(n, min(25.0, n - 1.0), seed)
    g = Graph(n, u, v, w, kind, drop_self_loops=problem == C.PROBLEM_MDP)
    m = max(1, n // 8) if problem == C.PROBLEM_MDP else n // 2
    specs = [BatchJobSpec(g, problem, m=m, max_iter=iters, tenure_policy=C.TENURE_FIXED,
                          tenure=20 if problem == C.PROBLEM_MDP else 50, seed=s + 1, cluster=cluster)
             for s in range(jobs)]
    try:
        b = Batch(specs, max_bytes=8 << 30)
        try:
            b.launch()
            b.sync()
            t0 = time.perf_counter()
            b.launch()
            b.sync()
            dt = time.perf_counter() - t0
            res = b.results(best_solutions=False)
        finally:
            b.close()
    finally:
        g.close()
    return sum(m * (n - m) * r.iterations for r in res) / dt


def autotune(buckets=DEFAULT_BUCKETS, kinds=("csr", "wswap", "csr-bb"), clusters=(1, 2, 4),
             jobs: int = 296, iters: int = 60, seed: int = 123, budget_s: float = 60.0) -> Table:
    """Times every candidate on the geometric middle of each bucket; stops
    exploring (keeping the best so far) once `budget_s` is spent."""
    t_start = time.perf_counter()
    table = Table(buckets)
    for problem in (C.PROBLEM_MDP, C.PROBLEM_MAXBS):
        for b, (lo, hi) in enumerate(buckets):
            n = int(np.sqrt(lo * (hi - 1)))
            best = None
            for kind in kinds:
                if kind == "wswap" and problem == C.PROBLEM_MAXBS and n > 8000:
                    continue  # n^2/4 int32 matrix per solve
                for cs in clusters:
                    if time.perf_counter() - t_start > budget_s and best is not None:
                        break
                    rate = _trial(problem, n, kind, cs, jobs, iters, seed + b)
                    table.trials.append({"problem": problem, "n": n, "structure": kind, "cluster": cs,
                                         "pairs_per_s": rate})
                    if best is None or rate > best.pairs_per_s:
                        best = Choice(kind, cs, rate)
            table.choice[(problem, b)] = best
    return table
