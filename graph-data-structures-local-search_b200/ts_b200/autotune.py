"""Size-bucket autotuner for the batched form.

For every (problem, size bucket) it times short batches of a representative
instance on each candidate lookup structure, cluster size (CTAs per solve)
and pair sweep (the tile pass: 32 rows per tile, one structure query per
column; or the per-row pass: a few rows per tile, one lookup per pair) and
keeps the fastest, measured as swap pairs evaluated per second of device
time.  Results do not depend on the choice -- every structure, cluster size
and sweep gives the same trajectory -- so the table only decides speed.
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
    sweep: int = C.PASS_AUTO


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

    def pick_sweep(self, problem: int, n: int) -> int:
        c = self.choice.get((problem, self.bucket_of(n)))
        return C.PASS_AUTO if c is None else c.sweep

    def as_dict(self) -> dict:
        out = {}
        for (p, b), c in sorted(self.choice.items()):
            lo, hi = self.buckets[b]
            out[f"{'mdp' if p == C.PROBLEM_MDP else 'maxbs'} n in [{lo},{hi})"] = {
                "structure": c.kind, "cluster": c.cluster, "pairs_per_s": c.pairs_per_s,
                "sweep": {C.PASS_AUTO: "auto", C.PASS_TILE: "tile", C.PASS_ROWS: "rows"}[c.sweep]}
        return out


def _trial(problem: int, n: int, kind: str, cluster: int, jobs: int, iters: int, seed: int,
           sweep: int = C.PASS_AUTO) -> float:
    u, v, w, _ = gen.erdos_renyi(n, min(25.0, n - 1.0), seed)
    g = Graph(n, u, v, w, kind, drop_self_loops=problem == C.PROBLEM_MDP)
    m = max(1, n // 8) if problem == C.PROBLEM_MDP else n // 2
    specs = [BatchJobSpec(g, problem, m=m, max_iter=iters, tenure_policy=C.TENURE_FIXED,
                          tenure=20 if problem == C.PROBLEM_MDP else 50, seed=s + 1, cluster=cluster,
                          sweep=sweep)
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


def autotune(buckets=DEFAULT_BUCKETS, kinds=("csr", "wswap", "csr-bb", "hash"), clusters=(1, 2, 4),
             sweeps=(C.PASS_TILE, C.PASS_ROWS), jobs: int = 296, iters: int = 60, seed: int = 123,
             budget_s: float = 60.0) -> Table:
    """Times every candidate on the geometric middle of each bucket; each
    (problem, bucket) gets an equal share of `budget_s`, after which it keeps
    the best candidate timed so far."""
    table = Table(buckets)
    share = budget_s / (2 * len(buckets))
    for problem in (C.PROBLEM_MDP, C.PROBLEM_MAXBS):
        for b, (lo, hi) in enumerate(buckets):
            n = int(np.sqrt(lo * (hi - 1)))
            best = None
            t_start = time.perf_counter()
            budget = share
            for kind in kinds:
                if kind == "wswap" and problem == C.PROBLEM_MAXBS and n > 8000:
                    continue  # n^2/4 int32 matrix per solve
                for cs in clusters:
                    for sw in sweeps:
                        if kind == "wswap" and sw == C.PASS_TILE:
                            continue  # the matrix has one sweep
                        if time.perf_counter() - t_start > budget and best is not None:
                            break
                        try:
                            rate = _trial(problem, n, kind, cs, jobs, iters, seed + b, sw)
                        except C.TsError as e:  # this shape does not fit the device: not a candidate
                            table.trials.append({"problem": problem, "n": n, "structure": kind, "cluster": cs,
                                                 "sweep": sw, "unavailable": str(e)})
                            continue
                        table.trials.append({"problem": problem, "n": n, "structure": kind, "cluster": cs,
                                             "sweep": sw, "pairs_per_s": rate})
                        if best is None or rate > best.pairs_per_s:
                            best = Choice(kind, cs, rate, sw)
            table.choice[(problem, b)] = best
    return table
